"""The drop-in CLI rejects bad arguments before it touches a device (exit
status 2 for usage errors, 1 for a scan_cmd file it cannot read), so these
run on the CPU."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "rtscan_b200", "rtscan_b200_cli")


def run(*args, cwd=None):
    if not os.path.exists(CLI):
        pytest.skip("the CLI is not built")
    return subprocess.run([CLI, *args], capture_output=True, text=True, timeout=60, cwd=cwd)


def test_help():
    r = run("-h")
    assert r.returncode == 0 and "Usage:" in r.stdout and "-m auto|scan|bindex|batch" in r.stdout


@pytest.mark.parametrize("args,code,msg", [
    ((), 2, "need -f <column-file> and -b <ncols>"),
    (("-f", "cols.bin"), 1, "Fail to open scan_cmd file test/scan_cmd.txt"),  # one column, the default file
    (("-f", "cols.bin", "-b", "0"), 2, "need -f <column-file> and -b <ncols>"),
    (("-f", "cols.bin", "-b", "2", "-m", "fast"), 2, "unknown mode fast"),
    (("-f", "cols.bin", "-b", "2", "-y", "0"), 2, "-y 0 needs -q <queries>"),
    (("-f", "cols.bin", "-b", "2", "-p", "/nonexistent/scan_cmd.txt"), 1, "Fail to open scan_cmd file"),
    (("-z",), 2, "see -h for the options"),
])
def test_argument_errors_before_any_device_work(args, code, msg, tmp_path):
    r = run(*args, cwd=str(tmp_path))
    assert r.returncode == code, (r.returncode, r.stderr)
    assert msg in r.stderr
    assert "[ERROR] open" not in r.stderr  # rejected before opening a device
