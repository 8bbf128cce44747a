"""The drop-in driver rtscan_b200_cli on a column file and a scan_cmd file:
every plan (-m), the rank-encoded table (-e) and index files (-I) report
the scalar filter's hit count and pass the self-check."""
import os
import re
import subprocess

import numpy as np
import pytest

from oracle import oracle as O
from rtscan_b200 import datagen as D

pytestmark = pytest.mark.gpu
CLI = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "rtscan_b200", "rtscan_b200_cli")


def run_cli(args):
    r = subprocess.run([CLI] + args, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    return r.stdout


@pytest.fixture(scope="module")
def table(tmp_path_factory):
    d = tmp_path_factory.mktemp("cli")
    n = 400_009
    cols = [D.zipf(n, 1, 1.3), D.uniform(n, 2), D.uniform(n, 3, 256)]
    data = str(d / "cols.bin")
    D.write_columns(data, cols)
    qs = D.batch_queries(cols, 12, seed=4, min_cols=1, max_cols=3)
    qs.append([(2, 7, 7)])
    cmd = str(d / "cmd.txt")
    with open(cmd, "w") as f:
        f.write(D.to_scan_cmd(qs, 3))
    want = [int(O.range_scan([cols[c] for c, _, _ in q], [t[1] for t in q], [t[2] for t in q])[1]) for q in qs]
    return d, data, cmd, want


@pytest.mark.parametrize("extra", [["-m", "auto"], ["-m", "scan"], ["-m", "batch"], ["-m", "bindex", "-K", "32"],
                                   ["-m", "scan", "-e"], ["-m", "bindex", "-e"]])
def test_cli_counts_and_check(table, extra):
    d, data, cmd, want = table
    out = run_cli(["-f", data, "-b", "3", "-p", cmd] + extra)
    got = [int(x) for x in re.findall(r"\[RESULT\] query \d+ count (\d+)", out)]
    assert got == want
    checks = re.findall(r"\[CHECK\]hit (\d+)/(\d+)", out)
    assert len(checks) == len(want) and all(a == b for a, b in checks)
    assert "[ERROR]" not in out
    if "-e" in extra:
        assert "[Time] Encode Time" in out


def test_cli_index_files(table):
    d, data, cmd, want = table
    prefix = str(d / "idx")
    first = run_cli(["-f", data, "-b", "3", "-p", cmd, "-m", "bindex", "-I", prefix])
    assert all(os.path.exists(f"{prefix}.{c}.bdx") for c in range(3))
    second = run_cli(["-f", data, "-b", "3", "-p", cmd, "-m", "bindex", "-I", prefix])  # loads the files
    for out in (first, second):
        assert [int(x) for x in re.findall(r"\[RESULT\] query \d+ count (\d+)", out)] == want


def test_cli_query_count_and_generated_queries(table):
    d, data, cmd, want = table
    out = run_cli(["-f", data, "-b", "3", "-p", cmd, "-m", "scan", "-q", "5"])
    assert [int(x) for x in re.findall(r"\[RESULT\] query \d+ count (\d+)", out)] == want[:5]
    assert "[Mem] columns:" in out
    cols = D.read_columns(data, 3, 400_009)
    for g, op in ((1, "lt"), (0, "eq")):
        out = run_cli(["-f", data, "-b", "3", "-y", "0", "-q", "6", "-g", str(g), "-m", "batch"])
        span = 0xFFFFFFFF // 7
        exp = []
        for i in range(6):
            t = (i + 1) * span
            hit = np.ones(len(cols[0]), bool)
            for c in cols:
                hit &= (c < t) if op == "lt" else (c == t)
            exp.append(int(hit.sum()))
        assert [int(x) for x in re.findall(r"\[RESULT\] query \d+ count (\d+)", out)] == exp
