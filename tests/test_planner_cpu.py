"""The query planners on the CPU.  tests/planner_check.cu includes the batch
planner's translation unit, plans seeded random batches (1-10 columns,
query counts at every pass-routing edge, three table budgets, empty and
merged terms) on a context without a device, and checks each plan's
routing, mask bits, bucket index and shared-memory fit.
tests/bindex_plan_check.cu checks the BinDex planner's rank windows and its
choice of filter vectors on random sorted columns.  Both are compiled here
with nvcc against the library's other objects (built by
__graft_entry__.build)."""
import glob
import os
import re
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def compile_check(tmp_path_factory, source, replaces):
    """Build tests/<source> with the library's objects except `replaces`
    (the translation unit it includes)."""
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    objs = [o for o in glob.glob(os.path.join(ROOT, "rtscan_b200", "_build", "*.o"))
            if not o.endswith(replaces + ".o")]
    if not os.path.exists(nvcc) or not objs:
        pytest.skip("needs nvcc and the library's objects (run the build first)")
    out = str(tmp_path_factory.mktemp("check") / source.replace(".cu", ""))
    cmd = [nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-O2", "-std=c++17",
           "-I", os.path.join(ROOT, "include"), "--expt-relaxed-constexpr",
           os.path.join(ROOT, "tests", source), *objs, "-lcuda", "-o", out]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-3000:]
    return out


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    return compile_check(tmp_path_factory, "planner_check.cu", "batch.cu")


@pytest.fixture(scope="module")
def bindex_harness(tmp_path_factory):
    return compile_check(tmp_path_factory, "bindex_plan_check.cu", "bindex.cu")


@pytest.mark.parametrize("seed", [1, 2, 3, 4, 5])
def test_planner_invariants(harness, seed):
    r = subprocess.run([harness, str(seed), "30"], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    m = re.search(r"(\d+) kernel queries, (\d+) table passes, (\d+) term-by-term passes, (\d+) mask bits", r.stdout)
    assert m, r.stdout
    queries, tables, few, bits = (int(x) for x in m.groups())
    assert queries > 1000 and tables > 0 and few > 0 and bits > 100_000, r.stdout
    shared = re.search(r"(\d+) plans with shared positions \((\d+) lookups\), (\d+) queries dropped", r.stdout)
    assert shared and int(shared.group(1)) >= 1 and int(shared.group(2)) > 1000, r.stdout
    assert int(shared.group(3)) > 1000, r.stdout  # batch_plan_drop exercised


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_bindex_planner_windows_and_choices(bindex_harness, seed):
    r = subprocess.run([bindex_harness, str(seed), "40"], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    m = re.search(r"(\d+) bounds", r.stdout)
    assert m and int(m.group(1)) >= 8000, r.stdout
