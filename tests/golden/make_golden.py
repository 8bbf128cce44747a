"""Generate the golden fixtures from the reference itself.

Runs the reference's own CPU path (bindex.cpp compiled unmodified from the
reference source tree and driven by oracle/ref_harness.cpp; build it with
`make -C oracle ref REF=<reference dir>`) on seeded columns and scan_cmd
texts, and records per query:
  * the scalar-filter hit count and the sha256 of its bitmap (raw_scan +
    AND merge, bindex.cpp:1851-1957) -- the authority;
  * the BinDex hit count, its bitmap hash and whether it equals the scalar
    filter (bindex_scan_*, bindex.cpp:1365-1691).
The data is regenerated by tests from (kind, seed) with rtscan_b200.datagen;
a sha256 of each generated column is stored so generator drift is caught.

    python tests/golden/make_golden.py [--out tests/golden/golden.json]

Only needs to run where the reference tree and the harness exist; the JSON
it writes is committed and read by the tests on any machine.
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from rtscan_b200 import datagen as D  # noqa: E402

N = 1 << 20           # compile-time row count of the harness (DATA_N)
N_ODD = 1_000_003     # a row count that is not a multiple of 32
N_C1 = 1 << 24        # the plain single-column scan at its own size


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<u4").tobytes()).hexdigest()


def masked(bm: np.ndarray, n: int) -> np.ndarray:
    bm = bm.copy()
    rem = n & 31
    if rem:
        bm[n >> 5] &= np.uint32((0xFFFFFFFF << (32 - rem)) & 0xFFFFFFFF)
    return bm


def sweep_lt(ncols, thresholds):
    lines = []
    for t in thresholds:
        lines += [f"lt {t}"] * ncols
    return lines


def cases():
    """(name, n, [(kind, seed)...], scan_cmd lines)"""
    out = []
    u32 = [1] + [int(i * 0xFFFFFFFF / 10) for i in range(1, 10)] + [0xFFFFFFFF]
    # uniform 2^32 sweeps for 1..4 columns (the shape of test/scan_cmd_32_{1..4}c.txt)
    for nc in (1, 2, 3, 4):
        out.append((f"uniform32_sweep_{nc}c", N, [("uniform", 100 + c) for c in range(nc)], sweep_lt(nc, u32)))
    # small domains, 3 columns (test/scan_cmd_2p6.txt, scan_cmd_2p8.txt shapes)
    out.append(("uniform2p6_sweep_3c", N, [("uniform2p6", 200 + c) for c in range(3)],
                sweep_lt(3, [0, 7, 13, 19, 26, 33, 39, 45, 51, 58, 64])))
    out.append(("uniform2p8_sweep_3c", N, [("uniform2p8", 210 + c) for c in range(3)],
                sweep_lt(3, [0, 25, 51, 75, 101, 127, 153, 177, 203, 229, 256])))
    # skewed columns at ~90% (test/zipf1.*.txt, normal.txt shapes), thresholds from the data
    for kind, seed in (("zipf1.1", 300), ("zipf1.3", 310), ("zipf1.5", 320), ("normal", 330)):
        cols = [D.column(kind, N, seed + c) for c in range(3)]
        ths = [int(np.sort(c)[int(0.9 * N)]) for c in cols]
        lines = [f"lt {t}" for t in ths]
        # plus a few two-sided and point predicates per column
        rng = np.random.default_rng(seed)
        for _ in range(6):
            ln = []
            for c in cols:
                a, b = sorted(int(x) for x in rng.choice(c, 2))
                op = rng.integers(0, 5)
                ln.append([f"bt {a} {b + 1}", f"ge {a}", f"gt {a}", f"le {b}", f"eq {a}"][op])
            lines += ln
        out.append((f"{kind}_3c", N, [(kind, seed + c) for c in range(3)], lines))
    # every operator on one uniform column, including the domain edges
    col = D.uniform(N, 400)
    s = np.sort(col)
    lines = []
    for t in (0, 1, int(s[0]), int(s[1000]), int(s[N // 2]), int(s[-1]), 0xFFFFFFFE, 0xFFFFFFFF):
        for op in ("lt", "le", "gt", "ge"):
            lines.append(f"{op} {t}")
    for i in (10, 5000, N // 3, N - 10):
        lines.append(f"eq {int(s[i])}")
    rng = np.random.default_rng(1)
    for _ in range(12):
        a, b = sorted(int(x) for x in rng.integers(0, 1 << 32, size=2))
        lines.append(f"bt {a} {b}")
        lines.append(f"bt {b} {a}")
    out.append(("uniform32_ops_1c", N, [("uniform", 400)], lines))
    # a row count that is not a multiple of 32
    lines = []
    col = D.uniform(N_ODD, 500, 1000)
    for t in (0, 1, 499, 999, 1000):
        lines += [f"lt {t}", f"ge {t}"]
    lines += ["bt 100 900", "eq 7", "le 0"]
    out.append(("uniform1000_odd_1c", N_ODD, [("uniform1000", 500)], lines))
    # the plain single-column scan at its own size: 2^24 rows uniform on
    # [0, 2^32) from default_rng(42), the 10 % range [q45, q55] of the data
    # written as the reference's exclusive `bt` (1,677,722 rows), plus one
    # 10 % range at each end of the domain
    out.append(("c1_uniform32_2p24_1c", N_C1, [("uniform", 42)],
                ["bt 1932185501 2361592940", "lt 429496730", "ge 3865470566"]))
    return out


def column(kind, n, seed):
    if kind == "uniform1000":
        return D.uniform(n, seed, 1000)
    return D.column(kind, n, seed)


def run_case(harness_dir, name, n, specs, lines):
    cols = [column(k, n, s) for k, s in specs]
    ncols = len(cols)
    binary = os.path.join(harness_dir, f"ref_bindex_{n}")
    if not os.access(binary, os.X_OK):
        raise SystemExit(f"missing {binary}: make -C oracle ref REF=<reference> REF_NS='{N} {N_ODD} {N_C1}'")
    with tempfile.TemporaryDirectory() as td:
        data = os.path.join(td, "cols.bin")
        D.write_columns(data, cols)
        cmd = os.path.join(td, "cmd.txt")
        with open(cmd, "w") as f:
            f.write("\n".join(lines) + "\nexit\n")
        r = subprocess.run([binary, "-f", data, "-b", str(ncols), "-p", cmd, "-o", td], capture_output=True,
                           text=True, timeout=3600)
        if r.returncode != 0:
            raise SystemExit(f"{name}: harness failed ({r.returncode}): {r.stderr[-400:]}")
        qlines = [l.split() for l in r.stdout.splitlines() if l.startswith("query ")]
        queries = []
        for i, ql in enumerate(qlines):
            bidx = np.fromfile(os.path.join(td, f"q{i:05d}_bindex.bin"), dtype="<u4")
            raw = np.fromfile(os.path.join(td, f"q{i:05d}_raw.bin"), dtype="<u4")
            queries.append({
                "lines": lines[i * ncols:(i + 1) * ncols],
                "raw_hits": int(ql[5]), "raw_sha": sha(masked(raw, n)),
                "bindex_hits": int(ql[3]), "bindex_sha": sha(masked(bidx, n)),
                "bindex_equal": ql[7] == "1",
            })
    return {"name": name, "n": n, "columns": [{"kind": k, "seed": s, "sha": sha(column(k, n, s))} for k, s in specs],
            "queries": queries}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--harness", default=os.path.join(ROOT, "oracle", "_ref"))
    ap.add_argument("--out", default=os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden.json"))
    a = ap.parse_args()
    out = {"generator": "tests/golden/make_golden.py", "reference": "AntaresAlice/RTScan bindex.cpp (VAREA_N=128)",
           "cases": []}
    for name, n, specs, lines in cases():
        c = run_case(a.harness, name, n, specs, lines)
        bad = sum(not q["bindex_equal"] for q in c["queries"])
        print(f"{name}: {len(c['queries'])} queries, {bad} where the reference BinDex differs from its scalar filter",
              flush=True)
        out["cases"].append(c)
    with open(a.out, "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
