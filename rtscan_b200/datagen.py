"""Seeded synthetic columns and queries in the reference's formats.

The reference's generators (tools/generate_uniform_data_n_col.cpp:13-58,
tools/generate_zipf_data.py:10-12, tools/generate_normal_data.py:10-13) are
unseeded; these are seeded (numpy PCG64) so every run and every fixture can
be regenerated bit for bit.  Files use the reference's column layout:
`ncols` columns of `nrows` little-endian uint32, back to back, no header
(getDataFromFile, bindex_cuda.cpp:1269-1286).

Distributions:
  * uniform over [0, domain)                      (domain 2^32, 2^8, 2^6 ...)
  * finite zipf with exponent s over `distinct` values 0..distinct-1, drawn
    by inverse CDF over ranks (the reference draws np.random.zipf % (2^32-1),
    which is unbounded)
  * rounded normal, mean 2^31, sd 2^28, clipped to [0, 2^32-1] (the
    reference uses sd = 1)
"""
from __future__ import annotations

import math
from typing import Dict, List, Sequence, Tuple

import numpy as np

U32_MAX = 0xFFFFFFFF


def uniform(n: int, seed: int, domain: int = 1 << 32) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return rng.integers(0, domain, size=n, dtype=np.uint64).astype(np.uint32)


def zipf(n: int, seed: int, s: float = 1.3, distinct: int = 1 << 20) -> np.ndarray:
    rng = np.random.default_rng(seed)
    ranks = np.arange(1, distinct + 1, dtype=np.float64)
    cdf = np.cumsum(ranks ** (-s))
    cdf /= cdf[-1]
    u = rng.random(n)
    return np.minimum(np.searchsorted(cdf, u, side="right"), distinct - 1).astype(np.uint32)


def normal(n: int, seed: int, mean: float = 2.0 ** 31, sd: float = 2.0 ** 28) -> np.ndarray:
    rng = np.random.default_rng(seed)
    x = np.rint(rng.normal(mean, sd, size=n))
    return np.clip(x, 0, U32_MAX).astype(np.uint32)


def column(kind: str, n: int, seed: int) -> np.ndarray:
    """Named column kinds used by tests and the benchmark."""
    if kind == "uniform":
        return uniform(n, seed)
    if kind.startswith("uniform"):  # uniform2p6, uniform2p8
        return uniform(n, seed, 1 << int(kind.split("2p")[1]))
    if kind.startswith("zipf"):
        return zipf(n, seed, float(kind[4:]))
    if kind == "normal":
        return normal(n, seed)
    raise ValueError(kind)


def write_columns(path: str, cols: Sequence[np.ndarray]) -> None:
    with open(path, "wb") as f:
        for c in cols:
            np.ascontiguousarray(c, dtype="<u4").tofile(f)


def read_columns(path: str, ncols: int, nrows: int) -> List[np.ndarray]:
    a = np.fromfile(path, dtype="<u4", count=ncols * nrows)
    return [a[i * nrows:(i + 1) * nrows].copy() for i in range(ncols)]


def range_for_selectivity(sample_sorted: np.ndarray, sel: float, center: float = 0.5) -> Tuple[int, int]:
    """Inclusive [lo, hi] covering about `sel` of the rows, from sample
    quantiles [q(center - sel/2), q(center + sel/2)]."""
    m = len(sample_sorted)
    a = center - sel / 2
    b = center + sel / 2
    if a < 0.0:  # pushed against an end: keep the width
        a, b = 0.0, min(1.0, sel)
    elif b > 1.0:
        a, b = max(0.0, 1.0 - sel), 1.0
    lo = int(sample_sorted[min(m - 1, int(a * m))])
    hi = int(sample_sorted[min(m - 1, max(0, int(math.ceil(b * m)) - 1))])
    return lo, max(lo, hi)


def sweep_queries(col: np.ndarray, sels: Sequence[float], seed: int = 0) -> List[List[Tuple[int, int, int]]]:
    """One single-column query per selectivity (bounds at sample quantiles)."""
    rng = np.random.default_rng(seed)
    sample = np.sort(col[rng.integers(0, len(col), size=min(len(col), 1 << 20))])
    return [[(0, *range_for_selectivity(sample, s))] for s in sels]


def batch_queries(cols: Sequence[np.ndarray], nq: int, seed: int, min_sel: float = 1e-4, max_sel: float = 0.9,
                  min_cols: int = 1, max_cols: int = 4, per_column_sel: bool = True
                  ) -> List[List[Tuple[int, int, int]]]:
    """Queries touching `min_cols..max_cols` random columns each, with a
    log-uniform target selectivity in [min_sel, max_sel] for the whole query
    (split evenly over its terms when per_column_sel), bounds from sample
    quantiles at a random centre."""
    rng = np.random.default_rng(seed)
    ncols = len(cols)
    samples = []
    for c in cols:
        idx = rng.integers(0, len(c), size=min(len(c), 1 << 18))
        samples.append(np.sort(c[idx]))
    out = []
    for _ in range(nq):
        k = int(rng.integers(min_cols, min(max_cols, ncols) + 1))
        which = sorted(rng.choice(ncols, size=k, replace=False).tolist())
        sel = math.exp(rng.uniform(math.log(min_sel), math.log(max_sel)))
        per = sel ** (1.0 / k) if per_column_sel else sel
        q = []
        for c in which:
            center = rng.uniform(per / 2, 1 - per / 2) if per < 1 else 0.5
            lo, hi = range_for_selectivity(samples[c], per, center)
            q.append((c, lo, hi))
        out.append(q)
    return out


def to_scan_cmd(queries: Sequence[Sequence[Tuple[int, int, int]]], ncols: int) -> str:
    """scan_cmd text for inclusive-range queries: one line per column per
    query, `bt lo-1 hi+1` for two-sided ranges and lt/gt/le/ge/eq where they
    express the range exactly; unconstrained columns get `ge 0`."""
    lines = []
    for q in queries:
        by = {c: (lo, hi) for c, lo, hi in q}
        for c in range(ncols):
            if c not in by:
                lines.append("ge 0")
                continue
            lo, hi = by[c]
            if lo == hi:
                lines.append(f"eq {lo}")
            elif lo == 0:
                lines.append(f"le {hi}")
            elif hi == U32_MAX:
                lines.append(f"ge {lo}")
            else:
                lines.append(f"bt {lo - 1} {hi + 1}")
    lines.append("exit")
    return "\n".join(lines) + "\n"
