"""Workload generators: bounds from sample quantiles must cover the asked
share of the rows, at any centre, without rounding pushing a range to an
end of the domain."""
import numpy as np
import pytest

from rtscan_b200 import datagen as D


@pytest.fixture(scope="module")
def sample():
    rng = np.random.default_rng(1)
    return np.sort(rng.integers(0, 1 << 32, size=1 << 18, dtype=np.uint64).astype(np.uint32))


@pytest.mark.parametrize("sel", [1e-4, 1e-3, 0.01, 0.1, 0.5, 0.9, 1.0])
@pytest.mark.parametrize("center", [0.5, 0.3, 0.77, 0.0, 1.0])
def test_range_covers_the_asked_share(sample, sel, center):
    lo, hi = D.range_for_selectivity(sample, sel, center)
    assert lo <= hi
    got = ((sample >= lo) & (sample <= hi)).mean()
    assert abs(got - sel) <= max(3.0 / len(sample), 0.02 * sel), (sel, center, lo, hi, got)


def test_range_centre_is_kept_away_from_the_ends(sample):
    """A range not pushed against an end sits around its centre (a rounding
    slip once moved it to the top of the domain)."""
    for center in np.linspace(0.1, 0.9, 81):
        lo, hi = D.range_for_selectivity(sample, 0.001, float(center))
        mid = np.searchsorted(sample, (lo + hi) // 2) / len(sample)
        assert abs(mid - center) < 0.002, (center, lo, hi, mid)


def test_batch_queries_have_the_asked_shape():
    rng = np.random.default_rng(2)
    cols = [rng.integers(0, 1 << 32, size=200_000, dtype=np.uint64).astype(np.uint32) for _ in range(4)]
    qs = D.batch_queries(cols, 500, seed=3)
    assert len(qs) == 500
    single = 0
    for q in qs:
        assert 1 <= len(q) <= 4
        assert len({c for c, _, _ in q}) == len(q)
        for c, lo, hi in q:
            assert lo <= hi
            single += lo == hi
    # log-uniform selectivity down to 1e-4 over up to 4 independent columns:
    # per-column shares of at least 1e-4 ** (1/k), never a single value of a
    # 2^32 domain
    assert single == 0
