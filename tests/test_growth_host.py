"""Host logic of the best-first growth (grow_indexed_region.m:32-137) and of the resident-map key,
without a GPU: the library's native walk (grc_walk_best_first, scores from a Python callback)
equals the oracle's numpy walk step for step, ties included, and the map key neither copies
nor misses a change."""
import numpy as np

from grainrecon_b200 import _lib
from grainrecon_b200 import forward as FW
from oracle import walk_oracle as WO


def _fake_scorer(dims, seed):
    """Deterministic per-voxel rows [Nr_simu, Nr_intersect, dis_median] with many tied ratios
    (dis_median float32-valued, as the scorer returns it)."""
    rng = np.random.default_rng(seed)
    ns = rng.integers(50, 60, dims).astype(float)
    ni = np.minimum(ns, np.round(ns * rng.choice([0.8, 0.9, 0.95, 1.0], dims)))
    dm = np.float32(rng.choice([0.1, 0.2, 0.3, 5.0], dims)).astype(float)

    def score(vox):
        ix = tuple((np.asarray(vox) - 1).T)
        return np.stack([ns[ix], ni[ix], dm[ix]], 1)

    return score


def test_native_walk_equals_oracle_walk():
    grown = 0
    for case in range(24):
        rng = np.random.default_rng(500 + case)
        dims = tuple(int(d) for d in rng.integers(6, 18, 3))
        Imask = (rng.random(dims) < 0.9).astype(float)
        I = np.where(rng.random(dims) < 0.3, rng.choice([0.5, 0.9], dims), 0.0)
        D = np.zeros(dims) + 20
        D[rng.random(dims) < 0.05] = np.nan  # MATLAB min ignores NaN in min(DisMedian, maxDmedian)
        N = rng.integers(0, 50, dims).astype(float)
        seed = np.array([rng.integers(1, d + 1) for d in dims])
        Imask[tuple(seed - 1)] = 1
        drop = (0.05, 0.2)[case % 2]
        a = WO.best_first_growth(_fake_scorer(dims, case), I, Imask, D, N, seed, drop, 3, 0.95, 10)
        b = _lib.walk_best_first(_fake_scorer(dims, case), I, Imask, D, N, seed, drop, 3, 0.95, 10)
        for x, y in zip(a, b):
            np.testing.assert_array_equal(np.asarray(x), np.asarray(y))
        grown += len(a[6])
    assert grown > 2000  # the cases grow real regions, not just the seed


def test_native_walk_reports_scorer_errors():
    dims = (5, 5, 5)
    one = np.ones(dims)

    def broken(vox):
        raise ValueError("scorer failed")

    try:
        _lib.walk_best_first(broken, np.zeros(dims), one, one * 20, one * 0, (3, 3, 3), 0.05, 3, 0.95, 10)
    except ValueError as e:
        assert "scorer failed" in str(e)
    else:
        raise AssertionError("the scorer's error was swallowed")


def test_map_key_samples_without_copy_and_sees_changes():
    FW.reset_masks()
    h = np.random.default_rng(0).random((9, 40, 48), dtype=np.float32)
    a = h.transpose(2, 1, 0)  # detz x dety x nrot view of a C-contiguous (nrot, dety, detz) map
    flat = FW._map_for_call(a)
    np.testing.assert_array_equal(flat, h.reshape(-1))  # reshape(proj_bin_bw,1,[]) order
    assert FW._map_for_call(a) is None  # resident: not uploaded again
    b = a.copy()
    b[0, 0, 0] += 1  # a different array object is uploaded even when its sample matches
    assert FW._map_for_call(b) is not None
    FW.reset_masks()
    assert FW._map_for_call(b) is not None
