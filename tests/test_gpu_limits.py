"""Parity at the size limits of the C ABI, on both scoring kernels.

* 128 reflections (GRC_MAX_NHKL): four reflections per lane in the prefilter.
* 1800 projections (GRC_MAX_NROT) with 36 reflections: 64,800 reflections per trial, the most
  the sweep's 16-bit histogram bins take; with 37 reflections (66,600) the sweep steps aside
  and the per-trial kernel scores, whatever path was asked for.
* 1800 projections x 128 reflections: the largest trial, 1800 omega rows in shared memory.
* One past each limit is refused with GRC_ECAPACITY and the context stays usable.

Counts and completeness bit-exact against the oracle for every trial without an edge
reflection, dis_median to 1e-6 relative, as in the other parity tests.  With 1800 projections
almost every trial holds some reflection within 1e-4 px of a pixel edge (about 10^4 selected
reflections per trial), so the tests also ask that at least 99% of all trials agree with the
oracle in every column: an edge reflection changes a decision only when the two FP64 forms
round differently, which is far rarer than being near an edge."""
import dataclasses

import numpy as np
import pytest

from grainrecon_b200 import geometry as G
from grainrecon_b200 import synth
from grainrecon_b200._lib import GRC_ECAPACITY, Context, GrcError
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", params=[1, 2], ids=["per-trial", "sweep"])
def path(request):
    return request.param


def _sample(nrot, nhkl):
    s = synth.make_sample("fe_small", seed=3, rot_angles=np.arange(nrot) * (360.0 / nrot))
    hkl = G.gen_hkl(229, 8)  # the first 8 BCC families: 140 reflections
    assert len(hkl) >= nhkl
    return dataclasses.replace(s, hkl=hkl[:nhkl])


def _parity(path, nrot, nhkl, n_or):
    s = _sample(nrot, nhkl)
    with Context(0) as ctx:
        ctx.set_path(path)
        host = synth.device_maps(s, ctx, keep_host_map=True)
        S9, B9, hkl, rot, R9, p = s.mex_arrays()
        idx = s.voxel_indices()
        rng = np.random.default_rng(nrot + nhkl)
        q = np.concatenate([s.grain_q, G.cubic_fz_orientations(n_or, nrot)]).astype(np.float32)
        n_clean = n_same = n_all = 0
        for v in idx[rng.choice(len(idx), 2, replace=False)]:
            pos = s.vol.pos_of_index(v).astype(np.float32)
            gpu = ctx.forward_comp(pos, q, S9, B9, hkl, None, rot, R9, p).reshape(-1, 4)
            used = ctx.last_stats()["path"]
            ref, _, edges = O.orientation_scan(pos, q, S9, B9, hkl, host, rot, R9, p, tight=True)
            ref = ref.reshape(-1, 4)
            clean = edges == 0
            n_clean += int(clean.sum())
            np.testing.assert_array_equal(gpu[clean, :3], ref[clean, :3])
            np.testing.assert_allclose(gpu[clean, 3], ref[clean, 3], rtol=1e-6)
            d = np.abs(gpu[~clean, :2] - ref[~clean, :2]).max(axis=1) if (~clean).any() else np.zeros(0)
            assert np.all(d <= edges[~clean])
            same = (gpu[:, :2] == ref[:, :2]).all(axis=1) & (
                (gpu[:, 2] == ref[:, 2]) | (np.isnan(gpu[:, 2]) & np.isnan(ref[:, 2]))) & np.isclose(
                gpu[:, 3], ref[:, 3], rtol=1e-6, atol=0)
            n_same += int(same.sum())
            n_all += len(same)
            assert gpu[s.grain_id[tuple(v - 1)] - 1, 2] >= 0.9  # the voxel's own grain is (almost) complete
        assert n_same >= 0.99 * n_all, (n_same, n_all)
        return n_clean, used, ref


def test_most_reflections(path):
    n_clean, used, ref = _parity(path, 37, 128, 400)
    assert used == path and n_clean > 300
    assert ref[:, 0].max() > 0


def test_most_projections_on_the_sweep(path):
    n_clean, used, ref = _parity(path, 1800, 36, 200)
    assert used == path


def test_sweep_steps_aside_above_its_bound(path):
    n_clean, used, ref = _parity(path, 1800, 37, 200)
    assert used == 1  # 1800 x 37 > 65,535: the per-trial kernel scores


def test_largest_trial(path):
    n_clean, used, ref = _parity(path, 1800, 128, 100)
    assert used == 1


def test_one_past_each_limit_is_refused():
    s = _sample(37, 86)
    S9, B9, hkl, rot, R9, p = s.mex_arrays()
    with Context(0) as ctx:
        synth.device_maps(s, ctx)
        one = np.array([1, 0, 0, 0], np.float32)
        p1 = p.copy()
        p1[0] = 129
        with pytest.raises(GrcError) as e:
            ctx.forward_comp(np.zeros(3), one, S9, B9, np.zeros(3 * 129), None, rot, R9, p1)
        assert e.value.code == GRC_ECAPACITY
        p2 = p.copy()
        p2[1] = 1801
        with pytest.raises(GrcError) as e:
            ctx.forward_comp(np.zeros(3), one, S9, B9, hkl, None, np.zeros(1801), R9, p2)
        assert e.value.code == GRC_ECAPACITY
        p3 = p.copy()
        p3[10], p3[11] = 1_000_001, 8
        with pytest.raises(GrcError) as e:
            ctx.forward_comp(np.zeros(3), one, S9, B9, hkl, None, rot, R9, p3)
        assert e.value.code == GRC_ECAPACITY
        p4 = p.copy()
        p4[10], p4[11] = 50_000, 50_000  # 2.5e9 pixels per projection
        with pytest.raises(GrcError) as e:
            ctx.forward_comp(np.zeros(3), one, S9, B9, hkl, None, rot, R9, p4)
        assert e.value.code == GRC_ECAPACITY
        out = ctx.forward_comp(np.zeros(3), one, S9, B9, hkl, None, rot, R9, p)  # still usable
        assert out.shape == (4,)
