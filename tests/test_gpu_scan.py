"""The completeness-only scan (bit-packed hit mask) and the first maximum per group.

* With the median switched off (grc_set_median(ctx, 0)) the seeding-scan entries count Nr_simu and
  Nr_intersect from a bit-packed hit mask; columns 1-3 must equal the oracle's on every trial
  without a tight edge reflection, column 4 is NaN, on every kernel path.
* The first maximum of completeness per voxel (grc_forward_comp_argmax_device) and per group of
  consecutive trials (grc_score_trials_argmax_device) equals MATLAB's max over column 3 (first
  maximum, NaN ignored) of the same call's output -- whether the warp scan folds it in (completeness
  mode) or a separate warp-shuffle kernel reads the trial results (full mode, per-trial kernel).
* The packed mask follows the hit threshold and a new map."""
import numpy as np
import pytest

from grainrecon_b200 import geometry as G
from grainrecon_b200 import synth
from grainrecon_b200._lib import Context, GrcError, GRC_EINVAL
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _first_max(c):
    c = np.where(np.isnan(c), -np.inf, c)
    return int(np.argmax(c)), (float(c.max()) if np.isfinite(c).any() else float("nan"))


@pytest.fixture(scope="module")
def scene():
    s = synth.make_sample("al_small", seed=2)
    dmap = synth.distance_map(synth.simulate_mask(s, stride=2))
    ctx = Context(0)
    S9, B9, hkl, rot, R9, p = s.mex_arrays()
    ctx.set_geometry(S9, B9, hkl, rot, R9, p)
    ctx.upload_masks(dmap, s.geom.detzsize, s.geom.detysize, s.geom.nrot)
    yield s, dmap, ctx
    ctx.close()


@pytest.mark.parametrize("path", [1, 2, 3])
def test_completeness_only_scan_matches_oracle(scene, path):
    s, dmap, ctx = scene
    S9, B9, hkl, rot, R9, p = s.mex_arrays()
    idx = s.voxel_indices()
    rng = np.random.default_rng(11)
    q = np.concatenate([s.grain_q, G.cubic_fz_orientations(3000, 5)]).astype(np.float32)
    ctx.set_path(path)
    ctx.set_median(False)
    try:
        for v in idx[rng.choice(len(idx), 3, replace=False)]:
            pos = s.vol.pos_of_index(v).astype(np.float32)
            gpu = ctx.forward_comp(pos, q, S9, B9, hkl, None, rot, R9, p).reshape(-1, 4)
            assert ctx.last_stats()["path"] == path
            ref, _, tight = O.orientation_scan(pos, q, S9, B9, hkl, dmap, rot, R9, p, tight=True)
            ref = ref.reshape(-1, 4)
            exact = tight == 0
            assert exact.sum() >= len(q) - 3
            np.testing.assert_array_equal(gpu[exact, :3], ref[exact, :3])
            assert np.isnan(gpu[:, 3]).all()
    finally:
        ctx.set_path(0)
        ctx.set_median(True)


@pytest.mark.parametrize("median,path", [(False, 2), (True, 2), (False, 3), (True, 3), (True, 1), (False, 1)])
def test_argmax_per_voxel(scene, median, path):
    import torch
    s, dmap, ctx = scene
    idx = s.voxel_indices()
    rng = np.random.default_rng(3)
    vox = idx[rng.choice(len(idx), 5, replace=False)]
    pos = torch.from_numpy(s.vol.pos_of_index(vox).astype(np.float32).reshape(-1)).cuda()
    q = np.concatenate([s.grain_q, G.cubic_fz_orientations(2500, 9)]).astype(np.float32)
    n_q = len(q)
    d_q = torch.from_numpy(q.reshape(-1)).cuda()
    out = torch.empty(5 * n_q * 4, dtype=torch.float32, device="cuda")
    best = torch.full((5,), -1, dtype=torch.int32, device="cuda")
    best_c = torch.empty(5, dtype=torch.float32, device="cuda")
    ctx.set_path(path)
    ctx.set_median(median)
    try:
        ctx.forward_comp_argmax_device(pos, 5, d_q, n_q, out, best, best_c)
        torch.cuda.synchronize()
        o = out.view(5, n_q, 4).cpu().numpy()
        for v in range(5):
            i, c = _first_max(o[v, :, 2])
            assert int(best[v]) == i and float(best_c[v]) == c
        # the same without the per-trial output
        best2 = torch.full((5,), -1, dtype=torch.int32, device="cuda")
        ctx.forward_comp_argmax_device(pos, 5, d_q, n_q, None, best2, None)
        torch.cuda.synchronize()
        assert torch.equal(best, best2)
    finally:
        ctx.set_path(0)
        ctx.set_median(True)


@pytest.mark.parametrize("median,path", [(False, 2), (True, 2), (False, 3), (True, 3), (False, 1)])
def test_argmax_per_group_of_trials(scene, median, path):
    """Local-refine shape: groups of 729 consecutive trials of one voxel (one candidate grid each)."""
    import torch
    s, dmap, ctx = scene
    idx = s.voxel_indices()
    vox = idx[[5, 400]]
    pos = torch.from_numpy(s.vol.pos_of_index(vox).reshape(-1).astype(np.float64)).cuda()
    gsize, n_groups = 729, 12  # unique(q,'rows') keeps 729 or 730 rows of a 9^3 grid + centre
    cand = np.concatenate([s.grain_q[:4], G.cubic_fz_orientations(n_groups - 4, 21)])
    grids = np.concatenate([G.ori_local_sampling(c, 8, 0.004)[:gsize] for c in cand])
    assert grids.shape == (gsize * n_groups, 4)
    d_q = torch.from_numpy(grids.astype(np.float64).reshape(-1)).cuda()
    n = gsize * n_groups
    tv = torch.from_numpy(np.repeat(np.arange(2, dtype=np.int32), n // 2)).cuda()
    to = torch.arange(n, dtype=torch.int32, device="cuda")
    out = torch.empty(n * 4, dtype=torch.float32, device="cuda")
    best = torch.full((n_groups,), -1, dtype=torch.int32, device="cuda")
    best_c = torch.empty(n_groups, dtype=torch.float32, device="cuda")
    ctx.set_median(median)
    ctx.set_path(path)
    try:
        ctx.score_trials_argmax_device(pos, 2, d_q, n, tv, to, n, gsize, out, best, best_c)
        torch.cuda.synchronize()
        o = out.view(n_groups, gsize, 4).cpu().numpy()
        assert ctx.last_stats()["path"] == path
        for g in range(n_groups):
            i, c = _first_max(o[g, :, 2])
            assert int(best[g]) == i and (float(best_c[g]) == c or (np.isnan(c) and np.isnan(float(best_c[g]))))
        with pytest.raises(GrcError) as e:  # n_trials must be a multiple of group_size
            ctx.score_trials_argmax_device(pos, 2, d_q, n, tv, to, n - 1, gsize, out, best, best_c)
        assert e.value.code == GRC_EINVAL
    finally:
        ctx.set_median(True)
        ctx.set_path(0)


def test_first_max_of_all_nan_is_the_first_index():
    """A geometry where no reflection lands gives 0/0 = NaN completeness on every trial; MATLAB's
    max then returns the first index, and the decoded completeness is NaN."""
    import torch
    s = synth.make_sample("fe_tiny", seed=1)
    dmap = synth.distance_map(synth.simulate_mask(s))
    S9, B9, hkl, rot, R9, p = s.mex_arrays()
    p_none = p.copy()
    p_none[17], p_none[18] = 50.0, 60.0  # wavelength window no reflection reaches: every trial is 0/0
    q = G.cubic_fz_orientations(64, 1).astype(np.float32)
    with Context(0) as ctx:
        ctx.set_geometry(S9, B9, hkl, rot, R9, p_none)
        ctx.upload_masks(dmap, s.geom.detzsize, s.geom.detysize, s.geom.nrot)
        pos = torch.zeros(3, dtype=torch.float32, device="cuda")
        d_q = torch.from_numpy(q.reshape(-1)).cuda()
        best = torch.full((1,), -1, dtype=torch.int32, device="cuda")
        best_c = torch.zeros(1, dtype=torch.float32, device="cuda")
        for median in (True, False):
            ctx.set_median(median)
            ctx.forward_comp_argmax_device(pos, 1, d_q, len(q), None, best, best_c)
            torch.cuda.synchronize()
            assert int(best[0]) == 0 and np.isnan(float(best_c[0]))


def test_packed_mask_follows_threshold_and_map(scene):
    s, dmap, ctx = scene
    S9, B9, hkl, rot, R9, p = s.mex_arrays()
    idx = s.voxel_indices()
    pos = s.vol.pos_of_index(idx[len(idx) // 3]).astype(np.float32)
    q = np.concatenate([s.grain_q, G.cubic_fz_orientations(2000, 2)]).astype(np.float32)
    ctx.set_path(2)
    try:
        for thr in (1.5, 3.0, 0.5):
            ctx.set_options(hit_threshold=thr)
            ctx.set_median(True)
            full = ctx.forward_comp(pos, q, S9, B9, hkl, None, rot, R9, p).reshape(-1, 4)
            ctx.set_median(False)
            comp = ctx.forward_comp(pos, q, S9, B9, hkl, None, rot, R9, p).reshape(-1, 4)
            np.testing.assert_array_equal(comp[:, :3], full[:, :3])
        # a new map: the packed mask is rebuilt from it
        dmap2 = np.ascontiguousarray(dmap[:, ::-1, :])
        ctx.upload_masks(dmap2, s.geom.detzsize, s.geom.detysize, s.geom.nrot)
        ctx.set_median(True)
        full = ctx.forward_comp(pos, q, S9, B9, hkl, None, rot, R9, p).reshape(-1, 4)
        ctx.set_median(False)
        comp = ctx.forward_comp(pos, q, S9, B9, hkl, None, rot, R9, p).reshape(-1, 4)
        np.testing.assert_array_equal(comp[:, :3], full[:, :3])
    finally:
        ctx.upload_masks(dmap, s.geom.detzsize, s.geom.detysize, s.geom.nrot)
        ctx.set_options()
        ctx.set_median(True)
        ctx.set_path(0)


def test_argmax_entries_refuse_host_buffers(scene):
    import torch
    s, dmap, ctx = scene
    q = G.cubic_fz_orientations(8, 1).astype(np.float32)
    with pytest.raises(GrcError) as e:
        ctx.forward_comp_argmax_device(torch.zeros(3), 1, torch.from_numpy(q.reshape(-1)), 8, None,
                                       torch.zeros(1, dtype=torch.int32, device="cuda"), None)
    assert e.value.code == GRC_EINVAL


def test_keyed_upload_follows_content(scene):
    """grc_upload_masks_if_changed: a map with the same content in a new buffer is not uploaded
    again; a changed map, or any upload in between, is."""
    s, dmap, ctx = scene
    g = s.geom
    dims = (g.detzsize, g.detysize, g.nrot)
    S9, B9, hkl, rot, R9, p = s.mex_arrays()
    pos = s.vol.pos_of_index(s.voxel_indices()[7]).astype(np.float32)
    q = G.cubic_fz_orientations(500, 4).astype(np.float32)
    ref = ctx.forward_comp(pos, q, S9, B9, hkl, None, rot, R9, p)
    try:
        assert ctx.upload_masks_if_changed(dmap, *dims)            # the fixture's upload had no key
        assert not ctx.upload_masks_if_changed(dmap.copy(), *dims)  # same content, other buffer
        changed = dmap.copy().reshape(-1)
        changed[0] = changed[0] + 1.0
        assert ctx.upload_masks_if_changed(changed, *dims)
        assert ctx.upload_masks_if_changed(dmap, *dims)
        ctx.upload_masks(dmap, *dims)                               # clears the recorded key
        assert ctx.upload_masks_if_changed(dmap, *dims)
        np.testing.assert_array_equal(ctx.forward_comp(pos, q, S9, B9, hkl, None, rot, R9, p), ref)
    finally:
        ctx.upload_masks(dmap, *dims)


def test_size_rule_picks_kernel_by_output_mode(scene):
    """grc_set_path(ctx, 0): full-output calls of more than two warp-scan rounds take the CTA sweep,
    shorter ones and every completeness-only call the warp scan; the output does not depend on it."""
    import torch
    s, dmap, ctx = scene
    idx = s.voxel_indices()
    q = G.cubic_fz_orientations(30000, 13).astype(np.float32)
    d_q = torch.from_numpy(q.reshape(-1)).cuda()
    n_sm = torch.cuda.get_device_properties(0).multi_processor_count
    rnd = n_sm * 3 * 64  # trials of one warp-scan round at 3 CTAs per SM
    cases = ((1, True, 3), (3, True, 2 if 3 * len(q) > 2 * rnd else 3), (3, False, 3))
    try:
        for n_vox, median, path in cases:
            pos = torch.from_numpy(s.vol.pos_of_index(idx[[9, 200, 333][:n_vox]]).astype(np.float32).reshape(-1)).cuda()
            out = torch.empty(n_vox * len(q) * 4, dtype=torch.float32, device="cuda")
            ctx.set_median(median)
            ctx.set_path(0)
            ctx.forward_comp_device(pos, n_vox, d_q, len(q), out)
            torch.cuda.synchronize()
            assert ctx.last_stats()["path"] == path
            ref = torch.empty_like(out)
            ctx.set_path(3 if path == 2 else 2)
            ctx.forward_comp_device(pos, n_vox, d_q, len(q), ref)
            torch.cuda.synchronize()
            assert torch.equal(out.view(-1, 4)[:, :3], ref.view(-1, 4)[:, :3])
            if median:
                assert torch.equal(out.view(-1, 4)[:, 3], ref.view(-1, 4)[:, 3])
    finally:
        ctx.set_median(True)
        ctx.set_path(0)
