"""GPU seeding stage: FP64 trial lists, the batched orientation fit and the seed indexer against
the oracle's one-seed-at-a-time restatement; the in-order engine end to end.

Bar: counts, completeness and every decision bit-exact for trials with no edge reflection; a
seed whose oracle trace met an edge reflection (landing within 1e-4 px of a pixel boundary)
may differ and is listed.  Fitted parameters agree to 1e-12 (the two sides evaluate
sin/asin with different libraries, within an ulp)."""
import math

import numpy as np
import pytest

from grainrecon_b200 import geometry as G
from grainrecon_b200 import seeding as S
from grainrecon_b200 import synth
from grainrecon_b200._lib import Context, GrcError
from oracle import seed_oracle as SO
from spot_fixtures import measured_spots

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def scene():
    s = synth.make_sample("fe_small", seed=1)
    dmap = synth.distance_map(synth.simulate_mask(s))
    ctx = Context(0)
    S9, B9, hkl, rot, R9, p = s.mex_arrays()
    ctx.set_geometry(S9, B9, hkl, rot, R9, p)
    ctx.upload_masks(dmap.reshape(-1), s.geom.detzsize, s.geom.detysize, s.geom.nrot)
    yield s, ctx, SO.Scene(S9, B9, hkl, rot, R9, p, dmap), dmap
    ctx.close()


def _voxels(s, n, seed):
    idx = s.voxel_indices()
    rng = np.random.default_rng(seed)
    v = idx[rng.choice(len(idx), n, replace=False)]
    return v, s.vol.pos_of_index(v)


_OPS = [G.quat_to_u(o) for o in G._cubic_ops()]


def _misori_deg(Ua, Ub):
    """Cubic-symmetry-reduced misorientation angle [deg]."""
    c = max((np.trace(Ua.T @ Ub @ C) - 1) / 2 for C in _OPS)
    return float(np.degrees(np.arccos(np.clip(c, -1, 1))))


def _near(q, rng, scale):
    x = np.asarray(q, np.float64)[1:] + rng.uniform(-scale, scale, 3)
    return np.array([math.sqrt(1 - float(x @ x)), *x])


def test_trial_list_matches_oracle(scene):
    import torch
    s, ctx, sc, _ = scene
    rng = np.random.default_rng(5)
    vox, pos = _voxels(s, 8, 1)
    qs = np.array([_near(s.grain_q[rng.integers(len(s.grain_q))], rng, 0.01) for _ in range(40)])
    tv = rng.integers(0, 8, 300).astype(np.int32)
    to = rng.integers(0, 40, 300).astype(np.int32)
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    out = torch.empty(300 * 4, dtype=torch.float32, device="cuda")
    ctx.score_trials_device(d(pos), 8, d(qs), 40, d(tv), d(to), 300, out)
    gpu = out.view(-1, 4).cpu().numpy()
    n_clean = 0
    for t in range(300):
        r = sc.score_u(SO.quat_u(*qs[to[t]]), pos[tv[t]])
        if r[3] == 0:
            n_clean += 1
            assert gpu[t, 0] == r[0] and gpu[t, 1] == r[1], t
            assert gpu[t, 2] == np.float32(r[1] / r[0])
            np.testing.assert_allclose(gpu[t, 3], r[2], rtol=1e-6)
        else:
            assert np.abs(gpu[t, :2] - r[:2]).max() <= r[3]
    assert n_clean > 150
    # diagonal form: trial t = (voxel t, orientation t)
    out2 = torch.empty(8 * 4, dtype=torch.float32, device="cuda")
    ctx.score_trials_device(d(pos), 8, d(qs[:8]), 8, None, None, 8, out2)
    for t in range(8):
        r = sc.score_u(SO.quat_u(*qs[t]), pos[t])
        if r[3] == 0:
            assert out2[4 * t].item() == r[0] and out2[4 * t + 1].item() == r[1]
    bad = to.copy()
    bad[7] = 40
    with pytest.raises(GrcError):
        ctx.score_trials_device(d(pos), 8, d(qs), 40, d(tv), d(bad), 300, out)


def test_trial_list_voxel_orders(scene):
    """The sweep sizes its per-tile voxel rows from the list's voxel-run starts (the most starts in
    any aligned block of 32 trials).  Lists in several voxel orders -- seed-major (730 trials per
    voxel, as the local refine builds them), runs of 10, runs of 1-3, two voxels alternating in
    pairs, and all of them concatenated -- must score identically on the sweep and on the
    per-trial kernel, which keeps no per-tile rows."""
    import torch
    s, ctx, sc, _ = scene
    rng = np.random.default_rng(9)
    vox, pos = _voxels(s, 40, 3)
    qs = np.array([_near(s.grain_q[k % len(s.grain_q)], rng, 0.002 if k < 120 else 0.05) for k in range(730)])
    n = 40 * 730
    runs = np.repeat(np.arange(40), 10)
    short = rng.integers(1, 4, n)
    orders = {
        "seed-major": np.repeat(np.arange(40), 730),
        "runs of 10": np.resize(runs, n),
        "runs of 1-3": np.resize(np.repeat(rng.integers(0, 40, n), short), n),
        "alternating pairs": np.resize(np.array([5, 5, 9, 9]), n),
    }
    orders["concatenated"] = np.concatenate([v[: n // 4] for v in orders.values()])[:n]
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    try:
        for name, tv in orders.items():
            tv = tv.astype(np.int32)
            to = rng.integers(0, 730, n).astype(np.int32)
            res = {}
            for path in (2, 3, 1):
                ctx.set_path(path)
                out = torch.empty(n * 4, dtype=torch.float32, device="cuda")
                ctx.score_trials_device(d(pos), 40, d(qs), 730, d(tv), d(to), n, out)
                res[path] = out.view(-1, 4).cpu().numpy()
                assert ctx.last_stats()["path"] == path, name
            np.testing.assert_array_equal(res[2], res[1], err_msg=name)
            np.testing.assert_array_equal(res[3], res[1], err_msg=name)
            assert np.nanmax(res[2][:, 2]) > 0.9, name  # near-true orientations are scored
    finally:
        ctx.set_path(0)


def test_orientation_fit_matches_oracle_fminsearchbnd(scene):
    import torch
    s, ctx, sc, _ = scene
    rng = np.random.default_rng(6)
    vox, pos = _voxels(s, 12, 2)
    gid = s.grain_id[tuple((vox - 1).T)]
    x0 = np.array([_near(s.grain_q[g - 1], rng, 0.008)[1:] for g in gid])
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    n = len(x0)
    x = torch.empty(n, 3, dtype=torch.float64, device="cuda")
    fval = torch.empty(n, dtype=torch.float64, device="cuda")
    ev, it, fl = (torch.empty(n, dtype=torch.int32, device="cuda") for _ in range(3))
    ctx.fit_orientation_nm(d(pos), d(x0), n, x, fval, ev, it, fl)
    # the iterations run as one graph whose conditional WHILE node stops on the device
    assert ctx.last_stats()["device_loop"] == 1
    x, fval, ev, it, fl = (a.cpu().numpy() for a in (x, fval, ev, it, fl))
    same = 0
    for i in range(n):
        lb = [max(v - 0.02, -1.0) for v in x0[i]]
        ub = [min(v + 0.02, 1.0) for v in x0[i]]
        xo, fo, eo, io, flo, extra = SO.fminsearchbnd(SO.nm_objective(sc, pos[i]), list(x0[i]), lb, ub)
        if sum(extra) == 0 or (ev[i] == eo and fval[i] == fo):
            assert ev[i] == eo and it[i] == io and fl[i] == flo, (i, ev[i], eo, it[i], io)
            assert fval[i] == fo
            np.testing.assert_allclose(x[i], xo, rtol=0, atol=1e-12)
            same += 1
    assert same >= n - 1
    assert np.median(fval) < 0.05  # the fit finds (almost) complete orientations
    assert np.all(fl >= 0)


def test_seed_indexer_matches_oracle(scene):
    s, ctx, sc, _ = scene
    q_grid = np.concatenate([s.grain_q, G.cubic_fz_orientations(300, 17)]).astype(np.float32)
    vox, pos = _voxels(s, 4, 3)
    ix = S.SeedIndexer(ctx, q_grid, nr_seed=3)
    rows, cid = ix.index([1, 2, 3, 4], pos)
    same = 0
    for i in range(4):
        ro, co, edges, _ = SO.index_seed(sc, pos[i], q_grid, 3, seed_id=i + 1)
        ok = (rows[i, 4:6] == ro[4:6]).all() and cid[i] == co
        if ok:
            assert rows[i, 6] == ro[6]
            np.testing.assert_allclose(rows[i, 7], ro[7], rtol=1e-6)
            np.testing.assert_allclose(rows[i, 8:11], ro[8:11], rtol=0, atol=1e-7)
            np.testing.assert_allclose(rows[i, 14:18], ro[14:18], rtol=0, atol=1e-9)
            same += 1
        else:
            assert edges > 0, (i, rows[i], ro)
    assert same >= 3
    for i in range(4):  # each seed finds one of the sample's grains (at 0.27 mm pixels a seed
        # near a boundary can take its neighbour)
        Uf = G.quat_to_u(rows[i, 14:18])
        assert rows[i, 6] > 0.9
        assert min(_misori_deg(G.quat_to_u(q), Uf) for q in s.grain_q) < 1.0
    assert ix.stats["local_trials"] == 4 * 3 * 730


def test_engine_indexes_the_sample(scene):
    s, _, _, dmap = scene
    g = s.geom
    S9, B9, hkl, rot, R9, p = s.mex_arrays()
    dims = s.grain_id.shape
    DS = {"Mask": (s.grain_id > 0).astype(np.float64), "Completeness": np.zeros(dims),
          "GrainId": np.zeros(dims), "Dismedian": np.zeros(dims) + 10, "Ninter": np.zeros(dims),
          "VisitFlag": np.zeros(dims), "EulerZXZ": np.zeros((3,) + dims), "Rodrigues": np.zeros((3,) + dims),
          "IPF001": np.zeros((3,) + dims)}
    vox, pos = _voxels(s, 12, 4)
    q_grid = np.concatenate([s.grain_q, G.cubic_fz_orientations(300, 17)]).astype(np.float32)
    ts = {"Center": np.array(s.vol.center), "Dimension": np.array(s.vol.dimension)}
    rvp = np.array([[1, dims[0]], [1, dims[1]], [1, dims[2]]])
    hkl3 = s.hkl
    out, pos_new, DSo, nvox = S.GrainMapping_engine_gpu_comp(
        pos, {"q": q_grid}, g.rot_det, None, dmap.transpose(2, 1, 0), g.rot_angles, s.S, s.B, hkl3, len(hkl3),
        g.theta_max, g.lambda_min, g.lambda_max, g.lss, g.lsd, 0.85, 0.5, 0.5 * g.pxy, g.dety00, g.detz00, g.p0y,
        g.p0z, g.rot_axis_offset, g.pxy, g.pxz, g.detysize / 2 + 0.5, g.detzsize / 2 + 0.5, g.detysize, g.detzsize,
        g.beamstop_y, g.beamstop_z, 0.05, 3, DS, ts, s.vol.vox_size, rvp, 1, s.vol.simap, 10, 3, batch=8)
    mask = s.grain_id > 0
    got = DSo["GrainId"] > 0
    assert got[mask].mean() > 0.6, got[mask].mean()
    assert not got[~mask].any()
    # every indexed voxel carries one of the sample's grain orientations (at 0.27 mm pixels the
    # whole 0.1 mm sample spans under half a pixel, so growth cannot see grain boundaries; the
    # reference leaves those to its compete pass)
    eul = DSo["EulerZXZ"][:, got]
    Ug = [G.quat_to_u(q) for q in s.grain_q]
    bad = 0
    for k in range(eul.shape[1]):
        Uf = G.euler_to_u(*np.radians(eul[:, k]))
        bad += min(_misori_deg(U, Uf) for U in Ug) > 1.0
    assert bad == 0
    ids = np.unique(DSo["GrainId"][got])
    assert len(ids) >= 1 and np.all(nvox[ids.astype(int) - 1] > 0)
    assert out[:, 6].max() > 0.9
    assert DSo["indexer_stats"]["fit_seeds"] >= 1


def test_engine_with_measured_spots(scene):
    """With spots, every accepted seed is paired, its centre fitted to the pairs, and the growth box
    follows the spot size; the indexed orientations are still the sample's."""
    s, _, sc, dmap = scene
    g = s.geom
    dims = s.grain_id.shape
    DS = {"Mask": (s.grain_id > 0).astype(np.float64), "Completeness": np.zeros(dims),
          "GrainId": np.zeros(dims), "Dismedian": np.zeros(dims) + 10, "Ninter": np.zeros(dims),
          "VisitFlag": np.zeros(dims), "EulerZXZ": np.zeros((3,) + dims)}
    vox, pos = _voxels(s, 6, 9)
    q_grid = np.concatenate([s.grain_q, G.cubic_fz_orientations(300, 17)]).astype(np.float32)
    ts = {"Center": np.array(s.vol.center), "Dimension": np.array(s.vol.dimension)}
    rvp = np.array([[1, dims[0]], [1, dims[1]], [1, dims[2]]])
    spots = measured_spots(s, sc, 0.3, 11)
    out, pos_new, DSo, nvox = S.GrainMapping_engine_gpu_comp(
        pos, {"q": q_grid}, g.rot_det, spots, dmap.transpose(2, 1, 0), g.rot_angles, s.S, s.B, s.hkl, len(s.hkl),
        g.theta_max, g.lambda_min, g.lambda_max, g.lss, g.lsd, 0.85, 0.5, 0.5 * g.pxy, g.dety00, g.detz00, g.p0y,
        g.p0z, g.rot_axis_offset, g.pxy, g.pxz, g.detysize / 2 + 0.5, g.detzsize / 2 + 0.5, g.detysize, g.detzsize,
        g.beamstop_y, g.beamstop_z, 0.05, 3, DS, ts, s.vol.vox_size, rvp, 1, s.vol.simap, 10, 3, batch=4)
    pairs = DSo["spots_pair"]
    assert len(pairs) >= 1 and all(len(p) > 20 for p in pairs.values())
    got = DSo["GrainId"] > 0
    assert got[s.grain_id > 0].mean() > 0.5
    Ug = [G.quat_to_u(q) for q in s.grain_q]
    for k in range(int(got.sum())):
        e = DSo["EulerZXZ"][:, got][:, k]
        assert min(_misori_deg(U, G.euler_to_u(*np.radians(e))) for U in Ug) < 1.0


def test_engine_small_spots_take_the_best_first_growth(scene):
    """Spots of 1-3 px^2 give Spot_L <= 2 px, so every accepted seed grows voxel by voxel
    (grow_indexed_region) instead of within a bounding volume."""
    s, _, sc, dmap = scene
    g = s.geom
    dims = s.grain_id.shape
    DS = {"Mask": (s.grain_id > 0).astype(np.float64), "Completeness": np.zeros(dims),
          "GrainId": np.zeros(dims), "Dismedian": np.zeros(dims) + 10, "Ninter": np.zeros(dims),
          "VisitFlag": np.zeros(dims), "EulerZXZ": np.zeros((3,) + dims)}
    vox, pos = _voxels(s, 4, 13)
    q_grid = np.concatenate([s.grain_q, G.cubic_fz_orientations(300, 17)]).astype(np.float32)
    ts = {"Center": np.array(s.vol.center), "Dimension": np.array(s.vol.dimension)}
    rvp = np.array([[1, dims[0]], [1, dims[1]], [1, dims[2]]])
    spots = measured_spots(s, sc, 0.2, 12, area=(1, 3))
    out, pos_new, DSo, nvox = S.GrainMapping_engine_gpu_comp(
        pos, {"q": q_grid}, g.rot_det, spots, dmap.transpose(2, 1, 0), g.rot_angles, s.S, s.B, s.hkl, len(s.hkl),
        g.theta_max, g.lambda_min, g.lambda_max, g.lss, g.lsd, 0.85, 0.5, 0.5 * g.pxy, g.dety00, g.detz00, g.p0y,
        g.p0z, g.rot_axis_offset, g.pxy, g.pxz, g.detysize / 2 + 0.5, g.detzsize / 2 + 0.5, g.detysize, g.detzsize,
        g.beamstop_y, g.beamstop_z, 0.05, 3, DS, ts, s.vol.vox_size, rvp, 1, s.vol.simap, 10, 3, batch=4)
    pairs = DSo["spots_pair"]
    assert pairs and all(np.sqrt((p["area"].mean() + 2 * p["area"].std(ddof=1)) / np.pi) <= 2 for p in pairs.values())
    got = DSo["GrainId"] > 0
    assert got.sum() > 5 and not got[s.grain_id == 0].any()
    for gid in np.unique(DSo["GrainId"][got]):
        region = DSo["GrainId"] == gid
        # best-first growth walks through face/edge neighbours: one connected region per seed
        from scipy import ndimage
        lab, n = ndimage.label(region, structure=ndimage.generate_binary_structure(3, 2))
        assert n == 1
