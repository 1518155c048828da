"""Device ordering work of the seeding stage against the oracle's restatement.

* grc_local_grid_device: ori_local_sampling grids (ori_local_sampling.m:12-34) in unique(q,'rows')
  order, bit-identical to the oracle's rows (a row equal to another, which unique drops, stays
  beside it);
* grc_seed_candidates_device: the scan's first n_top rows of sortrows(Output, 3, 'descend') (NaN
  first, equal values in grid order), checked against the oracle's sortrows on the same call's
  output column 3;
* grc_seed_refine_device: each candidate grid's first maximum and the candidates in sortrows order,
  checked against a host reduction of the same grids scored through grc_score_trials_device."""
import numpy as np
import pytest

from grainrecon_b200 import geometry as G
from grainrecon_b200 import synth
from grainrecon_b200._lib import Context
from oracle import seed_oracle as SO

pytestmark = pytest.mark.gpu


def _twins_out(a):
    keep = np.ones(len(a), bool)
    keep[1:] = np.any(a[1:] != a[:-1], axis=1)
    return a[keep]


@pytest.fixture(scope="module")
def scene():
    s = synth.make_sample("al_small", seed=2)
    dmap = synth.distance_map(synth.simulate_mask(s, stride=2))
    ctx = Context(0)
    S9, B9, hkl, rot, R9, p = s.mex_arrays()
    ctx.set_geometry(S9, B9, hkl, rot, R9, p)
    ctx.upload_masks(dmap, s.geom.detzsize, s.geom.detysize, s.geom.nrot)
    yield s, ctx
    ctx.close()


@pytest.mark.parametrize("nr", [4, 8])
def test_local_grid_matches_oracle(scene, nr):
    import torch
    s, ctx = scene
    rng = np.random.default_rng(nr)
    qc = rng.normal(size=(7, 4))
    qc[:, 0] = np.abs(qc[:, 0]) + 1.5  # every grid point inside the unit ball
    qc /= np.linalg.norm(qc, axis=1, keepdims=True)
    qc[0] = s.grain_q[0]
    L = (nr + 1) ** 3 + 1
    rows = torch.empty(7 * L * 4, dtype=torch.float64, device="cuda")
    rows32 = torch.empty(7 * L * 4, dtype=torch.float32, device="cuda")
    ctx.local_grid_device(torch.from_numpy(qc.reshape(-1).copy()).cuda(), 7, nr, 0.004, rows, rows32)
    g = rows.view(7, L, 4).cpu().numpy()
    g32 = rows32.view(7, L, 4).cpu().numpy()
    np.testing.assert_array_equal(g32, g.astype(np.float32))
    for i in range(7):
        ref = SO.ori_local(qc[i], nr, 0.004)
        np.testing.assert_array_equal(_twins_out(g[i]), ref)


def test_seed_candidates_match_sortrows(scene):
    import torch
    s, ctx = scene
    idx = s.voxel_indices()
    rng = np.random.default_rng(4)
    vox = idx[rng.choice(len(idx), 6, replace=False)]
    pos = s.vol.pos_of_index(vox).astype(np.float32)
    q64 = np.concatenate([s.grain_q, G.cubic_fz_orientations(3000, 3)])
    q32 = q64.astype(np.float32)
    n, N, k = 6, len(q64), 400
    d_idx = torch.empty(n * k, dtype=torch.int32, device="cuda")
    d_cand = torch.empty(n * k * 4, dtype=torch.float64, device="cuda")
    d_out = torch.empty(n * N * 4, dtype=torch.float32, device="cuda")
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a).reshape(-1)).cuda()
    ctx.seed_candidates_device(d(pos), n, d(q32), N, k, d_idx, d_cand, d_out, d(q64))
    out = d_out.view(n, N, 4).cpu().numpy()
    got = d_idx.view(n, k).cpu().numpy()
    cand = d_cand.view(n, k, 4).cpu().numpy()
    assert np.isnan(out[:, :, 3]).all()  # completeness only
    for v in range(n):
        ref = SO.top(out[v].astype(np.float64), k)
        np.testing.assert_array_equal(got[v], ref)
        np.testing.assert_array_equal(cand[v], q64[ref])
        assert len(np.unique(out[v, :, 2])) < N  # equal completeness values occur: the order is stable


def test_seed_refine_matches_host_reduction(scene):
    import torch
    s, ctx = scene
    idx = s.voxel_indices()
    rng = np.random.default_rng(9)
    vox = idx[rng.choice(len(idx), 3, replace=False)]
    pos = s.vol.pos_of_index(vox).astype(np.float64)
    n, k, nr = 3, 24, 8
    L = (nr + 1) ** 3 + 1
    cand = np.concatenate([s.grain_q[:8], G.cubic_fz_orientations(3 * k - 8, 17)]).reshape(n, k, 4)
    d_cand = torch.from_numpy(cand.reshape(-1).copy()).cuda()
    pos32 = pos.astype(np.float32).astype(np.float64)
    d_pos = torch.from_numpy(pos32.reshape(-1).copy()).cuda()
    best_q = torch.empty(n * k * 4, dtype=torch.float64, device="cuda")
    best_c = torch.empty(n * k, dtype=torch.float32, device="cuda")
    order = torch.empty(n * k, dtype=torch.int32, device="cuda")
    x0 = torch.empty(n * 2 * 3, dtype=torch.float64, device="cuda")
    ctx.seed_refine_device(d_pos, n, d_cand, k, nr, 0.004, best_q, best_c, order, 2, x0)
    bq = best_q.view(n, k, 4).cpu().numpy()
    bc = best_c.view(n, k).cpu().numpy()
    od = order.view(n, k).cpu().numpy()
    xx = x0.view(n, 2, 3).cpu().numpy()
    # host reduction: the same grids scored through the FP64 trial entry (completeness only)
    grid = torch.empty(n * k * L * 4, dtype=torch.float64, device="cuda")
    grid32 = torch.empty(n * k * L * 4, dtype=torch.float32, device="cuda")
    ctx.local_grid_device(d_cand, n * k, nr, 0.004, grid, grid32)
    q_r = grid32.double()
    tv = torch.from_numpy(np.repeat(np.arange(n, dtype=np.int32), k * L)).cuda()
    to = torch.arange(n * k * L, dtype=torch.int32, device="cuda")
    out = torch.empty(n * k * L * 4, dtype=torch.float32, device="cuda")
    ctx.set_median(False)
    try:
        ctx.score_trials_device(d_pos, n, q_r, n * k * L, tv, to, n * k * L, out)
    finally:
        ctx.set_median(True)
    C = out.view(n, k, L, 4)[..., 2].cpu().numpy()
    g = grid.view(n, k, L, 4).cpu().numpy()
    for sd in range(n):
        first = [SO.first_max(C[sd, j]) for j in range(k)]
        cbest = np.array([C[sd, j, first[j]] for j in range(k)])
        ref_order = SO.top(np.stack([cbest, cbest, cbest], 1).astype(np.float64), k)
        np.testing.assert_array_equal(od[sd], ref_order)
        np.testing.assert_array_equal(bc[sd], cbest[ref_order])
        np.testing.assert_array_equal(bq[sd], np.array([g[sd, j, first[j]] for j in ref_order]))
        np.testing.assert_array_equal(xx[sd], bq[sd, :2, 1:])
