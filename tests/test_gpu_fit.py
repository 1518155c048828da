"""GPU spot-centroid fits: tangent Jacobians against the FP64 complex-step oracle and central
finite differences (1e-6 relative), and convergence of the Levenberg-Marquardt fits."""
import numpy as np
import pytest

from grainrecon_b200 import fit as F
from grainrecon_b200 import geometry as G
from grainrecon_b200 import synth
from grainrecon_b200._lib import Context
from oracle import oracle as O

pytestmark = pytest.mark.gpu
REL = 1e-6  # derivative agreement bar


@pytest.fixture(scope="module")
def env():
    import torch
    s = synth.make_sample("fe_small", seed=2)
    ctx = Context(0)
    S9, B9, hkl, rot, R9, p = s.mex_arrays()
    ctx.set_geometry(S9, B9, hkl, rot, R9, p)
    geo = F.geo10_of(s.geom)
    truth = F.random_grains(60, 0.05, 0.1, seed=4)
    d_truth = torch.from_numpy(truth.reshape(-1).copy()).cuda()
    spots = F.simulate_spots(ctx, geo, d_truth, noise_px=0.3, seed=9)
    yield s, ctx, geo, truth, d_truth, spots
    ctx.close()


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("mode", [0, 1])
def test_jacobian_vs_complex_step_oracle(env, mode):
    s, ctx, geo, truth, d_truth, spots = env
    res, jac = F.residual_jacobian(ctx, mode, geo, d_truth, spots)
    res, jac = res.cpu().numpy(), jac.cpu().numpy()
    uvm = spots.uv.cpu().numpy().reshape(-1, 2)
    g = spots.grain.cpu().numpy()
    iw = spots.iw.cpu().numpy()
    ih = spots.ih.cpu().numpy()
    S = G.flat_rowmajor(s.S).astype(np.float64)
    B = G.flat_rowmajor(s.B).astype(np.float64)
    hkl = G.flat_hkl(s.hkl).astype(np.float64).reshape(-1, 3)
    rot = np.asarray(s.geom.rot_angles, np.float32).astype(np.float64)
    p = s.geom.param20(s.nhkl).astype(np.float64)
    rng = np.random.default_rng(0)
    for i in rng.choice(spots.n, 150, replace=False):
        uv, ju, jv = O.fit_uv_jac(mode, truth[g[i]], geo, S, B, hkl[ih[i]], rot[iw[i]], p[8], p[9],
                                  p[10] / 2 + 0.5, p[11] / 2 + 0.5)
        np.testing.assert_allclose(res[i] + uvm[i], uv, rtol=0, atol=1e-7)
        assert _rel(jac[i, 0], ju) < REL and _rel(jac[i, 1], jv) < REL, (i, jac[i], ju, jv)


@pytest.mark.parametrize("mode", [0, 1])
def test_jacobian_vs_central_differences(env, mode):
    import torch
    s, ctx, geo, truth, d_truth, spots = env
    _, jac = F.residual_jacobian(ctx, mode, geo, d_truth, spots)
    jac = jac.cpu().numpy()
    K = jac.shape[2]
    fd = np.zeros_like(jac)
    for k in range(K):
        h = 1e-6 * (1.0 if mode == 0 or k in (4, 5, 6) else 10.0)
        if mode == 0:
            a, b = truth.copy(), truth.copy()
            a[:, k] += h
            b[:, k] -= h
            ra, _ = F.residual_jacobian(ctx, 0, geo, torch.from_numpy(a.reshape(-1).copy()).cuda(), spots)
            rb, _ = F.residual_jacobian(ctx, 0, geo, torch.from_numpy(b.reshape(-1).copy()).cuda(), spots)
        else:
            a, b = geo.copy(), geo.copy()
            a[k] += h
            b[k] -= h
            ra, _ = F.residual_jacobian(ctx, 1, a, d_truth, spots)
            rb, _ = F.residual_jacobian(ctx, 1, b, d_truth, spots)
        fd[:, :, k] = ((ra - rb) / (2 * h)).cpu().numpy()
    scale = np.abs(jac).max(axis=(0, 1))
    err = np.abs(fd - jac).max(axis=(0, 1)) / scale
    assert np.all(err < REL), err


def test_grain_lm_converges_below_0p1_px(env):
    import torch
    s, ctx, geo, truth, d_truth, spots = env
    start = F.perturb_grains(truth, 1.0, 0.005, seed=5)
    d = torch.from_numpy(start.reshape(-1).copy()).cuda()
    lam = torch.full((len(truth),), 1e-3, dtype=torch.float64, device="cuda")
    rms0 = F.grains_rms(ctx, geo, d, d_truth, spots).cpu().numpy()
    assert rms0.min() > 1.0
    for _ in range(12):
        if F.grains_lm(ctx, geo, d, spots, lam, 1) == 0:
            break
    rms = F.grains_rms(ctx, geo, d, d_truth, spots).cpu().numpy()
    assert np.all(rms < 0.1), rms.max()


def test_grain_nm_baseline_reduces_residual(env):
    import torch
    s, ctx, geo, truth, d_truth, spots = env
    n = 8
    sub_off = spots.offsets[: n + 1]
    sub = F.Spots(spots.grain, spots.iw, spots.ih, spots.uv, sub_off)
    start = F.perturb_grains(truth, 1.0, 0.005, seed=6)
    d = torch.from_numpy(start.reshape(-1).copy()).cuda()
    rms0 = F.grains_rms(ctx, geo, d, d_truth, spots).cpu().numpy()[:n]
    hw = np.array([0.03, 0.03, 0.03, 0.02, 0.02, 0.02])
    F.grains_nm(ctx, geo, d, sub, hw, max_evals=1500)
    rms = F.grains_rms(ctx, geo, d, d_truth, spots).cpu().numpy()[:n]
    assert np.all(rms < rms0)


def test_geometry_lm_multistart(env):
    import torch
    s, ctx, geo, truth, d_truth, spots = env
    rng = np.random.default_rng(3)
    starts = np.repeat(geo[None], 4, 0)
    starts[:, 0:2] += rng.uniform(-0.3, 0.3, (4, 2))
    starts[:, 2:4] += rng.uniform(-0.5, 0.5, (4, 2))
    starts[:, 4:7] += rng.uniform(-0.5, 0.5, (4, 3))
    d_s = torch.from_numpy(starts.reshape(-1).copy()).cuda()
    lam = torch.full((4,), 1e-3, dtype=torch.float64, device="cuda")
    for _ in range(40):
        if F.geometry_lm(ctx, d_s, d_truth, spots, lam, 1) == 0:
            break
    rms = F.geometry_rms(ctx, d_s, geo, d_truth, spots).cpu().numpy()
    assert np.all(rms < 0.1), rms


def test_batched_nelder_mead_geometry_decreases(env):
    import torch
    s, ctx, geo, truth, d_truth, spots = env
    starts = np.repeat(geo[None], 3, 0)
    starts[:, 1] += np.array([0.2, -0.2, 0.1])
    lb = geo - np.array([0.5, 0.5, 0.7, 0.7, 1, 1, 1, 0.05, 0.05, 0.05])
    ub = geo + np.array([0.5, 0.5, 0.7, 0.7, 1, 1, 1, 0.05, 0.05, 0.05])

    def f(x):
        return F.geometry_cost(ctx, torch.from_numpy(np.ascontiguousarray(x).reshape(-1)).cuda(), d_truth,
                               spots).cpu().numpy()

    nm = F.BatchedNelderMead(f, starts, lb, ub)
    f0 = nm.F.min(1).copy()
    for _ in range(30):
        nm.step()
    assert np.all(nm.F.min(1) <= f0) and np.any(nm.F.min(1) < f0)


def test_completeness_with_fitted_geometry_matches_oracle(env):
    """Fit the 10 geometry parameters, then score completeness with the fitted geometry: the
    CUDA scorer and the oracle agree bit-exactly on every edge-free trial, and the ground-truth
    orientation of each voxel's grain stays (almost) complete."""
    import torch
    s, ctx, geo, truth, d_truth, spots = env
    start = geo.copy()
    start[0:2] += (0.2, -0.15)
    start[2:4] += (0.3, -0.2)
    start[4:7] += (0.3, -0.2, 0.25)
    d_s = torch.from_numpy(start.copy()).cuda()
    lam = torch.full((1,), 1e-3, dtype=torch.float64, device="cuda")
    for _ in range(40):
        if F.geometry_lm(ctx, d_s, d_truth, spots, lam, 1) == 0:
            break
    fitted = d_s.cpu().numpy()
    assert F.geometry_rms(ctx, d_s, geo, d_truth, spots).cpu().numpy()[0] < 0.1
    dmap = synth.distance_map(synth.simulate_mask(s))
    gf = F.geometry_with(s.geom, fitted)
    S9, B9, hkl, rot, _, _ = s.mex_arrays()
    R9, p = G.flat_rowmajor(gf.rot_det), gf.param20(s.nhkl)
    q = np.concatenate([s.grain_q, G.cubic_fz_orientations(500, 31)]).astype(np.float32)
    idx = s.voxel_indices()
    rng = np.random.default_rng(11)
    for v in idx[rng.choice(len(idx), 3, replace=False)]:
        pos = s.vol.pos_of_index(v).astype(np.float32)
        gpu = ctx.forward_comp(pos, q, S9, B9, hkl, dmap, rot, R9, p).reshape(-1, 4)
        ref, _, edges = O.orientation_scan(pos, q, S9, B9, hkl, dmap, rot, R9, p, tight=True)
        ref = ref.reshape(-1, 4)
        clean = edges == 0
        assert clean.sum() > len(q) // 2
        np.testing.assert_array_equal(gpu[clean, :3], ref[clean, :3])
        np.testing.assert_allclose(gpu[clean, 3], ref[clean, 3], rtol=1e-6)
        d = np.abs(gpu[~clean, :2] - ref[~clean, :2]).max(axis=1)
        assert np.all(d <= edges[~clean])
        assert gpu[s.grain_id[tuple(v - 1)] - 1, 2] >= 0.9
