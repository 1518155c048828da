"""Spot pairing (grc_pair_spots) against the oracle's restatement of forward_comp_pair_spots.m,
and the grain-centre fit on paired spots.

Measured spots are synthesised: every grain's continuous landings (oracle, FP64) at the grain's
mean voxel position, with Gaussian centroid noise and random areas, plus spurious spots.  Bar:
the pair lists are identical (projection, reflection, paired spot, pixels, centroid, area,
distance value; energy to 1e-12 relative) for every trial whose hits carry no edge reflection."""
import math

import numpy as np
import pytest

from grainrecon_b200 import geometry as G
from grainrecon_b200 import seeding as S
from grainrecon_b200 import synth
from grainrecon_b200._lib import Context, GrcError
from oracle import seed_oracle as SO
from oracle import oracle as O
from spot_fixtures import measured_spots as _measured_spots

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def scene():
    s = synth.make_sample("fe_small", seed=1)
    dmap = synth.distance_map(synth.simulate_mask(s))
    ctx = Context(0)
    S9, B9, hkl, rot, R9, p = s.mex_arrays()
    ctx.set_geometry(S9, B9, hkl, rot, R9, p)
    ctx.upload_masks(dmap.reshape(-1), s.geom.detzsize, s.geom.detysize, s.geom.nrot)
    sc = SO.Scene(S9, B9, hkl, rot, R9, p, dmap)
    yield s, ctx, sc
    ctx.close()


def test_pairs_match_oracle(scene):
    s, ctx, sc = scene
    spots = _measured_spots(s, sc, 0.4, 3)
    off = np.concatenate([[0], np.cumsum([len(a) for a in spots])])
    idx = s.voxel_indices()
    rng = np.random.default_rng(4)
    vox = idx[rng.choice(len(idx), 10, replace=False)]
    pos = s.vol.pos_of_index(vox)
    gid = s.grain_id[tuple((vox - 1).T)]
    quats = np.array([s.grain_q[k - 1] for k in gid], np.float64)
    pairs = S.pair_spots(ctx, pos, quats, spots, s.geom.nrot)
    assert len(pairs) > 100
    assert np.all(np.diff(pairs["trial"].astype(np.int64) * 10 ** 6 + pairs["iw"] * 1000 + pairs["ih"]) > 0)
    n_clean = 0
    for t in range(len(pos)):
        ref, edges = SO.pair_spots(sc, G.quat_to_u(quats[t]), pos[t], spots)
        got = pairs[pairs["trial"] == t]
        if edges:
            continue
        n_clean += 1
        assert len(got) == len(ref), (t, len(got), len(ref))
        for a, r in zip(got, ref):
            iw, ih, j, dety, detz, ey, ez, area, ekev, dis = r
            assert (a["iw"], a["ih"], a["spot"]) == (iw, ih, off[iw] + j)
            assert (a["dety"], a["detz"], a["exp_y"], a["exp_z"], a["area"]) == (dety, detz, ey, ez, area)
            assert a["dis"] == np.float32(dis)
            np.testing.assert_allclose(a["energy_kev"], ekev, rtol=1e-12)
    assert n_clean >= 5


def test_pair_capacity_and_empty_spots(scene):
    import torch
    s, ctx, sc = scene
    pos = s.vol.pos_of_index(s.voxel_indices()[:2])
    q = np.array(s.grain_q[:2], np.float64)
    d = lambda a: torch.as_tensor(np.ascontiguousarray(a), device="cuda")
    empty = [np.zeros((0, 3))] * s.geom.nrot
    assert len(S.pair_spots(ctx, pos, q, empty, s.geom.nrot)) == 0
    spots = _measured_spots(s, sc, 0.0, 5, spurious=0)
    sp, off = S.spot_arrays(spots, s.geom.nrot)
    import ctypes as C
    d_pos, d_q, d_sp, d_off = d(pos.reshape(-1)), d(q.reshape(-1)), d(sp.reshape(-1)), d(off)
    buf = torch.empty(4 * 72, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    n = C.c_int64()
    rc = ctx.L.grc_pair_spots(ctx.h, d_pos.data_ptr(), d_q.data_ptr(), 2, d_sp.data_ptr(), len(sp),
                              d_off.data_ptr(), buf.data_ptr(), 4, C.byref(n))
    assert rc == 2 and n.value > 4  # GRC_ECAPACITY, with the count needed
    full = ctx.pair_spots(d_pos, d_q, 2, d_sp, len(sp), d_off)
    assert len(full) == n.value
    bad = d(np.concatenate([off[:-1], [off[-1] + 1]]))
    with pytest.raises(GrcError):
        ctx.pair_spots(d_pos, d_q, 2, d_sp, len(sp), bad)


def test_forward_comp_pair_spots_wrapper(scene):
    s, ctx, sc = scene
    g = s.geom
    spots = _measured_spots(s, sc, 0.3, 6)
    idx = s.voxel_indices()
    v = idx[len(idx) // 2]
    pos = s.vol.pos_of_index(v)
    U = G.quat_to_u(s.grain_q[s.grain_id[tuple(v - 1)] - 1])
    dmap = sc.dmap
    ns, ni, med, simu, hit = S.forward_comp_pair_spots(
        U, dmap.transpose(2, 1, 0), spots, pos, g.rot_angles, s.S, s.B, s.hkl, len(s.hkl), g.rot_det, g.theta_max,
        g.lambda_min, g.lambda_max, g.lss, g.lsd, 0.5 * g.pxy, g.dety00, g.detz00, g.p0y, g.p0z, g.rot_axis_offset,
        g.pxy, g.pxz, g.detysize / 2 + 0.5, g.detzsize / 2 + 0.5, g.detysize, g.detzsize, g.beamstop_y,
        g.beamstop_z)
    r = sc.score_u(U, pos)
    if r[3] == 0:
        assert (ns, ni) == (r[0], r[1])
    assert hit.shape[1] == 23 and len(hit) > 0
    np.testing.assert_allclose(hit[0, 0:9], U.T.reshape(-1))         # reshape(U,1,9) is column-major
    np.testing.assert_allclose(hit[:, 9:12], np.repeat(pos[None], len(hit), 0))
    assert np.all(np.isin(hit[:, 16], g.rot_angles))
    assert np.all(np.hypot(hit[:, 17] - hit[:, 20], hit[:, 18] - hit[:, 21]) < 15)


def test_grain_centre_fit_recovers_the_grain(scene):
    """Exact centroids of every grain; the fit of one grain starts 4 um and 0.15 deg away.  At
    0.27 mm pixels a simulated pixel sometimes takes a neighbouring centroid (the nearest-spot
    rule of the reference), so the bar is on the recovered parameters, not on a zero residual."""
    s, ctx, sc = scene
    g = s.geom
    k = 1
    spots = _measured_spots(s, sc, 0.0, 7, spurious=0, exact=True)
    idx = s.voxel_indices()
    gid = s.grain_id[tuple((idx - 1).T)]
    pos0 = s.vol.pos_of_index(idx[gid == k + 1]).mean(0)
    q0 = np.asarray(s.grain_q[k], np.float64)
    rng = np.random.default_rng(8)
    ax = rng.normal(size=3)
    ax /= np.linalg.norm(ax)
    a = math.radians(0.15)
    dq = np.array([math.cos(a / 2), *(math.sin(a / 2) * ax)])
    w0, v0 = dq[0], dq[1:]
    w1, v1 = q0[0], q0[1:]
    qs = np.array([w0 * w1 - v0 @ v1, *(w0 * v1 + w1 * v0 + np.cross(v0, v1))])
    ps = pos0 + 0.004 * np.array([0.6, -0.5, 0.62])
    pairs = S.pair_spots(ctx, ps, qs, spots, g.nrot)
    assert len(pairs) > 20
    geo10 = np.array([g.lss, g.lsd, g.dety00, g.detz00, *S.det_tilts(g.rot_det), g.p0y, g.p0z, g.rot_axis_offset])
    fit_out, rms, qf = S.fit_grain_COM(ctx, pairs, ps, qs, geo10)
    U0, Uf = G.quat_to_u(q0), G.euler_to_u(*np.radians(fit_out[3:6]))
    ang = math.degrees(math.acos(min(1.0, (np.trace(U0.T @ Uf) - 1) / 2)))
    dpos = float(np.abs(fit_out[:3] - pos0).max())
    assert rms < 0.1 and ang < 0.01 and dpos < 1e-3, (rms, ang, dpos)
