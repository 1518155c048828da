"""The MATLAB-shaped wrappers of grainrecon_b200.forward against the oracle: same argument lists
as the reference's .m files, map passed as a detz x dety x nrot array.  Bar as in the parity
tests: counts, completeness and decisions bit-exact for rows with no edge reflection."""
import numpy as np
import pytest

from grainrecon_b200 import forward as FW
from grainrecon_b200 import geometry as G
from grainrecon_b200 import synth
from grainrecon_b200._lib import GRC_EINVAL, GrcError
from oracle import oracle as O
from oracle import walk_oracle as WO

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def scene():
    s = synth.make_sample("fe_small", seed=1)
    dmap = synth.distance_map(synth.simulate_mask(s))
    FW.reset_masks()
    return s, dmap, dmap.transpose(2, 1, 0)


def _geo_args(s):
    g = s.geom
    return dict(Lsam2sou=g.lss, Lsam2det=g.lsd, P0y=g.p0y, P0z=g.p0z, RotAxisOffset=g.rot_axis_offset,
                dety00=g.dety00, detz00=g.detz00, pixelysize=g.pxy, pixelzsize=g.pxz, detysize=g.detysize,
                detzsize=g.detzsize, BeamStopY=g.beamstop_y, BeamStopZ=g.beamstop_z, thetamax=g.theta_max,
                lambda_min=g.lambda_min, lambda_max=g.lambda_max)


def _tomo(s):
    dims = s.grain_id.shape
    return ({"Center": np.array(s.vol.center), "Dimension": np.array(s.vol.dimension)},
            np.array([[1, dims[0]], [1, dims[1]], [1, dims[2]]]))


def test_forward_calc_or_space(scene):
    s, dmap, pbb = scene
    g = s.geom
    q = np.concatenate([s.grain_q, G.cubic_fz_orientations(200, 3)]).astype(np.float32)
    v = s.voxel_indices()[10]
    pos = s.vol.pos_of_index(v)
    out = FW.ForwardCalc_OR_space_comp_cuda(pos, q, s.S, s.B, s.hkl, len(s.hkl), pbb, g.rot_angles, g.rot_det,
                                            **_geo_args(s))
    assert out.shape == (len(q), 8)
    np.testing.assert_array_equal(out[:, 4:], q.astype(np.float64))
    S9, B9, hkl, rot, R9, p = s.mex_arrays()
    ref, _, edges = O.orientation_scan(pos.astype(np.float32), q, S9, B9, hkl, dmap, rot, R9, p, tight=True)
    ref = ref.reshape(-1, 4)
    clean = edges == 0
    assert clean.sum() > len(q) // 2
    np.testing.assert_array_equal(out[clean, :3], ref[clean, :3])
    np.testing.assert_allclose(out[clean, 3], ref[clean, 3], rtol=1e-6)


def test_allvoxel_and_grow(scene):
    s, dmap, pbb = scene
    g = s.geom
    dims = s.grain_id.shape
    ts, rvp = _tomo(s)
    S9, B9, hkl, rot, R9, p = s.mex_arrays()
    idx = s.voxel_indices()
    k = 2
    U = G.quat_to_u(s.grain_q[k - 1])
    vox = idx[s.grain_id[tuple((idx - 1).T)] == k][:40]
    I = np.zeros(dims)
    Imask = (s.grain_id > 0).astype(np.float64)
    Dm = np.zeros(dims) + 20
    Ni = np.zeros(dims)
    geo = _geo_args(s)

    def oracle_rows(v, seed_comp, drop_off):
        rows6 = np.zeros((len(v), 6), np.float32)
        rows6[:, :3] = v
        rows6[:, 3] = I[tuple((v - 1).T)]
        rows6[:, 4] = Imask[tuple((v - 1).T)]
        rows6[:, 5] = Dm[tuple((v - 1).T)]
        p1 = np.array([*rvp[:, 0], s.vol.simap, s.vol.vox_size, *s.vol.center, *s.vol.dimension, seed_comp,
                       drop_off, 10], np.float32)
        out, _, edges = O.grow(rows6, G.flat_rowmajor(U), S9, B9, hkl, dmap, rot, R9, p, p1, tight=True)
        return out.reshape(-1, 7), edges

    C_out, D_out, N_out, cmax = FW.Forward_calc_comp_allvoxel_cuda(
        I, Imask, Dm, Ni, vox, 3, U, pbb, g.rot_angles, s.S, s.B, s.hkl, len(s.hkl), g.rot_det, geo["thetamax"],
        geo["lambda_min"], geo["lambda_max"], g.lss, g.lsd, g.dety00, g.detz00, g.p0y, g.p0z, g.rot_axis_offset,
        g.pxy, g.pxz, g.detysize, g.detzsize, g.beamstop_y, g.beamstop_z, rvp, ts, s.vol.vox_size, s.vol.simap, 10)
    ref, edges = oracle_rows(vox, 0.0, 0.0)
    cs = []
    for i, v in enumerate(vox):
        c = C_out[tuple(v - 1)]
        cs.append(c)
        if edges[i] == 0:
            assert c == ref[i, 4] / ref[i, 3]
            assert N_out[tuple(v - 1)] == ref[i, 4]
            np.testing.assert_allclose(D_out[tuple(v - 1)], ref[i, 5], rtol=1e-6)
    assert cmax == np.nanmax(cs)
    # region growth from a seed voxel with the grain's own U
    seed = vox[0]
    J, C2, D2, N2, center, rc, grown = FW.grow_indexed_region_cuda(
        I, Imask, Dm, Ni, seed, 20, 0.05, 3, 0.95, U, pbb, g.rot_angles, s.S, s.B, s.hkl, len(s.hkl), g.rot_det,
        geo["thetamax"], geo["lambda_min"], geo["lambda_max"], g.lss, g.lsd, g.dety00, g.detz00, g.p0y, g.p0z,
        g.rot_axis_offset, g.pxy, g.pxz, g.detysize, g.detzsize, g.beamstop_y, g.beamstop_z, rvp, ts,
        s.vol.vox_size, s.vol.simap, 10)
    assert J.shape == dims and J[tuple(seed - 1)]
    assert len(grown) == int(J.sum()) and len(grown) > 5
    others = np.array([v for v in grown if not np.array_equal(v, seed)])
    ref, edges = oracle_rows(others, 0.95, 0.05)  # every grown voxel passes the oracle's accept rule
    for i, v in enumerate(others):
        if edges[i] == 0:
            assert ref[i, 6] == 1, (v, ref[i])
            assert C2[tuple(v - 1)] == ref[i, 4] / ref[i, 3]
    assert len(center) == 3 and rc in (0, 1)


def test_compete(scene):
    s, dmap, pbb = scene
    g = s.geom
    dims = s.grain_id.shape
    ts, rvp = _tomo(s)
    S9, B9, hkl, rot, R9, p = s.mex_arrays()
    idx = s.voxel_indices()
    rng = np.random.default_rng(2)
    vox = idx[rng.choice(len(idx), 160, replace=False)]
    ng = len(s.grain_q)
    euler = np.degrees(np.array([G.u_to_euler(G.quat_to_u(q)) for q in s.grain_q]))  # degrees, as DS holds
    ids = np.concatenate([rng.permutation(ng) + 1 for _ in vox]).astype(np.float64)
    rng_idx = np.stack([np.arange(len(vox)) * ng + 1, np.arange(len(vox)) * ng + ng], 1).astype(np.float64)
    DS = {"EulerAngle": euler, "Completeness": np.zeros(dims), "GrainId": np.zeros(dims),
          "Dismedian": np.zeros(dims) + 10, "Ninter": np.zeros(dims), "VisitFlag": np.zeros(dims)}
    geo = _geo_args(s)
    DS_out, out = FW.grow_unindexed_compete_comp_cuda(
        DS, vox, ids, rng_idx, pbb, g.rot_angles, s.S, s.B, s.hkl, len(s.hkl), g.rot_det, geo["thetamax"],
        geo["lambda_min"], geo["lambda_max"], g.lss, g.lsd, g.dety00, g.detz00, g.p0y, g.p0z, g.rot_axis_offset,
        g.pxy, g.pxz, g.detysize, g.detzsize, g.beamstop_y, g.beamstop_z, rvp, ts, s.vol.vox_size, s.vol.simap)
    rows5 = np.concatenate([vox, rng_idx], 1).astype(np.float32)
    p1 = np.array([*rvp[:, 0], s.vol.simap, s.vol.vox_size, *s.vol.center, *s.vol.dimension], np.float32)
    ref, _, edges = O.compete(rows5, ids.astype(np.float32), euler.astype(np.float32), S9, B9, hkl, dmap, rot, R9,
                              p, p1, tight=True)
    ref = ref.reshape(-1, 8)
    clean = edges == 0  # edges summed over a row's six candidates
    assert clean.sum() >= 20
    np.testing.assert_array_equal(out[clean, :7], ref[clean, :7])
    np.testing.assert_allclose(out[clean, 7], ref[clean, 7], rtol=1e-6)
    for i, v in enumerate(vox):
        assert DS_out["GrainId"][tuple(v - 1)] == out[i, 4] and DS_out["VisitFlag"][tuple(v - 1)] == 0.5


def test_best_first_growth_matches_oracle_walk(scene):
    """grow_indexed_region (the CPU-path growth: the library's native walk on the GPU scorer)
    against the oracle's numpy walk scored by the FP64 oracle: identical regions, maps and centre."""
    s, dmap, pbb = scene
    g = s.geom
    dims = s.grain_id.shape
    ts, rvp = _tomo(s)
    S9, B9, hkl, rot, R9, p = s.mex_arrays()
    idx = s.voxel_indices()
    k = 3
    U = G.quat_to_u(s.grain_q[k - 1])
    seed = idx[s.grain_id[tuple((idx - 1).T)] == k][5]
    I = np.zeros(dims)
    Imask = (s.grain_id > 0).astype(np.float64)
    Dm = np.zeros(dims) + 20
    Ni = np.zeros(dims)
    geo = _geo_args(s)
    gpu = FW.grow_indexed_region(
        I, Imask, Dm, Ni, seed, 0.05, 3, 0.95, U, pbb, g.rot_angles, s.S, s.B, s.hkl, len(s.hkl), g.rot_det,
        geo["thetamax"], geo["lambda_min"], geo["lambda_max"], g.lss, g.lsd, 0.5 * g.pxy, g.dety00, g.detz00, g.p0y,
        g.p0z, g.rot_axis_offset, g.pxy, g.pxz, g.detysize / 2 + 0.5, g.detzsize / 2 + 0.5, g.detysize, g.detzsize,
        g.beamstop_y, g.beamstop_z, rvp, ts, s.vol.vox_size, s.vol.simap, 10)
    p1 = np.array([*rvp[:, 0], s.vol.simap, s.vol.vox_size, *s.vol.center, *s.vol.dimension, 0, 0, 10], np.float32)
    edges_seen = [0]

    def oracle_score(vox):
        rows6 = np.zeros((len(vox), 6), np.float32)
        rows6[:, :3] = vox
        out, _, edges = O.grow(rows6, G.flat_rowmajor(U), S9, B9, hkl, dmap, rot, R9, p, p1, tight=True)
        edges_seen[0] += int(edges.sum())
        return out.reshape(-1, 7)[:, 3:6]

    ref = WO.best_first_growth(oracle_score, I, Imask, Dm, Ni, seed, 0.05, 3, 0.95, 10)
    J, C, D, N, center, rc, grown = gpu
    assert J[tuple(seed - 1)] and len(grown) > 5
    # no scored voxel holds a reflection within 1e-9 px of a rounding boundary, so the walks must
    # be identical step for step (this is the branch that runs; a tight edge would need a new seed)
    assert edges_seen[0] == 0
    np.testing.assert_array_equal(J, ref[0])
    np.testing.assert_array_equal(grown, ref[6])
    np.testing.assert_array_equal(center, ref[4])
    assert rc == ref[5]
    m = J & (C > 0)
    np.testing.assert_array_equal(C[m], ref[1][m])
    np.testing.assert_array_equal(N[m], ref[3][m])
    np.testing.assert_allclose(D[m], ref[2][m], rtol=1e-6)


def test_native_walk_refuses_a_seed_outside_the_volume(scene):
    s, dmap, pbb = scene
    g = s.geom
    dims = s.grain_id.shape
    ts, rvp = _tomo(s)
    S9, B9, hkl, rot, R9, p = s.mex_arrays()
    Imask = (s.grain_id > 0).astype(np.float64)
    p1 = s.vol.param14(0, 0, 10)
    ctx = FW.context()
    with pytest.raises(GrcError) as e:
        ctx.grow_best_first(np.zeros(dims), Imask, np.zeros(dims) + 20, np.zeros(dims), (dims[0] + 1, 1, 1), 0.05,
                            3, 0.95, 10, G.flat_rowmajor(np.eye(3)), S9, B9, hkl, None, rot, R9, p, p1)
    assert e.value.code == GRC_EINVAL
    seed = s.voxel_indices()[0]  # the context stays usable
    out = ctx.grow_best_first(np.zeros(dims), Imask, np.zeros(dims) + 20, np.zeros(dims), seed, 0.05, 3, 0.95, 10,
                              G.flat_rowmajor(G.quat_to_u(s.grain_q[s.grain_id[tuple(seed - 1)] - 1])), S9, B9, hkl,
                              None, rot, R9, p, p1)
    assert out[0][tuple(seed - 1)] and len(out[6]) >= 1
