"""Host logic of the seeding stage against the oracle's restatement (no GPU needed)."""
import math

import numpy as np

from grainrecon_b200 import geometry as G
from grainrecon_b200 import seeding as S
from oracle import seed_oracle as SO


def test_euler_round_trip_matches_oracle_and_keeps_u():
    rng = np.random.default_rng(0)
    for _ in range(300):
        q = rng.normal(size=4)
        q *= np.sign(q[0]) / np.linalg.norm(q)
        x = q[1:] * rng.uniform(0.1, 0.99)
        ang, rod, quat = S.fitted_orientation(x)
        ang_o, rod_o, quat_o = SO.euler_roundtrip(list(x))
        np.testing.assert_allclose(ang, ang_o, rtol=0, atol=1e-9)
        np.testing.assert_allclose(quat, quat_o, rtol=0, atol=1e-12)
        assert np.all((ang >= 0) & (ang < 360 + 1e-9))
        q0 = math.sqrt(1 - float(x @ x))
        np.testing.assert_allclose(G.quat_to_u(quat), G.quat_to_u(np.array([q0, *x])), atol=1e-12)


def test_oracle_sortrows_and_grid_rules():
    """The oracle's sortrows(.., 'descend') puts NaN first and keeps equal values in order, and its
    ori_local_sampling grid is the host restatement's (the GPU kernels are checked against both in
    tests/test_gpu_select.py)."""
    c = np.array([0.2, np.nan, 0.5, 0.2, np.nan, 0.5, 0.1])
    np.testing.assert_array_equal(SO.top(np.stack([c, c, c], 1), 7), [1, 4, 2, 5, 0, 3, 6])
    q = np.array([0.9, 0.3, -0.2, 0.2])
    q /= np.linalg.norm(q)
    np.testing.assert_array_equal(SO.ori_local(q, 4, 0.004), G.ori_local_sampling(q, 4, 0.004))


def test_oracle_fminsearchbnd_on_a_quadratic():
    target = [0.013, -0.004, 0.007]

    def f(x):
        return sum((a - b) ** 2 for a, b in zip(x, target)), 0

    x, fval, evals, iters, flag, _ = SO.fminsearchbnd(f, [0.0, 0.0, 0.0], [-0.02] * 3, [0.02] * 3, tol_x=1e-8,
                                                      tol_f=1e-14)
    assert flag == 1 and evals < 2000
    np.testing.assert_allclose(x, target, atol=1e-6)


def test_pos2ind_inverts_voxel_positions():
    vol = G.Volume(rec_volume_pixel=(1, 1, 1), simap=1, vox_size=0.005, center=(0.01, -0.02, 0.0),
                   dimension=(20, 20, 20))
    ts = {"Center": np.array(vol.center), "Dimension": np.array(vol.dimension)}
    rvp = np.array([[1, 20], [1, 20], [1, 20]])
    rng = np.random.default_rng(3)
    for _ in range(100):
        idx = rng.integers(1, 21, 3)
        pos = vol.pos_of_index(idx)
        got = S.pos2ind(pos, ts, vol.vox_size, rvp, (20, 20, 20), 1)
        assert np.all(np.abs(got - idx) <= 1) and np.all((got >= 1) & (got <= 20))


def test_seed_positions_keep_their_distance():
    from grainrecon_b200 import mapping as M
    dim = 40
    ax = np.arange(1, dim + 1)
    X, Y, Z = np.meshgrid(ax, ax, ax, indexing="ij")
    inside = (X - 20.5) ** 2 + (Y - 20.5) ** 2 <= 400
    allv = np.argwhere(inside) + 1
    ts = {"Center": np.zeros(3), "Dimension": np.array([dim] * 3)}
    for it in (1, 6, 11):
        pos = M.generate_seeding_indexing_pos(it, allv, ts, 0.005, 0, np.random.default_rng(it))
        vol = M.SEED_VOL_MIN[it - 1]
        dmin = max(0.25 * (3 * vol / (4 * np.pi)) ** (1 / 3) * 2, 3.0)
        idx = pos / 0.005 + dim / 2
        assert len(pos) >= 1 and len(pos) <= max(1, round(len(allv) / vol), round(len(allv) / 8))
        assert np.allclose(idx, np.round(idx))
        d = np.sqrt(((idx[:, None] - idx[None]) ** 2).sum(-1))
        assert len(pos) == 1 or d[np.triu_indices(len(pos), 1)].min() > dmin
        assert {tuple(r) for r in np.round(idx).astype(int)} <= {tuple(r) for r in allv}
    pos = M.generate_seeding_indexing_pos(1, allv, ts, 0.005, 1, np.random.default_rng(0))
    assert np.all(-pos[:, 0] / 0.005 + dim / 2 >= 1)  # the simap frame flips x and y


def test_init_ds_marks_the_sample():
    from grainrecon_b200 import mapping as M
    m = np.zeros((5, 6, 7))
    m[1:4, 2:5, 3:6] = 1
    DS = M.init_DS(m)
    assert DS["VisitFlag"][m > 0].min() == 0 and DS["VisitFlag"][m == 0].max() == -1
    assert DS["Dismedian"][m > 0].min() == 20 and DS["Dismedian"][m == 0].max() == 10
    assert DS["EulerZXZ"].shape == (3, 5, 6, 7)


def test_matlab_round_halves_away_from_zero():
    """round(...) in grow_indexed_region.m:132 and generate_seeding_indexing_pos.m:17-37 takes
    halves away from zero; numpy's round would take them to even."""
    np.testing.assert_array_equal(G.mround([0.5, 1.5, 2.5, -0.5, -2.5, 2.4999, 3.0]), [1, 2, 3, -1, -3, 2, 3])
    assert not np.array_equal(np.round([0.5, 2.5]), G.mround([0.5, 2.5]))
