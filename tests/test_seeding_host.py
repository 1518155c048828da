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


def test_sortrows_descend_nan_first_matches_oracle():
    import torch
    rng = np.random.default_rng(1)
    for _ in range(200):
        c = rng.integers(0, 6, 64).astype(np.float64) / 5
        c[rng.random(64) < 0.1] = np.nan
        got = S.sort_desc_nan_first(torch.tensor(c)).numpy()[:25]
        ref = SO.top(np.stack([c, c, c], 1), 25)
        np.testing.assert_array_equal(got, ref)


def test_local_grids_order_matches_unique_rows():
    """Same rows in ``unique(q,'rows')`` order; q0 may differ by 1 ulp where torch's CPU sqrt is
    not correctly rounded (b, c, d are exact)."""
    import torch
    rng = np.random.default_rng(2)
    for nr in (4, 8):
        qc = rng.normal(size=(5, 4))
        qc[:, 0] = np.abs(qc[:, 0]) + 1.5  # keep every grid point inside the unit ball
        qc /= np.linalg.norm(qc, axis=1, keepdims=True)
        grids = S.local_grids(torch.tensor(qc), nr, 0.004).numpy()
        assert grids.shape == (5, (nr + 1) ** 3 + 1, 4)
        for g, c in zip(grids, qc):
            ref = SO.ori_local(c, nr, 0.004)

            def twins_out(a):  # the centre and the grid centre, equal up to q0's last bit
                keep = np.ones(len(a), bool)
                keep[1:] = np.abs(a[1:] - a[:-1]).max(1) > 1e-15
                return a[keep]

            g, ref = twins_out(g), twins_out(ref)
            assert g.shape == ref.shape
            np.testing.assert_array_equal(g[:, 1:], ref[:, 1:])
            np.testing.assert_allclose(g[:, 0], ref[:, 0], rtol=0, atol=2.3e-16)
            np.testing.assert_array_equal(twins_out(G.ori_local_sampling(c, nr, 0.004)), ref)


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
