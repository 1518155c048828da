"""Outer mapping iteration (GrainMapping_fun.m:238-367) on the GPU engine: seeds are drawn,
indexed and grown iteration after iteration until the stop rules hold."""
import numpy as np
import pytest

from grainrecon_b200 import geometry as G
from grainrecon_b200 import mapping as M
from grainrecon_b200 import synth

pytestmark = pytest.mark.gpu

_OPS = [G.quat_to_u(o) for o in G._cubic_ops()]


def _misori_deg(Ua, Ub):
    c = max((np.trace(Ua.T @ Ub @ C) - 1) / 2 for C in _OPS)
    return float(np.degrees(np.arccos(np.clip(c, -1, 1))))


def test_iteration_indexes_the_sample():
    s = synth.make_sample("fe_small", seed=1)
    g = s.geom
    dmap = synth.distance_map(synth.simulate_mask(s))
    dims = s.grain_id.shape
    mask = (s.grain_id > 0).astype(np.float64)
    q_grid = np.concatenate([s.grain_q, G.cubic_fz_orientations(300, 17)]).astype(np.float32)
    ts = {"Center": np.array(s.vol.center), "Dimension": np.array(s.vol.dimension)}
    rvp = np.array([[1, dims[0]], [1, dims[1]], [1, dims[2]]])
    DS, rows, seeds, nvox, frac = M.GrainMapping_iterate(
        mask, {"q": q_grid}, g.rot_det, None, dmap.transpose(2, 1, 0), g.rot_angles, s.S, s.B, s.hkl, len(s.hkl),
        g.theta_max, g.lambda_min, g.lambda_max, g.lss, g.lsd, 0.85, 0.5, 0.5 * g.pxy, g.dety00, g.detz00, g.p0y,
        g.p0z, g.rot_axis_offset, g.pxy, g.pxz, g.detysize / 2 + 0.5, g.detzsize / 2 + 0.5, g.detysize,
        g.detzsize, g.beamstop_y, g.beamstop_z, 0.05, 3, ts, s.vol.vox_size, rvp, s.vol.simap, 10, iter_end=3,
        seed=2, batch=8, max_iter=4)
    assert 1 <= len(frac) <= 4
    assert all(b >= a for a, b in zip(frac, frac[1:]))
    assert frac[-1] > 0.7, frac
    got = DS["GrainId"] > 0
    assert not got[mask == 0].any()
    Ug = [G.quat_to_u(q) for q in s.grain_q]
    eul = DS["EulerZXZ"][:, got]
    for k in range(0, eul.shape[1], 7):
        assert min(_misori_deg(U, G.euler_to_u(*np.radians(eul[:, k]))) for U in Ug) < 1.0
    ids = np.unique(DS["GrainId"][got]).astype(int)
    first = np.concatenate([[1], 1 + np.cumsum([len(p) for p in seeds[:-1]])])
    assert ids.max() < first[-1] + len(seeds[-1])
