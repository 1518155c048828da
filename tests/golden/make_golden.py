"""Generate tests/golden/forward_comp_fe_tiny.npz.

The MATLAB reference cannot run here, so the expected values come from
oracle/matlab_port.py -- a statement-by-statement numpy transliteration of
forward_comp.m -- on a small seeded synthetic BCC-Fe sample.  Inputs are stored in
the MEX layouts (float32); the spot mask is stored bit-packed and the distance map
is rebuilt from it with an exact EDT (synth.distance_map) by the tests.

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from grainrecon_b200 import geometry as G  # noqa: E402
from grainrecon_b200 import synth  # noqa: E402
from oracle import matlab_port as MP  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "forward_comp_fe_tiny.npz")


def grow_rule(C, I, mask, dmed_row, med, seed_comp, drop_off, max_dmed):
    """grow_indexed_region_parallel.m:78-88 without the Ninter clause (GPU row layout)."""
    with np.errstate(invalid="ignore", divide="ignore"):
        cand = (mask > 0) & (C > I) & (med <= np.fmin(dmed_row, max_dmed))
        return (cand & (C >= seed_comp * (1 - drop_off))).astype(np.float32)


def main():
    s = synth.make_sample("fe_tiny", seed=3, beamstop_y=(60.0, 66.0), beamstop_z=(60.0, 70.0))
    mask = synth.simulate_mask(s)
    dmap = synth.distance_map(mask)
    S9, B9, hkl, rot, R9, param = s.mex_arrays()
    idx = s.voxel_indices()
    rng = np.random.default_rng(11)
    vsel = idx[rng.choice(len(idx), 3, replace=False)]
    pos = s.vol.pos_of_index(vsel).astype(np.float32)
    q = np.concatenate([s.grain_q, G.cubic_fz_orientations(40, 21)]).astype(np.float32)
    exp = np.zeros((len(pos), len(q), 4), np.float32)
    edges = np.zeros((len(pos), len(q)), np.int32)
    for i, p in enumerate(pos):
        for j, qq in enumerate(q):
            U = G.quat_to_u(qq.astype(np.float64))
            ns, ni, med, ne = MP.forward_comp_mex_args(U, p, S9, B9, hkl, dmap, rot, R9, param)
            exp[i, j] = [ns, ni, np.float32(ni / ns) if ns else np.nan, med]
            edges[i, j] = ne
    # grow case: every voxel of the sample against grain 1's orientation
    gid = s.grain_id[idx[:, 0] - 1, idx[:, 1] - 1, idx[:, 2] - 1]
    rows6 = np.zeros((len(idx), 6), np.float32)
    rows6[:, :3] = idx
    rows6[:, 3] = rng.uniform(0, 0.6, len(idx)).astype(np.float32)
    rows6[:, 4] = (rng.random(len(idx)) > 0.1).astype(np.float32)
    rows6[:, 5] = rng.uniform(0.5, 8, len(idx)).astype(np.float32)
    U1 = G.quat_to_u(s.grain_q[0].astype(np.float32).astype(np.float64))
    param1 = s.vol.param14(seed_comp=0.9, drop_off=0.3, max_dmedian=5.0)
    gexp = np.zeros((len(idx), 7), np.float32)
    gedges = np.zeros(len(idx), np.int32)
    p1 = param1.astype(np.float64)
    for i, r in enumerate(rows6):
        pp = ((r[:3].astype(np.float64) + p1[0:3] - 1) - p1[8:11] / 2) * p1[4] + p1[5:8]
        if p1[3] == 1:
            pp[0], pp[1] = -pp[0], -pp[1]
        ns, ni, med, ne = MP.forward_comp_mex_args(G.flat_rowmajor(U1).astype(np.float64).reshape(3, 3), pp, S9,
                                                   B9, hkl, dmap, rot, R9, param)
        C = ni / ns if ns else np.nan
        flag = grow_rule(C, float(r[3]), float(r[4]), float(r[5]), med, p1[11], p1[12], p1[13])
        gexp[i] = [r[0], r[1], r[2], ns, ni, med, flag]
        gedges[i] = ne
    np.savez_compressed(
        OUT, mask_bits=np.packbits(mask.reshape(-1)), mask_shape=np.array(mask.shape), S9=S9, B9=B9, hkl=hkl,
        rot=rot, R9=R9, param=param, pos=pos, q=q, expected=exp, edges=edges, rows6=rows6, U1=G.flat_rowmajor(U1),
        param1=param1, grow_expected=gexp, grow_edges=gedges, grain_id=gid.astype(np.int32))
    print(OUT, os.path.getsize(OUT), "bytes;", int((exp[..., 2] == 1).sum()), "C=1 trials;",
          int(gexp[:, 6].sum()), "grow flags;", int(edges.sum() + gedges.sum()), "edge reflections")


if __name__ == "__main__":
    main()
