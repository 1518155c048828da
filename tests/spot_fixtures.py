"""Synthetic measured spots for the pairing and engine tests (not a test module)."""
import numpy as np

from grainrecon_b200 import geometry as G
from oracle import oracle as O


def measured_spots(s, sc, noise_px, seed, spurious=20, exact=False, grains=None, area=(4, 40)):
    rng = np.random.default_rng(seed)
    g = s.geom
    idx = s.voxel_indices()
    gid = s.grain_id[tuple((idx - 1).T)]
    per = [[] for _ in range(g.nrot)]
    for k, q in enumerate(s.grain_q):
        if grains is not None and k not in grains:
            continue
        pos = s.vol.pos_of_index(idx[gid == k + 1]).mean(0)
        rec, _ = O.landings(G.quat_to_u(q), pos, sc.S9, sc.B9, sc.hkl, sc.dmap, sc.rot, sc.R9, sc.param)
        for j in np.nonzero(rec["sel"])[0]:
            u, v = rec["u"][j], rec["v"][j]
            if not exact:
                u, v = u + rng.normal(0, noise_px), v + rng.normal(0, noise_px)
            per[rec["iw"][j]].append((u, v, rng.uniform(*area)))
    for iw in range(g.nrot):
        for _ in range(spurious):
            per[iw].append((rng.uniform(1, g.detysize), rng.uniform(1, g.detzsize), 10.0))
        rng.shuffle(per[iw])
    return [np.array(p, np.float64).reshape(-1, 3) for p in per]
