"""CPU restatement of the region walk of grow_indexed_region.m -- TEST INFRASTRUCTURE ONLY.

Only tests/ use this module; the product package never does.  It is the checker of the
library's native walk (grc_walk_best_first / grc_grow_best_first): the same best-first growth
written independently in numpy, with a pluggable scorer (a fake one, the FP64 oracle's, or the
GPU's), so that walks can be compared step for step.  Parity status: unpinned (the MATLAB
reference cannot run here); it follows grow_indexed_region.m:32-137 line by line.
"""
from __future__ import annotations

import numpy as np


def _mround(x):
    """MATLAB round: halves away from zero."""
    x = np.asarray(x, np.float64)
    return np.sign(x) * np.floor(np.abs(x) + 0.5)


_NEIGB = np.array([[1, 1, 0], [1, -1, 0], [1, 0, 1], [1, 0, -1], [1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 1, 1],
                   [0, 0, 1], [0, -1, 1], [0, 1, -1], [0, 0, -1], [0, -1, -1], [-1, 1, 0], [-1, -1, 0], [-1, 0, 1],
                   [-1, 0, -1], [-1, 0, 0]], np.int64)  # grow_indexed_region.m:50-52, 18 neighbours


def best_first_growth(score, I, Imask, DisMedian, Ninter, pos_indices, drop_off, maxD, indexed_comp, maxDmedian,
                      stop_after=None):
    """The region walk of grow_indexed_region.m:6-137 with a pluggable scorer.

    ``score(vox)`` maps (k x 3) 1-based voxel indices to rows [Nr_simu, Nr_intersect, dis_median].
    From the current voxel every unvisited in-mask neighbour is scored (one batch per step; the
    scores do not depend on the region) and kept when it beats the map -- ``C > I`` with
    ``dis_median <= min(DisMedian, maxDmedian)``, or ``|C - I| <= 0.01`` with more
    intersections than ``Ninter`` (:78-79).  The walk then moves to the best kept voxel while its
    completeness stays above ``seed_comp * (1 - drop_off)``.  Returns (J, Completeness_out,
    DisMedian_out, Ninter_out, center, replace_center, indexed_indices)."""
    I = np.array(I, dtype=np.float64, copy=True)
    x, y, z = (int(p) for p in pos_indices)
    I[x - 1, y - 1, z - 1] = indexed_comp
    J = np.zeros(I.shape, np.int8)
    C_out = I.copy()
    D_out = np.array(DisMedian, dtype=np.float64, copy=True)
    N_out = np.array(Ninter, dtype=np.float64, copy=True)
    dims = np.array(I.shape)
    seed_comp = I[x - 1, y - 1, z - 1]
    csum = seed_comp
    cpos = seed_comp * np.array([x, y, z], np.float64)
    center0 = cpos / csum
    n_mask = int((np.asarray(Imask) > 0).sum())
    neg = np.empty((64, 6))  # kept voxels [x y z C dis_median Nr_intersect], first n rows live
    n = 0
    reg_size = 0
    Imask = np.asarray(Imask)
    D_in, N_in = np.asarray(DisMedian, np.float64), np.asarray(Ninter, np.float64)
    while True:
        nb = np.array([x, y, z]) + _NEIGB
        ins = np.all((nb >= 1) & (nb <= dims), axis=1)
        nb = nb[ins]
        keep = (J[tuple((nb - 1).T)] == 0) & (Imask[tuple((nb - 1).T)] > 0)
        nb = nb[keep]
        if len(nb):
            r = np.asarray(score(nb), np.float64).reshape(-1, 3)
            with np.errstate(invalid="ignore", divide="ignore"):
                c = r[:, 1] / r[:, 0]
            ix = tuple((nb - 1).T)
            i0, d0, n0 = I[ix], D_in[ix], N_in[ix]
            # grow_indexed_region.m:78-79; MATLAB min ignores NaN, as np.fmin does
            ok = ((c > i0) & (r[:, 2] <= np.fmin(d0, maxDmedian))) | ((np.abs(c - i0) <= 0.01) & (r[:, 1] > n0))
            k = np.nonzero(ok)[0]
            if len(k):
                if n + len(k) > len(neg):
                    neg = np.concatenate([neg, np.empty((max(len(neg), len(k)), 6))])
                neg[n:n + len(k), :3] = nb[k]
                neg[n:n + len(k), 3] = c[k]
                neg[n:n + len(k), 4] = r[k, 2]
                neg[n:n + len(k), 5] = r[k, 1]
                n += len(k)
                J[tuple((nb[k] - 1).T)] = 1
        J[x - 1, y - 1, z - 1] = 2
        if n == 0:
            break
        dist = neg[:n, 3] / seed_comp
        index = int(np.nanargmax(dist))
        reg_size += 1
        if stop_after is not None and reg_size > stop_after:
            break  # a bounded sample of the walk (timing only): stop after stop_after grown voxels
        if dist[index] > 1 - drop_off and reg_size < n_mask - 1:
            e = neg[index].copy()
            csum += e[3]
            cpos += e[3] * e[:3]
            xi, yi, zi = (int(v) - 1 for v in e[:3])
            C_out[xi, yi, zi], D_out[xi, yi, zi], N_out[xi, yi, zi] = e[3], e[4], e[5]
            x, y, z = xi + 1, yi + 1, zi + 1
            neg[index] = neg[n - 1]  # the last kept voxel takes the chosen one's place
            n -= 1
        else:
            break
    Jb = J > 1
    idx = np.argwhere(Jb.transpose(2, 1, 0))[:, ::-1] + 1
    center1 = cpos / csum
    if np.sqrt(((center1 - center0) ** 2).sum()) > max(maxD, maxD / 10000 * len(idx)):
        center, replace_center = _mround(center1), 1
    else:
        center, replace_center = center0, 0
    return Jb, C_out, D_out, N_out, center, replace_center, idx
