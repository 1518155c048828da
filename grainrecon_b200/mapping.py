"""Outer grain-mapping iteration around the seeding engine.

Mirrors GrainMapping_fun.m:129-367: the sample maps are initialised from the tomography mask
(:133-157), seed positions are drawn with generate_seeding_indexing_pos.m, and the engine
(``seeding.GrainMapping_engine_gpu_comp``, every scorer call on the GPU) runs iteration after
iteration with the reference's switches -- Nr_seed 400 -> 500 when fewer than a quarter of the
seeds index or after ``iter_end`` iterations, 2500 from iteration 10, the fit-all mode once more
than 95% of the voxels are indexed and the fraction stalls -- until its stop rules hold.  Between
iterations new seeds are drawn from the voxels not yet visited (:322-341), away from the trusted
ones once fewer than 1% (or 30,000) voxels are left.

MATLAB's ``randperm`` is replaced by a seeded numpy generator, so the seed positions follow the
reference's rules but not its random stream.
"""
from __future__ import annotations

import math

import numpy as np

from . import geometry as G

SEED_VOL_MIN = [v ** 3 for v in (45, 40, 35, 30, 25, 22, 19, 16, 13, 10, 6, 3)]  # generate_seeding_indexing_pos.m:2


def _setdiff_rows(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """MATLAB setdiff(a, b, 'rows'): rows of a not in b, unique and sorted."""
    if len(a) == 0:
        return a.reshape(0, 3)
    au = np.unique(a, axis=0)
    if len(b) == 0:
        return au
    bs = {tuple(r) for r in np.asarray(b, np.int64)}
    keep = np.array([tuple(r) not in bs for r in au], bool)
    return au[keep]


def generate_seeding_indexing_pos(it: int, allVoxel_indices, tomo_scale, VoxSize, simap_data_flag,
                                  rng: np.random.Generator):
    """Seed positions [mm] at least dmin voxels apart, drawn from ``allVoxel_indices`` (n x 3,
    1-based, in the full-volume frame) -- generate_seeding_indexing_pos.m:1-107."""
    allv = np.asarray(allVoxel_indices, np.int64).reshape(-1, 3)
    seed_vol_min = SEED_VOL_MIN[min(it, len(SEED_VOL_MIN)) - 1]
    total = len(allv)
    seed_nr = int(G.mround(total / seed_vol_min))
    if seed_nr < 1:
        seed_nr = int(G.mround(total / 8))
    elif seed_nr > 10000:
        seed_nr = 10000
    dseed = (3 * seed_vol_min / (4 * math.pi)) ** (1 / 3) * 2
    dmin = max(0.25 * dseed, 3.0)
    allv = allv[rng.permutation(total)]
    if seed_nr < 1000:
        sampling_nr = min(int(G.mround(seed_nr)), total)
    elif seed_nr < 5000:
        sampling_nr = min(int(G.mround(seed_nr / 3)), total)
    elif seed_nr < 8000:
        sampling_nr = min(int(G.mround(seed_nr / 6)), total)
    else:
        sampling_nr = min(int(G.mround(seed_nr / 50)), total)
    sample = allv[:sampling_nr]
    seeds = [sample[0]]
    temp = []
    pool = _setdiff_rows(sample, np.array(seeds))
    pool = pool[rng.permutation(len(pool))]
    count1 = count2 = 0
    cutoff = 4000
    i = 1

    def refill(c1):
        if sampling_nr * (c1 + 1) < total and 1 + c1 * sampling_nr < total:
            return allv[c1 * sampling_nr:sampling_nr * (c1 + 1)]
        return None

    while i <= seed_nr - 1 and len(pool):
        cand = pool[0]
        cur = np.array(seeds)
        dmin_all = np.sqrt(((cur - cand) ** 2).sum(1)).min()
        if len(cur) > 1:  # pdist over the existing seeds as well
            d = np.sqrt(((cur[:, None, :] - cur[None, :, :]) ** 2).sum(-1))
            dmin_all = min(dmin_all, d[np.triu_indices(len(cur), 1)].min())
        if dmin_all > dmin:
            seeds.append(cand)
            excl = np.array(seeds) if i < cutoff else np.array(temp + seeds)
            pool = _setdiff_rows(sample, excl)
            if len(pool) < 50:
                count1 += 1
                nxt = refill(count1)
                if nxt is None:
                    break
                sample = nxt
                pool = _setdiff_rows(sample, excl)
            i += 1
        else:
            count2 += 1
        if count2 > 30:
            count1 += 1
            nxt = refill(count1)
            if nxt is None:
                break
            sample = nxt
            excl = np.array(seeds) if i < cutoff else np.array(temp + seeds)
            pool = _setdiff_rows(sample, excl)
            count2 = 0
        pool = pool[rng.permutation(len(pool))]
        if i % cutoff == 0:
            temp += seeds[:-1]
            seeds = seeds[-1:]
    seed_list = np.array(temp + seeds if i >= cutoff else seeds, np.float64)
    pos = (seed_list - np.asarray(tomo_scale["Dimension"], np.float64) / 2) * VoxSize + \
        np.asarray(tomo_scale["Center"], np.float64)
    if simap_data_flag == 1:
        pos[:, 0], pos[:, 1] = -pos[:, 0], -pos[:, 1]
    return pos


def init_DS(mask: np.ndarray) -> dict:
    """Sample maps of GrainMapping_fun.m:133-157 for the reconstruction box ``mask`` (1 inside)."""
    dims = mask.shape
    m = mask > 0
    DS = {"PhaseId": m.astype(np.float64), "Mask": m.astype(np.float64), "Completeness": np.zeros(dims),
          "GrainId": np.zeros(dims), "Rodrigues": np.zeros((3,) + dims), "EulerZXZ": np.zeros((3,) + dims),
          "IPF001": np.zeros((3,) + dims), "Dismedian": np.zeros(dims) + 10, "Ninter": np.zeros(dims),
          "Icorr": np.zeros(dims), "VisitFlag": np.zeros(dims) - 1}
    DS["VisitFlag"][m] = 0
    DS["Dismedian"][m] = 20
    return DS


def _index_list(cond: np.ndarray) -> np.ndarray:
    """1-based (x, y, z) of the true voxels in MATLAB find() order (column-major)."""
    return np.argwhere(cond.transpose(2, 1, 0))[:, ::-1] + 1


def GrainMapping_iterate(mask, OR, RotDet, Spots, proj_bin_bw, rot_angles, S, B, Ahkl, nrhkl, thetamax, lambda_min,
                         lambda_max, Lsam2sou, Lsam2det, TrustComp, minComp, minEucDis, dety00, detz00, P0y, P0z,
                         RotAxisOffset, pixelysize, pixelzsize, dety0, detz0, detysize, detzsize, BeamStopY,
                         BeamStopZ, drop_off, maxD, tomo_scale, VoxSize, RecVolumePixel, simap_data_flag, maxDmedian,
                         iter_end: int = 10, seed: int = 0, batch: int = 64, max_iter: int = 30):
    """The iteration of GrainMapping_fun.m:238-367 on the GPU engine.

    ``mask``: the reconstruction box's tomography mask (1 = sample).  Returns (DS, indexing rows of
    every iteration, seed positions of every iteration, indexed voxels per seed, indexed voxel
    fraction per iteration)."""
    from scipy import ndimage

    from .seeding import GrainMapping_engine_gpu_comp
    rng = np.random.default_rng(seed)
    rvp = np.asarray(RecVolumePixel)
    DS = init_DS(mask)
    total = int((DS["Mask"] > 0).sum())
    all_idx = _index_list(DS["Mask"] > 0) + rvp[:, 0] - 1
    all_idx = all_idx[rng.permutation(len(all_idx))]
    pos_seed = generate_seeding_indexing_pos(1, all_idx, tomo_scale, VoxSize, simap_data_flag, rng)
    iter_end = min(iter_end, 10)
    Nr_seed, check_fit_all, it, first_id = 400, 0, 0, 1
    rows_all, seeds_all, nvox_all, frac = [], [], [], []
    while True:
        it += 1
        if it >= 10:
            Nr_seed = 2500
        rows, pos_new, DS_out, nvox = GrainMapping_engine_gpu_comp(
            pos_seed, OR, RotDet, Spots, proj_bin_bw, rot_angles, S, B, Ahkl, nrhkl, thetamax, lambda_min,
            lambda_max, Lsam2sou, Lsam2det, TrustComp, minComp, minEucDis, dety00, detz00, P0y, P0z, RotAxisOffset,
            pixelysize, pixelzsize, dety0, detz0, detysize, detzsize, BeamStopY, BeamStopZ, drop_off, maxD, DS,
            tomo_scale, VoxSize, RecVolumePixel, first_id, simap_data_flag, maxDmedian, Nr_seed, None, it,
            check_fit_all, batch=batch)
        rows_all.append(rows)
        seeds_all.append(pos_new)
        nvox_all.append(nvox)
        indexed = int((DS_out["GrainId"] > 0).sum())
        frac.append(indexed / total)
        tried = rows[:, 6] > 0
        success = (rows[tried, 6] >= minComp).mean() if tried.any() else 0.0
        if (success < 0.25 and Nr_seed < 500) or it >= iter_end:                       # :289-293
            Nr_seed = 500
        if it > 2 and frac[-1] > 0.95 and abs(frac[-1] - frac[-2]) < 0.04:             # :294-305
            check_fit_all = 1
            Nr_seed = max(Nr_seed, 500)
        stop = ((it >= 2 and frac[-1] > 0.999 and abs(frac[-1] - frac[-2]) * total <= 2) or   # :306-309
                (it == 1 and frac[-1] > 0.999) or
                (it >= iter_end and (frac[-1] > 0.995 or total - indexed < 30000)))
        if not stop:
            first_id += len(pos_seed)
            vf = DS_out["VisitFlag"]
            if frac[-1] > 0.99 or total - indexed < 30000:                               # :322-329
                trusted = (DS_out["Completeness"] >= TrustComp) | (vf == 1)
                dist = ndimage.distance_transform_edt(~trusted) if trusted.any() else np.full(vf.shape, np.inf)
                cand = (vf >= 0) & (vf <= 0.5) & (dist >= 3)
            else:
                cand = (vf >= 0) & (vf < 0.5)
            unv = _index_list(cand)
            if len(unv) < total * 0.05:                                                  # :330-334
                unv = _index_list((vf >= 0) & (vf < 0.5))
            if len(unv):
                pos_seed = generate_seeding_indexing_pos(it + 1, unv + rvp[:, 0] - 1, tomo_scale, VoxSize,
                                                         simap_data_flag, rng)
            else:
                stop = True
        DS = {k: v for k, v in DS_out.items() if k in DS}
        if stop or it >= max_iter:
            break
    return DS, rows_all, seeds_all, nvox_all, frac
