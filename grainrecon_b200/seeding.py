"""Seeding stage of the grain-mapping engine, batched on the GPU.

Mirrors GrainMapping_engine_gpu_comp.m:54-331 and its orientation fit
fit_OR_constrain_with_local_comp_cuda.m:1-185.  Per seed the reference runs, one seed
after the other:

1. the orientation scan ``cuda_forward_comp`` over the whole grid (:74-78);
2. ``sortrows(Output, 3, 'descend')`` and the top ``Nr_seed`` rows (:102-112);
3. a local refine: every candidate's ``ori_local_sampling(q, 8, 0.004)`` grid (730
   orientations) scored in one ``cuda_forward_comp`` call; the best of each grid, sorted
   by completeness (fit_OR_constrain_with_local_comp_cuda.m:12-49,100-112);
4. ``fminsearchbnd`` on 1 - completeness from the best one, ±0.02 on q1..q3, up to 2000
   evaluations of the CPU scorer (:115-126);
5. the Euler-angle round trip and a final scoring of the fitted orientation (:128-153);
6. the accept rule ``C >= minComp and C >= Completeness(seed) and median <= maxDmedian``
   (GrainMapping_engine_gpu_comp.m:180-181), then region growth.

Steps 1-5 depend only on the seed position and the static distance map, so here they run
for a whole batch of seeds at once: one call for the scan and the top-N selection
(grc_seed_candidates_device), one for the local refine of every candidate with its grid
maxima and their order (grc_seed_refine_device, n_seeds x Nr_seed x 730 trials), one
batched Nelder-Mead (every simplex on the device, one scorer launch per step for all
seeds), one final scoring.  Step 6 changes the sample maps and stays sequential:
``GrainMapping_engine_gpu_comp`` commits the batch's results in seed order, discarding a
result whose seed an earlier growth made redundant, and re-indexes a moved centre (the
replace_center loop, :256-300) on the spot.

Scans, sorts, grids and maxima all run in libgrainrecon_b200.so; torch only holds the
device buffers.  The scan and the refine read column 3 only (GrainMapping_engine_gpu_comp.m:103,
fit_OR_constrain_with_local_comp_cuda.m:105), so they run completeness-only on the
bit-packed hit mask; the final scoring computes the median the accept rule reads.
"""
from __future__ import annotations

import math

import numpy as np

from . import geometry as G

NR_LOCAL = 8          # fit_OR_constrain_with_local_comp_cuda.m:20
GRID_LOCAL = 0.004
NR_RECENTRE = 4       # GrainMapping_engine_gpu_comp.m:87 (126 orientations)
FIT_HALF_WIDTH = 0.02  # fit_OR_constrain_with_local_comp_cuda.m:124-125
FIT_MAX_EVALS = 2000   # :120-121 (MaxFunEvals = MaxIter = 2000, TolFun 1e-10; TolX default 1e-4)
FIT_TOL_F = 1e-10
FIT_TOL_X = 1e-4
TRIALS_PER_LAUNCH = 1 << 24


# ---- orientation conversions of the Euler round trip (:128-145) -------------------------------
# Restated from the Aerospace-toolbox semantics of quat2rod / rod2angle / angle2rod / rod2quat.

def quat2rod(q) -> np.ndarray:
    """Rodrigues vector of a quaternion [q0 q1 q2 q3] (normalised first; zero when q0 = 1)."""
    q = np.asarray(q, dtype=np.float64)
    qn = q / math.sqrt(float((q * q).sum()))
    thalf = math.acos(qn[0])
    if thalf == 0:
        return np.zeros(3)
    return qn[1:] / math.cos(thalf)


def rod2angle_zxz(R):
    """ZXZ rotation angles (radians) of a Rodrigues vector."""
    R = np.asarray(R, dtype=np.float64)
    n = math.sqrt(float((R * R).sum()))
    if n == 0:
        return 0.0, 0.0, 0.0
    th = 2 * math.atan(n)
    sx, sy, sz = R / n
    cth, sth = math.cos(th), math.sin(th)
    r11 = sx * sz * (1 - cth) + sy * sth
    r12 = sx * sth - sy * sz * (1 - cth)
    r21 = sz ** 2 + (1 - sz ** 2) * cth
    r31 = sx * sz * (1 - cth) - sy * sth
    r32 = sy * sz * (1 - cth) + sx * sth
    r21 = min(1.0, max(-1.0, r21))
    return math.atan2(r11, r12), math.acos(r21), math.atan2(r31, r32)


def angle2rod_zxz(r1, r2, r3) -> np.ndarray:
    """Rodrigues vector of ZXZ rotation angles (radians)."""
    cps, sps = math.cos(r1), math.sin(r1)
    cth, sth = math.cos(r2), math.sin(r2)
    cph, sph = math.cos(r3), math.sin(r3)
    tr = cph * cps - sph * cth * sps - sph * sps + cph * cth * cps + cth
    r31 = sth * sps - sph * sth
    r23 = cph * sth + sth * cps
    r12 = cph * sps + sph * cth * cps + sph * cps + cph * cth * sps
    th = math.acos(min(1.0, max(-1.0, (tr - 1) / 2)))
    if th == 0:
        return np.zeros(3)
    s2 = 2 * math.sin(th)
    return math.tan(th / 2) * np.array([r23 / s2, r31 / s2, r12 / s2])


def rod2quat(R) -> np.ndarray:
    """Quaternion of a Rodrigues vector (all zeros for a zero vector, as the reference returns)."""
    R = np.asarray(R, dtype=np.float64)
    n = math.sqrt(float((R * R).sum()))
    if n == 0:
        return np.zeros(4)
    thalf = math.atan(n)
    return np.concatenate([[math.cos(thalf)], R * math.sin(thalf) / n])


def fitted_orientation(x):
    """(euler_deg[3], rod[3], quat[4]) of fitted (q1, q2, q3), via the reference's Euler round trip."""
    x = [float(v) for v in x]
    q = np.array([math.sqrt(1 - x[0] ** 2 - x[1] ** 2 - x[2] ** 2), x[0], x[1], x[2]])
    ang = [a * 180 / math.pi for a in rod2angle_zxz(quat2rod(q))]
    ang = [a + 360 if a < 0 else a for a in ang]
    rod = angle2rod_zxz(*(a * math.pi / 180 for a in ang))
    return np.array(ang), rod, rod2quat(rod)


class SeedIndexer:
    """Steps 1-5 of the seeding stage for batches of seeds on one context.

    ``q_grid``: the orientation set (N x 4, [q0 q1 q2 q3]) scored at every seed."""

    def __init__(self, ctx, q_grid, nr_seed: int, fit: bool = True):
        import torch
        self.ctx = ctx
        self.dev = torch.device("cuda", torch.cuda.current_device())
        self.q = torch.as_tensor(np.ascontiguousarray(q_grid, np.float64), device=self.dev)
        self.q32 = self.q.float().contiguous()
        self.nr_seed = int(nr_seed)
        self.fit = fit
        self.stats = {"scan_trials": 0, "local_trials": 0, "fit_seeds": 0, "fit_evals": 0, "final_trials": 0}

    # 1-2. scan of the whole grid (ForwardCalc_OR_space_comp_cuda: float32 pos and q) and the top
    # Nr_seed rows by completeness
    def candidates(self, pos):
        """Scan of every seed (n x 3 mm) against the grid and the first ``nr_seed`` rows of
        sortrows(Output, 3, 'descend') per seed: (n, k, 4) float64 orientations of the grid."""
        import torch
        p = torch.as_tensor(np.ascontiguousarray(pos, np.float32), device=self.dev).reshape(-1, 3).contiguous()
        n, N = p.shape[0], self.q.shape[0]
        k = min(self.nr_seed, N)
        idx = torch.empty(n * k, dtype=torch.int32, device=self.dev)
        cand = torch.empty(n * k * 4, dtype=torch.float64, device=self.dev)
        self.ctx.seed_candidates_device(p, n, self.q32, N, k, idx, cand, None, self.q)
        self.stats["scan_trials"] += n * N
        return cand.view(n, k, 4)

    # 3. local refine of every candidate: each grid's first maximum, candidates in sortrows order
    def refine(self, pos, cand, n_x0: int, nr: int = NR_LOCAL, gridsize: float = GRID_LOCAL):
        """cand: (n, k, 4) float64.  Returns, per seed in sortrows(Output_max, 3, 'descend') order:
        best_q (n, k, 4) float64, best_c (n, k) float32 (NaN for 0/0), order (n, k) int32 (the
        candidate each row came from) and x0 (n, n_x0, 3), the fit's start points."""
        import torch
        n, k = cand.shape[0], cand.shape[1]
        pos32 = np.ascontiguousarray(pos, np.float64).reshape(-1, 3).astype(np.float32).astype(np.float64)
        d_pos = torch.as_tensor(pos32, device=self.dev).contiguous()
        L = (nr + 1) ** 3 + 1
        best_q = torch.empty(n, k, 4, dtype=torch.float64, device=self.dev)
        best_c = torch.empty(n, k, dtype=torch.float32, device=self.dev)
        order = torch.empty(n, k, dtype=torch.int32, device=self.dev)
        x0 = torch.empty(n, n_x0, 3, dtype=torch.float64, device=self.dev)
        per = max(1, TRIALS_PER_LAUNCH // max(1, k * L))
        cand = cand.contiguous()
        for s0 in range(0, n, per):
            s1 = min(n, s0 + per)
            self.ctx.seed_refine_device(d_pos[s0:s1], s1 - s0, cand[s0:s1], k, nr, gridsize, best_q[s0:s1],
                                        best_c[s0:s1], order[s0:s1], n_x0, x0[s0:s1])
            self.stats["local_trials"] += (s1 - s0) * k * L
        return best_q, best_c, order, x0

    # 4. batched fminsearchbnd on 1 - C
    def fit_nm(self, pos, x0):
        import torch
        p = torch.as_tensor(np.ascontiguousarray(pos, np.float64), device=self.dev).reshape(-1, 3).contiguous()
        x0 = x0.reshape(-1, 3).contiguous()
        n = x0.shape[0]
        x = torch.empty(n, 3, dtype=torch.float64, device=self.dev)
        fval = torch.empty(n, dtype=torch.float64, device=self.dev)
        ev = torch.empty(n, dtype=torch.int32, device=self.dev)
        it = torch.empty(n, dtype=torch.int32, device=self.dev)
        fl = torch.empty(n, dtype=torch.int32, device=self.dev)
        self.ctx.fit_orientation_nm(p, x0, n, x, fval, ev, it, fl, FIT_HALF_WIDTH, FIT_MAX_EVALS, FIT_MAX_EVALS,
                                    FIT_TOL_F, FIT_TOL_X)
        self.stats["fit_seeds"] += n
        self.stats["fit_evals"] += int(ev.cpu().numpy().sum())
        return x, fval, ev, it, fl

    # 5. Euler round trip and final scoring (FP64 U, FP64 pos)
    def final(self, pos, x):
        import torch
        xs = x.reshape(-1, 3).cpu().numpy()
        eul, rod, quat = zip(*(fitted_orientation(v) for v in xs))
        quat = np.array(quat)
        p = torch.as_tensor(np.ascontiguousarray(pos, np.float64), device=self.dev).reshape(-1, 3).contiguous()
        qd = torch.as_tensor(quat, device=self.dev).contiguous()
        out = torch.empty(len(xs) * 4, dtype=torch.float32, device=self.dev)
        self.ctx.score_trials_device(p, p.shape[0], qd, qd.shape[0], None, None, len(xs), out)
        self.stats["final_trials"] += len(xs)
        return out.view(-1, 4).cpu().numpy().astype(np.float64), np.array(eul), np.array(rod), quat

    def fit_candidates(self, seed_ids, pos, cand, fit_all: bool = False):
        """fit_OR_constrain_with_local_comp_cuda for a batch: cand (n, k, 4) -> rows (n, 18) and the
        1-based candidate index that gave each row (confident_index_list)."""
        pos = np.asarray(pos, np.float64).reshape(-1, 3)
        n, k = cand.shape[0], cand.shape[1]
        nfit = k if fit_all else 1
        _, _, order, x0 = self.refine(pos, cand, nfit)
        pos_rep = np.repeat(pos, nfit, axis=0)
        if self.fit:
            x, _, _, _, _ = self.fit_nm(pos_rep, x0.reshape(-1, 3))
        else:
            x = x0.reshape(-1, 3)
        out, eul, rod, quat = self.final(pos_rep, x)
        C = out[:, 1] / out[:, 0]                                                   # Nr_intersect / Nr_simu
        rows = np.zeros((n * nfit, 18))
        rows[:, 0] = np.repeat(np.asarray(seed_ids, np.float64), nfit)
        rows[:, 1:4] = pos_rep
        rows[:, 4], rows[:, 5], rows[:, 6], rows[:, 7] = out[:, 0], out[:, 1], C, out[:, 3]
        rows[:, 8:11], rows[:, 11:14], rows[:, 14:18] = eul, rod, quat
        rows = rows.reshape(n, nfit, 18)
        Cs = np.where(np.isnan(rows[:, :, 6]), -np.inf, rows[:, :, 6])
        pick = np.argmax(Cs, axis=1)                                                 # max(indexing_result(:,7))
        cand_id = order[:, :nfit].cpu().numpy()[np.arange(n), pick] + 1
        return rows[np.arange(n), pick], cand_id

    def index(self, seed_ids, pos, fit_all: bool = False):
        """Steps 1-5 for seeds at ``pos`` (n x 3 mm) against the full grid."""
        return self.fit_candidates(seed_ids, pos, self.candidates(pos), fit_all)

    def index_local(self, seed_id, pos, q_center, nr: int = NR_RECENTRE, gridsize: float = GRID_LOCAL):
        """Re-indexing at a moved centre: ori_local_sampling(q, 4) scanned, then steps 2-5."""
        import torch
        qc = torch.as_tensor(np.asarray(q_center, np.float64).reshape(4), device=self.dev)
        L = (nr + 1) ** 3 + 1
        grid = torch.empty(L * 4, dtype=torch.float64, device=self.dev)
        grid32 = torch.empty(L * 4, dtype=torch.float32, device=self.dev)
        self.ctx.local_grid_device(qc, 1, nr, gridsize, grid, grid32)
        p = np.asarray(pos, np.float64).reshape(1, 3)
        d_p = torch.as_tensor(p.astype(np.float32), device=self.dev).reshape(-1)
        k = min(self.nr_seed, L)
        idx = torch.empty(k, dtype=torch.int32, device=self.dev)
        cand = torch.empty(k * 4, dtype=torch.float64, device=self.dev)
        self.ctx.seed_candidates_device(d_p, 1, grid32, L, k, idx, cand, None, grid)
        self.stats["scan_trials"] += L
        return self.fit_candidates([seed_id], p, cand.view(1, k, 4))


# ---- measured spots: pairing and the grain-centre fit ------------------------------------------------

def spot_arrays(Spots, nrot: int):
    """(spots (m x 3) float64 [dety, detz, area], offsets (nrot + 1) int64) from per-projection spot
    tables: either the reference's Spots{i} rows (centroid in columns 9-10, area in column 11,
    get_spots.m:106-109) or (m x 3) arrays [dety, detz, area]."""
    rows, off = [], [0]
    for i in range(nrot):
        a = np.asarray(Spots[i] if i < len(Spots) else np.zeros((0, 3)), np.float64)
        if a.ndim == 1:
            a = a.reshape(-1, 3) if a.size % 3 == 0 and a.size < 11 else a.reshape(1, -1)
        a = a[:, 8:11] if a.shape[1] >= 11 else a[:, :3]
        rows.append(a)
        off.append(off[-1] + len(a))
    sp = np.concatenate(rows) if off[-1] else np.zeros((0, 3))
    return np.ascontiguousarray(sp), np.asarray(off, np.int64)


def pair_spots(ctx, pos, quats, Spots, nrot: int):
    """Pairs of every (pos, quaternion) trial with the measured spots (grc_pair_spots)."""
    import torch
    sp, off = spot_arrays(Spots, nrot)
    d = lambda a: torch.as_tensor(np.ascontiguousarray(a), device="cuda")
    pos = np.asarray(pos, np.float64).reshape(-1, 3)
    q = np.asarray(quats, np.float64).reshape(-1, 4)
    d_sp = d(sp.reshape(-1)) if len(sp) else torch.zeros(3, dtype=torch.float64, device="cuda")
    return ctx.pair_spots(d(pos.reshape(-1)), d(q.reshape(-1)), len(pos), d_sp, len(sp), d(off))


def hitted_spots_rows(pairs, U, pos, hkl, rot_angles):
    """HittedSpots rows of forward_comp_pair_spots.m:78-79: [reshape(U,1,9) pos hkl Energy omega
    exp_y exp_z area dety detz dis] (23 columns)."""
    U = np.asarray(U, np.float64)
    hkl = np.asarray(hkl, np.float64).reshape(-1, 3)
    rows = np.zeros((len(pairs), 23))
    rows[:, 0:9] = U.reshape(3, 3).T.reshape(-1)   # column-major, as reshape(U,1,9)
    rows[:, 9:12] = np.asarray(pos, np.float64)
    rows[:, 12:15] = hkl[pairs["ih"]]
    rows[:, 15] = pairs["energy_kev"]
    rows[:, 16] = np.asarray(rot_angles, np.float64)[pairs["iw"]]
    rows[:, 17], rows[:, 18], rows[:, 19] = pairs["exp_y"], pairs["exp_z"], pairs["area"]
    rows[:, 20], rows[:, 21], rows[:, 22] = pairs["dety"], pairs["detz"], pairs["dis"]
    return rows


def det_tilts(RotDet) -> tuple:
    """Tilts (degrees) with get_det_R.m's RotDet = Rz(tz) Ry(ty) Rx(tx)."""
    R = np.asarray(RotDet, np.float64).reshape(3, 3)
    ty = -math.asin(max(-1.0, min(1.0, R[2, 0])))
    tx = math.atan2(R[2, 1], R[2, 2])
    tz = math.atan2(R[1, 0], R[0, 0])
    return tuple(math.degrees(a) for a in (tx, ty, tz))


def fit_grain_COM(ctx, pairs, pos, quat, geo10, iters: int = 20):
    """Grain centre + orientation from paired spots (replaces fit_grain_COM.m:5-30).

    The reference minimises the mean distance between rounded simulated pixels and the paired
    centroids with Nelder-Mead over (pos, Euler); here Levenberg-Marquardt fits the continuous
    landings (grc_fit_grains_lm) from (pos, quat).  Returns (FitOutput = [pos(3) Euler ZXZ deg(3)],
    RMS residual [pixel], quaternion)."""
    import torch
    from . import fit as F
    m = len(pairs)
    d = lambda a, t: torch.as_tensor(np.ascontiguousarray(a), dtype=t, device="cuda")
    spots = F.Spots(d(np.zeros(m, np.int32), torch.int32), d(pairs["iw"], torch.int32), d(pairs["ih"], torch.int32),
                    d(np.stack([pairs["exp_y"], pairs["exp_z"]], 1).reshape(-1), torch.float64),
                    d(np.array([0, m], np.int64), torch.int64))
    q = np.asarray(quat, np.float64)
    g6 = np.concatenate([F.quat_to_rod(q * np.sign(q[0] if q[0] != 0 else 1.0)), np.asarray(pos, np.float64)])
    d_g = d(g6, torch.float64)
    lam = torch.full((1,), 1e-3, dtype=torch.float64, device="cuda")
    for _ in range(iters):
        if F.grains_lm(ctx, geo10, d_g, spots, lam, 1) == 0:
            break
    g6 = d_g.cpu().numpy()
    res, _ = F.residual_jacobian(ctx, 0, geo10, d_g, spots)
    rms = float(torch.sqrt((res ** 2).sum(1).mean()).item()) if m else float("nan")
    qf = F.rod_to_quat(g6[:3])
    ang = [a * 180 / math.pi for a in rod2angle_zxz(quat2rod(qf))]
    ang = [a + 360 if a < 0 else a for a in ang]
    return np.concatenate([g6[3:6], ang]), rms, qf


def forward_comp_pair_spots(U, proj_bin_bw, Spots, pos, rot_angles, S, B, Ahkl, nrhkl, RotDet, thetamax, lambda_min,
                            lambda_max, Lsam2sou, Lsam2det, minEucDis, dety00, detz00, P0y, P0z, RotAxisOffset,
                            pixelysize, pixelzsize, dety0, detz0, detysize, detzsize, BeamStopY, BeamStopZ):
    """forward_comp_pair_spots.m:3-93: (Nr_simu, Nr_intersect, dis_median, SimuSpots, HittedSpots).

    Counts and median come from the scorer, the pairs from grc_pair_spots; SimuSpots (the list of
    every selected reflection) is not produced (None).  ``minEucDis``, ``dety0`` and ``detz0``
    must equal the scorer's options."""
    import torch
    from . import forward as FW
    ctx = FW.context()
    hkl = FW._hkl(Ahkl, nrhkl)
    param = FW._param(hkl.shape[0], len(rot_angles), Lsam2sou, Lsam2det, P0y, P0z, dety00, detz00, pixelysize,
                      pixelzsize, detysize, detzsize, BeamStopY, BeamStopZ, thetamax, lambda_min, lambda_max,
                      RotAxisOffset)
    ctx.set_geometry(G.flat_rowmajor(S), G.flat_rowmajor(B), G.flat_hkl(hkl), np.asarray(rot_angles, np.float32),
                     G.flat_rowmajor(RotDet), param)
    flat = FW._map_for_call(proj_bin_bw)
    if flat is not None:
        a = np.asarray(proj_bin_bw)
        ctx.upload_masks(flat, a.shape[0], a.shape[1], a.shape[2])
    q = G.u_to_quat(np.asarray(U, np.float64))
    d = lambda a: torch.as_tensor(np.ascontiguousarray(a, np.float64), device="cuda")
    out = torch.empty(4, dtype=torch.float32, device="cuda")
    ctx.score_trials_device(d(np.asarray(pos).reshape(-1)), 1, d(q), 1, None, None, 1, out)
    o = out.cpu().numpy().astype(np.float64)
    pairs = pair_spots(ctx, np.asarray(pos).reshape(1, 3), q.reshape(1, 4), Spots, len(rot_angles))
    return o[0], o[1], o[3], None, hitted_spots_rows(pairs, U, pos, hkl, rot_angles)


# ---- the engine -----------------------------------------------------------------------------------

def pos2ind(pos_indexing, tomo_scale, VoxSize, RecVolumePixel, sz, simap_data_flag):
    """pos2ind.m: 1-based voxel indices of a position [mm], clipped to the volume."""
    p = np.asarray(pos_indexing, np.float64)
    c = np.asarray(tomo_scale["Center"], np.float64)
    d = np.asarray(tomo_scale["Dimension"], np.float64)
    if simap_data_flag == 1:
        pi = np.array([(-p[0] - c[0]) / VoxSize + d[0] / 2, (-p[1] - c[1]) / VoxSize + d[1] / 2,
                       (p[2] - c[2]) / VoxSize + d[2] / 2])
    else:
        pi = (p - c) / VoxSize + d / 2
    pi = np.ceil(pi - np.asarray(RecVolumePixel, np.float64)[:, 0] + 1)
    return np.clip(pi, 1, np.asarray(sz)).astype(np.int64)


def GrainMapping_engine_gpu_comp(pos_list, OR, RotDet, Spots, proj_bin_bw, rot_angles, S, B, Ahkl, nrhkl, thetamax,
                                 lambda_min, lambda_max, Lsam2sou, Lsam2det, TrustComp, minComp, minEucDis, dety00,
                                 detz00, P0y, P0z, RotAxisOffset, pixelysize, pixelzsize, dety0, detz0, detysize,
                                 detzsize, BeamStopY, BeamStopZ, drop_off, maxD, DS, tomo_scale, VoxSize,
                                 RecVolumePixel, FirstGrainID, simap_data_flag, maxDmedian, Nr_seed,
                                 OutputFolder=None, iter=1, check_fit_all=0, batch: int = 64):
    """GrainMapping_engine_gpu_comp.m:11-331 with batched, speculative seed indexing.

    ``OR``: dict with 'q' (N x 4); ``DS``: dict of the sample maps (Mask, Completeness,
    GrainId, Rodrigues 3 x dims, EulerZXZ 3 x dims, IPF001 3 x dims, Dismedian, Ninter,
    VisitFlag, ...), updated copies are returned.  ``Spots``: per projection the measured spots
    (the reference's Spots{i} rows, or [dety, detz, area] rows), or None.  With spots, each new
    seed's orientation is paired with them (grc_pair_spots), the grain centre and orientation are
    fitted to the pairs (``fit_grain_COM``, :126-161) and the growth follows the spot size
    (Spot_L, :201-231: best-first growth for spots of at most 2 px, else growth within a
    bounding volume; without spots Spot_L = 20 px as in the reference).  ``minEucDis``,
    ``dety0`` and ``detz0`` must equal the scorer's options (0.5 px threshold, detector centre);
    ``OutputFolder`` is not written.  Returns (indexing_final (n x 18), pos_list_new (n x 3), DS_out,
    Nr_indexed_voxel (n)).  Runs on the module context of ``grainrecon_b200.forward``, which
    keeps the distance map resident between this engine and the region grower.
    """
    from . import forward as FW
    ctx = FW.context()
    pos_list = np.asarray(pos_list, np.float64).reshape(-1, 3)
    n = len(pos_list)
    DSo = {k: np.array(v, copy=True) for k, v in DS.items()}
    Comp, VisitFlag, GrainId = DSo["Completeness"], DSo["VisitFlag"], DSo["GrainId"]
    Mask = DSo["Mask"]
    sz = Comp.shape
    hkl = FW._hkl(Ahkl, nrhkl)
    param = FW._param(hkl.shape[0], len(rot_angles), Lsam2sou, Lsam2det, P0y, P0z, dety00, detz00, pixelysize,
                      pixelzsize, detysize, detzsize, BeamStopY, BeamStopZ, thetamax, lambda_min, lambda_max,
                      RotAxisOffset)
    ctx.set_geometry(G.flat_rowmajor(S), G.flat_rowmajor(B), G.flat_hkl(hkl), np.asarray(rot_angles, np.float32),
                     G.flat_rowmajor(RotDet), param)
    flat = FW._map_for_call(proj_bin_bw)
    if flat is not None:
        a = np.asarray(proj_bin_bw)
        ctx.upload_masks(flat, a.shape[0], a.shape[1], a.shape[2])
    indexer = SeedIndexer(ctx, OR["q"], Nr_seed)
    indexing_final = np.zeros((n, 18))
    pos_list_new = np.zeros((n, 3))
    Nr_indexed_voxel = np.zeros(n)
    candidate_id = np.zeros(n)
    fit_all_track = np.zeros(n)
    SeedIndexing = np.zeros((n, 15))
    replace_count = np.zeros(n, np.int64)
    spec = {}
    ind_trusted = None

    def trusted_indices():
        idx = np.argwhere(Comp >= TrustComp) + 1
        if len(idx) == 0:
            idx = np.argwhere(Comp >= min(minComp * 1.5, TrustComp * 0.8)) + 1
        return idx

    if check_fit_all == 1:
        ind_trusted = trusted_indices()

    def skip(pi, count):
        c, v = Comp[tuple(pi - 1)], VisitFlag[tuple(pi - 1)]
        return not ((c < TrustComp or (count > 0 and c >= TrustComp)) and v != 1)

    def fit_all_for(pi):
        if check_fit_all != 1 or ind_trusted is None or len(ind_trusted) == 0:
            return False
        return bool(np.min(np.sqrt(((ind_trusted - pi) ** 2).sum(1))) > 2)

    def speculate(i0):
        """Index the next window of seeds that would be processed now, in one batch."""
        ids, fa = [], []
        for j in range(i0, min(n, i0 + batch)):
            if j in spec:
                continue
            pi = pos2ind(pos_list[j], tomo_scale, VoxSize, RecVolumePixel, sz, simap_data_flag)
            if j == i0 or not skip(pi, 0):
                ids.append(j)
                fa.append(fit_all_for(pi))
        for flag in (False, True):
            sel = [j for j, f in zip(ids, fa) if f == flag]
            if sel:
                rows, cid = indexer.index([j + 1 for j in sel], pos_list[sel], fit_all=flag)
                for r, j in enumerate(sel):
                    spec[j] = (rows[r], cid[r], flag)

    spots_pair = {}
    geo10 = np.array([Lsam2sou, Lsam2det, dety00, detz00, *det_tilts(RotDet), P0y, P0z, RotAxisOffset], np.float64)

    def _recentre_on_spots(i, pairs, pos_indexing, pi):
        """:126-161: fit the grain centre to the paired spots and move the seed there when the move
        exceeds maxD voxels and the new voxel is in the mask and less complete."""
        fit_out, _, _ = fit_grain_COM(ctx, pairs, pos_indexing, indexing_final[i, 14:18], geo10)
        if np.sqrt(((fit_out[:3] - indexing_final[i, 1:4]) ** 2).sum()) / VoxSize <= maxD:
            return pos_indexing, pi
        pt = pos2ind(fit_out[:3], tomo_scale, VoxSize, RecVolumePixel, sz, simap_data_flag)
        if not (Comp[tuple(pt - 1)] < indexing_final[i, 6] and Mask[tuple(pt - 1)] == 1):
            return pos_indexing, pi
        eul = fit_out[3:6]
        rod = angle2rod_zxz(*(a * math.pi / 180 for a in eul))
        indexing_final[i, 1:4] = fit_out[:3]
        indexing_final[i, 8:11] = eul
        indexing_final[i, 11:14] = rod
        indexing_final[i, 14:18] = rod2quat(rod)
        import torch
        q = G.u_to_quat(G.euler_to_u(*(a * math.pi / 180 for a in eul)))
        dd = lambda a: torch.as_tensor(np.ascontiguousarray(a, np.float64), device="cuda")
        o = torch.empty(4, dtype=torch.float32, device="cuda")
        ctx.score_trials_device(dd(fit_out[:3]), 1, dd(q), 1, None, None, 1, o)
        o = o.cpu().numpy().astype(np.float64)
        indexing_final[i, 4], indexing_final[i, 5], indexing_final[i, 7] = o[0], o[1], o[3]
        indexing_final[i, 6] = o[1] / o[0] if o[0] > 0 else math.nan
        return fit_out[:3].copy(), pt

    gid_prev = int((DS["GrainId"] > 0).sum())
    for i in range(n):
        stop = False
        pos_indexing = pos_list[i].copy()
        temp = None
        while not stop and replace_count[i] <= 3:
            pi = pos2ind(pos_indexing, tomo_scale, VoxSize, RecVolumePixel, sz, simap_data_flag)
            if not skip(pi, replace_count[i]):
                if replace_count[i] == 0:
                    if i not in spec:
                        speculate(i)
                    row, cid, fa = spec.pop(i)
                    indexing_final[i] = row
                    candidate_id[i] = cid
                    fit_all_track[i] = 1 if fa else 0
                    if Spots is not None:
                        pairs = pair_spots(ctx, pos_indexing, indexing_final[i, 14:18], Spots, len(rot_angles))
                        spots_pair[i] = pairs
                        if len(pairs):
                            pos_indexing, pi = _recentre_on_spots(i, pairs, pos_indexing, pi)
                else:
                    rows, _ = indexer.index_local(i + 1, pos_indexing, temp[14:18])
                    indexing_final[i] = rows[0]
                C, med = indexing_final[i, 6], indexing_final[i, 7]
                if C < minComp or C < Comp[tuple(pi - 1)] or med > maxDmedian:
                    stop = True
                    pos_list_new[i] = pos_indexing
                    VisitFlag[tuple(pi - 1)] = 0.8
                else:
                    temp = indexing_final[i].copy()
                    replace_center = 0
                    if temp[6] >= Comp[tuple(pi - 1)]:
                        Comp[tuple(pi - 1)] = temp[6]
                        UU = G.quat_to_u(temp[14:18])
                        pr = spots_pair.get(i)
                        if pr is not None and len(pr):  # :201-203, bounding half length of the spots
                            a = pr["area"]
                            spot_l = math.sqrt((a.mean() + 2 * (a.std(ddof=1) if len(a) > 1 else 0.0)) / math.pi)
                        else:
                            spot_l = 20.0
                        if spot_l <= 2:  # :207-214, small spots: best-first growth voxel by voxel
                            J, C_out, D_out, N_out, center, replace_center, idx = FW.grow_indexed_region(
                                Comp, Mask, DSo["Dismedian"], DSo["Ninter"], pi, drop_off, maxD, temp[6], UU,
                                proj_bin_bw, rot_angles, S, B, Ahkl, nrhkl, RotDet, thetamax, lambda_min,
                                lambda_max, Lsam2sou, Lsam2det, minEucDis, dety00, detz00, P0y, P0z, RotAxisOffset,
                                pixelysize, pixelzsize, dety0, detz0, detysize, detzsize, BeamStopY, BeamStopZ,
                                RecVolumePixel, tomo_scale, VoxSize, simap_data_flag, maxDmedian)
                        else:  # growth within a bounding volume around the seed
                            J, C_out, D_out, N_out, center, replace_center, idx = FW.grow_indexed_region_cuda(
                                Comp, Mask, DSo["Dismedian"], DSo["Ninter"], pi, spot_l, drop_off, maxD, temp[6],
                                UU, proj_bin_bw, rot_angles, S, B, Ahkl, nrhkl, RotDet, thetamax, lambda_min,
                                lambda_max, Lsam2sou, Lsam2det, dety00, detz00, P0y, P0z, RotAxisOffset, pixelysize,
                                pixelzsize, detysize, detzsize, BeamStopY, BeamStopZ, RecVolumePixel, tomo_scale,
                                VoxSize, simap_data_flag, maxDmedian)
                        ix = tuple((idx - 1).T)
                        Nr_indexed_voxel[i] = len(idx)
                        gid = i + FirstGrainID
                        GrainId[ix] = gid
                        if "Rodrigues" in DSo:
                            DSo["Rodrigues"][(slice(None),) + ix] = temp[11:14, None]
                        if "IPF001" in DSo:
                            DSo["IPF001"][(slice(None),) + ix] = (temp[8:11] / np.linalg.norm(temp[8:11]))[:, None]
                        if "EulerZXZ" in DSo:
                            DSo["EulerZXZ"][(slice(None),) + ix] = temp[8:11, None]
                        VisitFlag[ix] = 0.5
                        VisitFlag[tuple(pi - 1)] = 1
                        Comp[ix] = C_out[ix]
                        DSo["Dismedian"][ix] = D_out[ix]
                        DSo["Ninter"][ix] = N_out[ix]
                        center = np.asarray(center, np.float64)
                        if replace_center == 1 and GrainId[tuple(center.astype(np.int64) - 1)] != gid:
                            # ind2sub(find(GrainId == gid)): column-major order, so the first
                            # nearest voxel is the reference's
                            all_id = np.argwhere(GrainId.transpose(2, 1, 0) == gid)[:, ::-1] + 1
                            center = all_id[np.argmin(np.sqrt(((all_id - center) ** 2).sum(1)))].astype(np.float64)
                            replace_center = 1 if np.sqrt(((center - pi) ** 2).sum()) > maxD else 0
                    if replace_center == 0:
                        stop = True
                        pos_list_new[i] = pos_indexing
                    else:
                        replace_count[i] += 1
                        rvp = np.asarray(RecVolumePixel, np.float64)[:, 0]
                        newp = ((center + rvp - 1) - np.asarray(tomo_scale["Dimension"], np.float64) / 2) * VoxSize \
                            + np.asarray(tomo_scale["Center"], np.float64)
                        if simap_data_flag == 1:
                            newp[0], newp[1] = -newp[0], -newp[1]
                        pos_list_new[i] = newp
                        pos_indexing = newp
            else:
                stop = True
                pos_list_new[i] = pos_indexing
        spec.pop(i, None)
        n_gid = int((GrainId > 0).sum())
        SeedIndexing[i] = [*indexing_final[i, :11], Nr_indexed_voxel[i], n_gid - gid_prev, candidate_id[i],
                           fit_all_track[i]]
        gid_prev = n_gid
        # :300-316: switch the fit-all mode on (and stop early) when seeds stop producing grains
        if check_fit_all != 1 and i + 1 > 200 and np.any(SeedIndexing[i - 180:i + 1, 0] > 0):
            w = SeedIndexing[i - 180:i + 1]
            if (w[:, 12] > 0).sum() / (w[:, 0] > 0).sum() < 0.05:
                check_fit_all = 1
                ind_trusted = np.argwhere(DS["GrainId"] > 0) + 1
                spec.clear()
        if check_fit_all == 1 and i + 1 > 200 and np.any(SeedIndexing[i - 50:i + 1, 0] > 0):
            w = SeedIndexing[i - 50:i + 1]
            if (w[:, 12] > 0).sum() / (w[:, 0] > 0).sum() < 0.05:
                break
    DSo["SeedIndexing"] = SeedIndexing
    DSo["indexer_stats"] = indexer.stats
    DSo["spots_pair"] = spots_pair
    return indexing_final, pos_list_new, DSo, Nr_indexed_voxel
