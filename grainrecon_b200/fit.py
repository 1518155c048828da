"""Spot-centroid fits on the GPU: synthetic matched spots, Levenberg-Marquardt with
tangent-derived Jacobians, and the forward-only Nelder-Mead (fminsearchbnd) baseline.

Replaces the fminsearchbnd fits of fit_grain_COM.m:5-88 / fit_OR_constrain_* (per grain:
Rodrigues vector + centre) and GrainMapping_fit_geo.m / L_shift_tilt_fitting.m:23-50
(detector geometry) with least squares on the continuous landing point; the discrete
completeness stays the accept test (``grainrecon_b200.forward``).
"""
from __future__ import annotations

import math

import numpy as np

from . import geometry as G

GEO_NAMES = ("Lsam2sou", "Lsam2det", "dety00", "detz00", "tilt_x", "tilt_y", "tilt_z", "P0y", "P0z",
             "RotAxisOffset")


def geo10_of(geom: G.Geometry) -> np.ndarray:
    """The 10 fitted geometry parameters of a Geometry (tilts in degrees)."""
    return np.array([geom.lss, geom.lsd, geom.dety00, geom.detz00, *geom.tilt, geom.p0y, geom.p0z,
                     geom.rot_axis_offset], dtype=np.float64)


def geometry_with(geom: G.Geometry, geo10) -> G.Geometry:
    """A copy of ``geom`` carrying the 10 fitted parameters ``geo10``."""
    import dataclasses
    g = [float(v) for v in geo10]
    return dataclasses.replace(geom, lss=g[0], lsd=g[1], dety00=g[2], detz00=g[3], tilt=(g[4], g[5], g[6]),
                               p0y=g[7], p0z=g[8], rot_axis_offset=g[9])


def quat_to_rod(q) -> np.ndarray:
    q = np.asarray(q, dtype=np.float64)
    return q[..., 1:] / q[..., :1]


def rod_to_quat(r) -> np.ndarray:
    r = np.asarray(r, dtype=np.float64)
    q0 = 1.0 / np.sqrt(1.0 + (r * r).sum(-1, keepdims=True))
    return np.concatenate([q0, r * q0], -1)


def random_grains(n: int, radius_mm: float, height_mm: float, seed: int) -> np.ndarray:
    """n grains (rows: Rodrigues(3), centre(3) [mm]) uniform in a cylinder, cubic-FZ orientations."""
    rng = np.random.default_rng(seed)
    rr = radius_mm * np.sqrt(rng.random(n))
    ph = rng.random(n) * 2 * np.pi
    pos = np.stack([rr * np.cos(ph), rr * np.sin(ph), (rng.random(n) - 0.5) * height_mm], 1)
    q = G.cubic_fz_orientations(n, seed + 1)
    return np.concatenate([quat_to_rod(q), pos], 1)


def perturb_grains(grains: np.ndarray, deg: float, shift_mm: float, seed: int) -> np.ndarray:
    """Rotate every grain by ``deg`` about a random axis and move its centre by ``shift_mm``."""
    rng = np.random.default_rng(seed)
    n = len(grains)
    out = grains.copy()
    ax = rng.normal(size=(n, 3))
    ax /= np.linalg.norm(ax, axis=1, keepdims=True)
    dq = np.concatenate([np.full((n, 1), math.cos(math.radians(deg) / 2)), ax * math.sin(math.radians(deg) / 2)], 1)
    q = rod_to_quat(grains[:, :3])
    w1, x1, y1, z1 = dq.T
    w2, x2, y2, z2 = q.T
    qn = np.stack([w1 * w2 - x1 * x2 - y1 * y2 - z1 * z2, w1 * x2 + x1 * w2 + y1 * z2 - z1 * y2,
                   w1 * y2 - x1 * z2 + y1 * w2 + z1 * x2, w1 * z2 + x1 * y2 - y1 * x2 + z1 * w2], 1)
    qn[qn[:, 0] < 0] *= -1
    out[:, :3] = quat_to_rod(qn)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    out[:, 3:] += shift_mm * d
    return out


class Spots:
    """Matched spots on the device (torch tensors): grain, iw, ih (int32), uv (float64, 2 per spot)."""

    def __init__(self, grain, iw, ih, uv, offsets, exact_uv=None):
        self.grain, self.iw, self.ih, self.uv, self.offsets = grain, iw, ih, uv, offsets
        self.exact_uv = exact_uv
        self.n = int(grain.numel())

    def args(self):
        return (self.grain, self.iw, self.ih, self.uv)


def simulate_spots(ctx, geo10, d_grains, noise_px: float, seed: int) -> Spots:
    """Selected landings of every grain at geometry geo10 plus Gaussian centroid noise."""
    import torch
    from ._lib import _ptr
    n = d_grains.numel() // 6
    geo = np.ascontiguousarray(geo10, dtype=np.float64)
    counts = torch.zeros(n, dtype=torch.int64, device="cuda")
    ctx._dev(ctx.L.grc_fit_spot_count, _ptr(geo), _ptr(d_grains), n, _ptr(counts))
    offsets = torch.zeros(n + 1, dtype=torch.int64, device="cuda")
    offsets[1:] = torch.cumsum(counts, 0)
    ns = int(offsets[-1].item())
    grain = torch.empty(ns, dtype=torch.int32, device="cuda")
    iw = torch.empty(ns, dtype=torch.int32, device="cuda")
    ih = torch.empty(ns, dtype=torch.int32, device="cuda")
    uv = torch.empty(2 * ns, dtype=torch.float64, device="cuda")
    ctx._dev(ctx.L.grc_fit_spot_fill, _ptr(geo), _ptr(d_grains), n, _ptr(offsets), _ptr(grain), _ptr(iw),
                                       _ptr(ih), _ptr(uv))
    exact = uv.clone()
    if noise_px > 0:
        gen = torch.Generator(device="cuda").manual_seed(seed)
        uv += noise_px * torch.randn(uv.shape, dtype=torch.float64, device="cuda", generator=gen)
    return Spots(grain, iw, ih, uv, offsets, exact)


def residual_jacobian(ctx, mode: int, geo10, d_grains, spots: Spots):
    """(residuals [n,2], Jacobian [n,2,K]) from grc_centroid_residual_adjoint."""
    import torch
    from ._lib import _ptr
    K = 6 if mode == 0 else 10
    res = torch.empty(2 * spots.n, dtype=torch.float64, device="cuda")
    jac = torch.empty(2 * K * spots.n, dtype=torch.float64, device="cuda")
    geo = np.ascontiguousarray(geo10, dtype=np.float64)
    ctx._dev(ctx.L.grc_centroid_residual_adjoint, mode, _ptr(geo), _ptr(d_grains),
                                                   *[_ptr(a) for a in spots.args()], spots.n, _ptr(res), _ptr(jac))
    return res.view(-1, 2), jac.view(-1, 2, K)


def grains_lm(ctx, geo10, d_grains, spots: Spots, d_lambda, iters: int) -> int:
    """``iters`` Levenberg-Marquardt iterations on every grain (in place); returns #grains improved."""
    import ctypes as C
    from ._lib import _ptr
    geo = np.ascontiguousarray(geo10, dtype=np.float64)
    imp = C.c_int()
    ctx._dev(ctx.L.grc_fit_grains_lm, _ptr(geo), _ptr(d_grains), d_grains.numel() // 6,
                                       *[_ptr(a) for a in spots.args()], spots.n, _ptr(spots.offsets),
                                       _ptr(d_lambda), iters, C.byref(imp))
    return imp.value


def grains_nm(ctx, geo10, d_grains, spots: Spots, half_width, max_evals: int, checkpoint: int = 0, d_trace=None):
    """Forward-only batched Nelder-Mead with the fminsearchbnd sine transform (in place)."""
    from ._lib import _ptr
    geo = np.ascontiguousarray(geo10, dtype=np.float64)
    hw = np.ascontiguousarray(half_width, dtype=np.float64)
    n_ck = 0 if d_trace is None else d_trace.numel() // (6 * (d_grains.numel() // 6))
    ctx._dev(ctx.L.grc_fit_grains_nm, _ptr(geo), _ptr(d_grains), d_grains.numel() // 6,
                                       *[_ptr(a) for a in spots.args()], spots.n, _ptr(spots.offsets), _ptr(hw),
                                       max_evals, checkpoint, _ptr(d_trace), n_ck)


def grains_rms(ctx, geo10, d_grains, d_truth, spots: Spots):
    """Per-grain RMS [pixel] of predicted spots vs those of the true parameters (device tensor)."""
    import torch
    from ._lib import _ptr
    n = d_grains.numel() // 6
    rms = torch.empty(n, dtype=torch.float64, device="cuda")
    geo = np.ascontiguousarray(geo10, dtype=np.float64)
    ctx._dev(ctx.L.grc_fit_grains_rms, _ptr(geo), _ptr(d_grains), _ptr(d_truth), n,
                                        *[_ptr(a) for a in spots.args()], spots.n, _ptr(spots.offsets), _ptr(rms))
    return rms


def geometry_lm(ctx, d_starts, d_grains, spots: Spots, d_lambda, iters: int) -> int:
    import ctypes as C
    from ._lib import _ptr
    imp = C.c_int()
    ctx._dev(ctx.L.grc_fit_geometry_lm, _ptr(d_starts), d_starts.numel() // 10, _ptr(d_grains),
                                         *[_ptr(a) for a in spots.args()], spots.n, _ptr(d_lambda), iters,
                                         C.byref(imp))
    return imp.value


def geometry_cost(ctx, d_points, d_grains, spots: Spots):
    """Sum of squared residuals of each 10-parameter geometry point (device, forward only)."""
    import torch
    from ._lib import _ptr
    n = d_points.numel() // 10
    cost = torch.empty(2 * n, dtype=torch.float64, device="cuda")
    ctx._dev(ctx.L.grc_fit_geometry_cost, _ptr(d_points), n, _ptr(d_grains),
                                           *[_ptr(a) for a in spots.args()], spots.n, _ptr(cost))
    return cost.view(-1, 2)[:, 0]


def geometry_rms(ctx, d_starts, geo_truth10, d_grains, spots: Spots):
    import torch
    from ._lib import _ptr
    n = d_starts.numel() // 10
    acc = torch.empty(2 * n, dtype=torch.float64, device="cuda")
    geo = np.ascontiguousarray(geo_truth10, dtype=np.float64)
    ctx._dev(ctx.L.grc_fit_geometry_rms, _ptr(d_starts), n, _ptr(geo), _ptr(d_grains),
                                          *[_ptr(a) for a in spots.args()], spots.n, _ptr(acc))
    acc = acc.view(-1, 2)
    return torch.sqrt(acc[:, 0] / acc[:, 1])


class BatchedNelderMead:
    """Nelder-Mead on many starting points at once with fminsearchbnd's sine transform.

    The simplex bookkeeping runs on the host (numpy) and every objective evaluation is one
    device launch over all starts (``f`` maps an (n, d) array of points to n values).
    Moves follow fminsearch: reflection 1, expansion 2, contraction 1/2, shrink 1/2."""

    def __init__(self, f, x0, lb, ub):
        self.f, self.lb, self.ub = f, np.asarray(lb, float), np.asarray(ub, float)
        x0 = np.asarray(x0, float)
        n, d = x0.shape
        z0 = np.arcsin(np.clip(2 * (x0 - self.lb) / (self.ub - self.lb) - 1, -1, 1))
        self.S = np.repeat(z0[:, None, :], d + 1, 1)
        for k in range(d):
            self.S[:, k + 1, k] += 0.05 * np.pi / 2  # fminsearchbnd-style initial step in z
        self.F = np.stack([self._f(self.S[:, v]) for v in range(d + 1)], 1)
        self.evals = d + 1

    def x_of(self, z):
        return self.lb + (self.ub - self.lb) * (np.sin(z) + 1) / 2

    def _f(self, z):
        return np.asarray(self.f(self.x_of(z)), float)

    def best(self):
        i = np.argmin(self.F, 1)
        return self.x_of(self.S[np.arange(len(i)), i])

    def step(self):
        n, m, d = self.S.shape
        o = np.argsort(self.F, 1)
        self.S = np.take_along_axis(self.S, o[:, :, None], 1)
        self.F = np.take_along_axis(self.F, o, 1)
        cen = self.S[:, :-1].mean(1)
        zr = 2 * cen - self.S[:, -1]
        fr = self._f(zr)
        self.evals += 1
        exp_ = fr < self.F[:, 0]
        ze = 3 * cen - 2 * self.S[:, -1]
        fe = self._f(ze)
        self.evals += 1
        out = (fr >= self.F[:, -2]) & (fr < self.F[:, -1])
        zc = np.where(out[:, None], 1.5 * cen - 0.5 * self.S[:, -1], 0.5 * cen + 0.5 * self.S[:, -1])
        fc = self._f(zc)
        self.evals += 1
        new = self.S[:, -1].copy()
        fnew = self.F[:, -1].copy()
        a = exp_ & (fe < fr)
        b = exp_ & ~(fe < fr)
        c = ~exp_ & (fr < self.F[:, -2])
        cc = ~exp_ & ~c & (fc < np.where(out, fr, self.F[:, -1]))
        new[a], fnew[a] = ze[a], fe[a]
        new[b], fnew[b] = zr[b], fr[b]
        new[c], fnew[c] = zr[c], fr[c]
        new[cc], fnew[cc] = zc[cc], fc[cc]
        self.S[:, -1], self.F[:, -1] = new, fnew
        shrink = ~(a | b | c | cc)
        if shrink.any():
            for v in range(1, d + 1):
                self.S[shrink, v] = self.S[shrink, 0] + 0.5 * (self.S[shrink, v] - self.S[shrink, 0])
                fv = self._f(self.S[:, v])
                self.evals += 1
                self.F[shrink, v] = fv[shrink]


# ---- benchmarks: time to 0.1 px RMS, Levenberg-Marquardt vs forward-only Nelder-Mead --------

def _pooled_rms(rms, counts):
    rms, counts = np.asarray(rms, float), np.asarray(counts, float)
    ok = np.isfinite(rms)
    return float(np.sqrt((counts[ok] * rms[ok] ** 2).sum() / counts[ok].sum()))


def bench_grain_fit(ctx, geom: G.Geometry, n_grains=5000, noise_px=0.5, deg=1.0, shift_mm=0.005, seed=1,
                    radius_mm=0.05, height_mm=0.1, nm_evals=4000, nm_checkpoint=100, target_px=0.1):
    """Orientation + centre fit of many grains: time to reach ``target_px`` pooled RMS.

    Measured centroids = ground-truth landing + N(0, noise_px); starts rotated by ``deg`` and
    moved by ``shift_mm``.  RMS is the distance of the fitted model's spots from the
    ground-truth spots (the noise floor does not count)."""
    import time

    import torch
    geo = geo10_of(geom)
    truth = random_grains(n_grains, radius_mm, height_mm, seed)
    d_truth = torch.from_numpy(truth.reshape(-1).copy()).cuda()
    spots = simulate_spots(ctx, geo, d_truth, noise_px, seed + 1)
    counts = (spots.offsets[1:] - spots.offsets[:-1]).cpu().numpy()
    start = perturb_grains(truth, deg, shift_mm, seed + 2)
    out = {"grains": n_grains, "spots": spots.n, "noise_px": noise_px, "start": f"{deg} deg, {shift_mm * 1e3} um"}

    d = torch.from_numpy(start.reshape(-1).copy()).cuda()
    lam = torch.full((n_grains,), 1e-3, dtype=torch.float64, device="cuda")
    out["rms_start"] = _pooled_rms(grains_rms(ctx, geo, d, d_truth, spots).cpu().numpy(), counts)
    t_fit, it, hist = 0.0, 0, []
    reached = None
    while it < 30:
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        improved = grains_lm(ctx, geo, d, spots, lam, 1)
        torch.cuda.synchronize()
        t_fit += time.perf_counter() - t0
        it += 1
        r = grains_rms(ctx, geo, d, d_truth, spots).cpu().numpy()
        pr = _pooled_rms(r, counts)
        hist.append(pr)
        if reached is None and pr <= target_px:
            reached = {"seconds": t_fit, "iterations": it, "rms": pr, "frac_grains_below": float((r <= target_px).mean())}
        if improved == 0:
            break
    out["lm"] = {"reached": reached, "final_rms": hist[-1], "iterations_run": it, "seconds_run": t_fit,
                 "rms_history": hist[:12]}

    d = torch.from_numpy(start.reshape(-1).copy()).cuda()
    n_ck = nm_evals // nm_checkpoint
    trace = torch.zeros(n_ck * n_grains * 6, dtype=torch.float64, device="cuda")
    hw = np.array([0.03, 0.03, 0.03, 0.02, 0.02, 0.02])  # fminsearchbnd bounds: ~3.4 deg, 20 um
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    grains_nm(ctx, geo, d, spots, hw, nm_evals, nm_checkpoint, trace)
    torch.cuda.synchronize()
    t_nm = time.perf_counter() - t0
    tr = trace.view(n_ck, n_grains * 6)
    nm_hist, nm_reached = [], None
    for k in range(n_ck):
        r = grains_rms(ctx, geo, tr[k].contiguous(), d_truth, spots).cpu().numpy()
        pr = _pooled_rms(r, counts)
        nm_hist.append(pr)
        if nm_reached is None and pr <= target_px:
            ev = (k + 1) * nm_checkpoint
            nm_reached = {"seconds": t_nm * ev / nm_evals, "evaluations": ev, "rms": pr,
                          "frac_grains_below": float((r <= target_px).mean())}
    out["nm"] = {"reached": nm_reached, "evaluations_run": nm_evals, "seconds_run": t_nm, "final_rms": nm_hist[-1],
                 "rms_every_checkpoint": nm_hist[:: max(1, n_ck // 10)]}
    if reached and nm_reached:
        out["speedup_lm_vs_nm"] = nm_reached["seconds"] / reached["seconds"]
    elif reached:
        out["speedup_lm_vs_nm_lower_bound"] = t_nm / reached["seconds"]
    return out


def bench_geometry_fit(ctx, geom: G.Geometry, n_grains=2000, n_starts=64, noise_px=0.5, seed=1, radius_mm=0.2,
                       height_mm=0.4, nm_iters=400, target_px=0.1):
    """10-parameter geometry fit from ``n_starts`` perturbed starts (+-0.5 mm distances, +-1 deg
    tilts, +-20 px detector offsets, +-0.02 mm source/axis offsets), all in one batch."""
    import time

    import torch
    geo = geo10_of(geom)
    grains = random_grains(n_grains, radius_mm, height_mm, seed)
    d_grains = torch.from_numpy(grains.reshape(-1).copy()).cuda()
    spots = simulate_spots(ctx, geo, d_grains, noise_px, seed + 1)
    rng = np.random.default_rng(seed + 3)
    half = np.array([0.5, 0.5, 20 * geom.pxy, 20 * geom.pxz, 1, 1, 1, 0.02, 0.02, 0.02])
    starts = geo[None] + rng.uniform(-1, 1, (n_starts, 10)) * half
    out = {"grains": n_grains, "spots": spots.n, "starts": n_starts, "noise_px": noise_px,
           "start_spread": dict(zip(GEO_NAMES, half.tolist()))}

    d_s = torch.from_numpy(starts.reshape(-1).copy()).cuda()
    lam = torch.full((n_starts,), 1e-3, dtype=torch.float64, device="cuda")
    rms0 = geometry_rms(ctx, d_s, geo, d_grains, spots).cpu().numpy()
    out["rms_start_median"] = float(np.median(rms0))
    t_fit, it, first, allr, hist = 0.0, 0, None, None, []
    while it < 60:
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        improved = geometry_lm(ctx, d_s, d_grains, spots, lam, 1)
        torch.cuda.synchronize()
        t_fit += time.perf_counter() - t0
        it += 1
        r = geometry_rms(ctx, d_s, geo, d_grains, spots).cpu().numpy()
        hist.append(float(np.median(r)))
        n_ok = int((r <= target_px).sum())
        if first is None and n_ok > 0:
            first = {"seconds": t_fit, "iterations": it}
        if allr is None and n_ok == n_starts:
            allr = {"seconds": t_fit, "iterations": it}
        if improved == 0:
            break
    r = geometry_rms(ctx, d_s, geo, d_grains, spots).cpu().numpy()
    best = d_s.view(n_starts, 10)[int(np.argmin(r))].cpu().numpy()
    out["lm"] = {"first_start_below": first, "all_starts_below": allr, "accepted": int((r <= target_px).sum()),
                 "iterations_run": it, "seconds_run": t_fit, "median_rms_history": hist[:15],
                 "best_rms": float(r.min()), "best": dict(zip(GEO_NAMES, best.tolist()))}

    lb, ub = geo - 1.5 * half, geo + 1.5 * half

    def f(x):
        return geometry_cost(ctx, torch.from_numpy(np.ascontiguousarray(x).reshape(-1)).cuda(), d_grains,
                             spots).cpu().numpy()

    torch.cuda.synchronize()
    t0 = time.perf_counter()
    nm = BatchedNelderMead(f, starts, lb, ub)
    t_nm, nm_first, nm_hist = time.perf_counter() - t0, None, []
    for k in range(nm_iters):
        t0 = time.perf_counter()
        nm.step()
        t_nm += time.perf_counter() - t0
        if (k + 1) % 20 == 0:
            rr = geometry_rms(ctx, torch.from_numpy(nm.best().reshape(-1).copy()).cuda(), geo, d_grains,
                              spots).cpu().numpy()
            nm_hist.append(float(np.median(rr)))
            if nm_first is None and (rr <= target_px).any():
                nm_first = {"seconds": t_nm, "iterations": k + 1, "evaluations": nm.evals}
    out["nm"] = {"first_start_below": nm_first, "iterations_run": nm_iters, "evaluations_run": nm.evals,
                 "seconds_run": t_nm, "median_rms_every_20_iterations": nm_hist}
    if first and nm_first:
        out["speedup_lm_vs_nm"] = nm_first["seconds"] / first["seconds"]
    elif first:
        out["speedup_lm_vs_nm_lower_bound"] = t_nm / first["seconds"]
    out["fitted_geo"] = best
    out["grains_array"] = grains
    return out
