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
    ctx._check(ctx.L.grc_fit_spot_count(ctx.h, _ptr(geo), _ptr(d_grains), n, _ptr(counts)))
    offsets = torch.zeros(n + 1, dtype=torch.int64, device="cuda")
    offsets[1:] = torch.cumsum(counts, 0)
    ns = int(offsets[-1].item())
    grain = torch.empty(ns, dtype=torch.int32, device="cuda")
    iw = torch.empty(ns, dtype=torch.int32, device="cuda")
    ih = torch.empty(ns, dtype=torch.int32, device="cuda")
    uv = torch.empty(2 * ns, dtype=torch.float64, device="cuda")
    ctx._check(ctx.L.grc_fit_spot_fill(ctx.h, _ptr(geo), _ptr(d_grains), n, _ptr(offsets), _ptr(grain), _ptr(iw),
                                       _ptr(ih), _ptr(uv)))
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
    ctx._check(ctx.L.grc_centroid_residual_adjoint(ctx.h, mode, _ptr(geo), _ptr(d_grains),
                                                   *[_ptr(a) for a in spots.args()], spots.n, _ptr(res), _ptr(jac)))
    return res.view(-1, 2), jac.view(-1, 2, K)


def grains_lm(ctx, geo10, d_grains, spots: Spots, d_lambda, iters: int) -> int:
    """``iters`` Levenberg-Marquardt iterations on every grain (in place); returns #grains improved."""
    import ctypes as C
    from ._lib import _ptr
    geo = np.ascontiguousarray(geo10, dtype=np.float64)
    imp = C.c_int()
    ctx._check(ctx.L.grc_fit_grains_lm(ctx.h, _ptr(geo), _ptr(d_grains), d_grains.numel() // 6,
                                       *[_ptr(a) for a in spots.args()], spots.n, _ptr(spots.offsets),
                                       _ptr(d_lambda), iters, C.byref(imp)))
    return imp.value


def grains_nm(ctx, geo10, d_grains, spots: Spots, half_width, max_evals: int, checkpoint: int = 0, d_trace=None):
    """Forward-only batched Nelder-Mead with the fminsearchbnd sine transform (in place)."""
    from ._lib import _ptr
    geo = np.ascontiguousarray(geo10, dtype=np.float64)
    hw = np.ascontiguousarray(half_width, dtype=np.float64)
    n_ck = 0 if d_trace is None else d_trace.numel() // (6 * (d_grains.numel() // 6))
    ctx._check(ctx.L.grc_fit_grains_nm(ctx.h, _ptr(geo), _ptr(d_grains), d_grains.numel() // 6,
                                       *[_ptr(a) for a in spots.args()], spots.n, _ptr(spots.offsets), _ptr(hw),
                                       max_evals, checkpoint, _ptr(d_trace), n_ck))


def grains_rms(ctx, geo10, d_grains, d_truth, spots: Spots):
    """Per-grain RMS [pixel] of predicted spots vs those of the true parameters (device tensor)."""
    import torch
    from ._lib import _ptr
    n = d_grains.numel() // 6
    rms = torch.empty(n, dtype=torch.float64, device="cuda")
    geo = np.ascontiguousarray(geo10, dtype=np.float64)
    ctx._check(ctx.L.grc_fit_grains_rms(ctx.h, _ptr(geo), _ptr(d_grains), _ptr(d_truth), n,
                                        *[_ptr(a) for a in spots.args()], spots.n, _ptr(spots.offsets), _ptr(rms)))
    return rms


def geometry_lm(ctx, d_starts, d_grains, spots: Spots, d_lambda, iters: int) -> int:
    import ctypes as C
    from ._lib import _ptr
    imp = C.c_int()
    ctx._check(ctx.L.grc_fit_geometry_lm(ctx.h, _ptr(d_starts), d_starts.numel() // 10, _ptr(d_grains),
                                         *[_ptr(a) for a in spots.args()], spots.n, _ptr(d_lambda), iters,
                                         C.byref(imp)))
    return imp.value


def geometry_cost(ctx, d_points, d_grains, spots: Spots):
    """Sum of squared residuals of each 10-parameter geometry point (device, forward only)."""
    import torch
    from ._lib import _ptr
    n = d_points.numel() // 10
    cost = torch.empty(2 * n, dtype=torch.float64, device="cuda")
    ctx._check(ctx.L.grc_fit_geometry_cost(ctx.h, _ptr(d_points), n, _ptr(d_grains),
                                           *[_ptr(a) for a in spots.args()], spots.n, _ptr(cost)))
    return cost.view(-1, 2)[:, 0]


def geometry_rms(ctx, d_starts, geo_truth10, d_grains, spots: Spots):
    import torch
    from ._lib import _ptr
    n = d_starts.numel() // 10
    acc = torch.empty(2 * n, dtype=torch.float64, device="cuda")
    geo = np.ascontiguousarray(geo_truth10, dtype=np.float64)
    ctx._check(ctx.L.grc_fit_geometry_rms(ctx.h, _ptr(d_starts), n, _ptr(geo), _ptr(d_grains),
                                          *[_ptr(a) for a in spots.args()], spots.n, _ptr(acc)))
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
