"""CPU restatement of the seeding stage's orientation search -- TEST INFRASTRUCTURE ONLY.

Only tests/ and bench.py's CPU-baseline leg use this module; the product package never
does.  Parity status: unpinned (the MATLAB reference cannot run here).  One seed at a
time, as the reference runs it, on the FP64 C oracle scorer (``oracle.py``):

* ``scan``        -- cuda_forward_comp over a grid (float32 pos and q, as the MEX receives them);
* ``top``         -- sortrows(Output, 3, 'descend') and the first Nr_seed rows
                     (GrainMapping_engine_gpu_comp.m:102-112);
* ``ori_local``   -- ori_local_sampling.m:6-59 (grid, then unique(q,'rows'));
* ``fminsearchbnd`` -- fminsearchbnd.m:126-268 around MATLAB's fminsearch (Nelder-Mead of
                     Lagarias et al. 1998 with reflection 1, expansion 2, contraction 1/2,
                     shrink 1/2, 5 % initial steps), objective fit_OR_fun_local.m:2-98;
* ``euler_roundtrip`` -- fit_OR_constrain_with_local_comp_cuda.m:128-145;
* ``index_seed``  -- fit_OR_constrain_with_local_comp_cuda.m:12-160 for one seed.

Every scorer call also returns the count of edge reflections (landing within 1e-4 px of a
pixel boundary or lambda at the window edge); ``index_seed`` reports whether any trial it
relied on had one, so a test can list such seeds instead of demanding bit-equality.
"""
from __future__ import annotations

import math

import numpy as np

from . import oracle as O


class Scene:
    """MEX-layout scene arrays: S9, B9, hkl, rot, R9, param (float32) and the distance map."""

    def __init__(self, S9, B9, hkl, rot, R9, param, dmap):
        self.S9, self.B9, self.hkl, self.rot, self.R9, self.param, self.dmap = S9, B9, hkl, rot, R9, param, dmap

    def scan(self, pos, q):
        out, edges = O.orientation_scan(np.asarray(pos, np.float32), np.asarray(q, np.float32), self.S9, self.B9,
                                        self.hkl, self.dmap, self.rot, self.R9, self.param)
        return out.reshape(-1, 4).astype(np.float64), edges

    def score_u(self, U, pos):
        """forward_comp with an FP64 U and pos: (Nr_simu, Nr_intersect, dis_median, n_edge)."""
        return O.forward_comp(U, np.asarray(pos, np.float64), self.S9, self.B9, self.hkl, self.dmap, self.rot,
                              self.R9, self.param)


def quat_u(q0, q1, q2, q3):
    """quaternion2U.m / fit_OR_fun_local.m:14-25."""
    return np.array([[2 * (q0 * q0 + q1 * q1) - 1, 2 * (q1 * q2 - q0 * q3), 2 * (q1 * q3 + q0 * q2)],
                     [2 * (q1 * q2 + q0 * q3), 2 * (q0 * q0 + q2 * q2) - 1, 2 * (q2 * q3 - q0 * q1)],
                     [2 * (q1 * q3 - q0 * q2), 2 * (q2 * q3 + q0 * q1), 2 * (q0 * q0 + q3 * q3) - 1]])


def top(out, nr_seed):
    """Row order of sortrows(Output, 3, 'descend'): stable, NaN first; the first nr_seed rows."""
    c = out[:, 2]
    nan = np.isnan(c)
    order = np.concatenate([np.nonzero(nan)[0], np.nonzero(~nan)[0][np.argsort(-c[~nan], kind="stable")]])
    return order[:nr_seed]


def ori_local(q, nr, gridsize=0.004):
    q = np.asarray(q, np.float64)
    rows = [q]
    steps = [k * gridsize - gridsize * nr / 2 for k in range(nr + 1)]
    for sb in steps:
        for sc in steps:
            for sd in steps:
                b, c, d = q[1] + sb, q[2] + sc, q[3] + sd
                rows.append([math.sqrt(1 - (b * b + c * c + d * d)), b, c, d])
    return np.unique(np.array(rows), axis=0)


def first_max(c):
    """MATLAB [~, i] = max(c): NaN ignored, first maximum; index 0 when all are NaN."""
    c = np.where(np.isnan(c), -np.inf, c)
    return int(np.argmax(c))


def _eps(x):
    x = abs(x)
    if not math.isfinite(x):
        return math.nan
    if x < 2.2250738585072014e-308:
        return 5e-324
    m, e = math.frexp(x)
    return math.ldexp(1.0, e - 53)


def _nanmax(vals):
    v = [a for a in vals if not math.isnan(a)]
    return max(v) if v else math.nan


def fminsearchbnd(f, x0, lb, ub, max_evals=2000, max_iter=2000, tol_f=1e-10, tol_x=1e-4):
    """fminsearchbnd with both bounds on every variable.  Returns (x, fval, evals, iters, flag, trace)
    where trace lists every evaluated point's f(x) extra info as returned by ``f``."""
    n = len(x0)
    lb, ub = [float(v) for v in lb], [float(v) for v in ub]

    def xt(z):
        x = []
        for k in range(n):
            t = (math.sin(z[k]) + 1) / 2
            t = t * (ub[k] - lb[k]) + lb[k]
            x.append(max(lb[k], min(ub[k], t)))
        return x

    extra = []

    def F(z):
        val, info = f(xt(z))
        extra.append(info)
        return val

    z0 = []
    for k in range(n):
        if x0[k] <= lb[k]:
            z0.append(-math.pi / 2)
        elif x0[k] >= ub[k]:
            z0.append(math.pi / 2)
        else:
            u = 2 * (x0[k] - lb[k]) / (ub[k] - lb[k]) - 1
            z0.append(2 * math.pi + math.asin(max(-1.0, min(1.0, u))))
    V = [list(z0)]
    for k in range(n):
        y = list(z0)
        y[k] = (1 + 0.05) * y[k] if y[k] != 0 else 0.00025
        V.append(y)
    FV = [F(v) for v in V]

    def srt():
        key = sorted(range(n + 1), key=lambda i: (math.isnan(FV[i]), 0.0 if math.isnan(FV[i]) else FV[i]))
        return [V[i] for i in key], [FV[i] for i in key]

    V, FV = srt()
    evals, iters = n + 1, 1
    flag = 0
    while evals < max_evals and iters < max_iter:
        df = _nanmax([abs(FV[0] - FV[j]) for j in range(1, n + 1)])
        dx = _nanmax([abs(V[j][k] - V[0][k]) for j in range(1, n + 1) for k in range(n)])
        tf = _nanmax([tol_f, 10 * _eps(FV[0])])
        tx = _nanmax([tol_x, 10 * _eps(_nanmax(V[0]))])
        if df <= tf and dx <= tx:
            flag = 1
            break
        xb = [sum(V[j][k] for j in range(n)) / n for k in range(n)]
        w = V[n]
        xr = [2 * xb[k] - 1 * w[k] for k in range(n)]
        fr = F(xr)
        evals += 1
        shrink = False
        if fr < FV[0]:
            xe = [3 * xb[k] - 2 * w[k] for k in range(n)]
            fe = F(xe)
            evals += 1
            V[n], FV[n] = (xe, fe) if fe < fr else (xr, fr)
        elif fr < FV[n - 1]:
            V[n], FV[n] = xr, fr
        elif fr < FV[n]:
            xc = [1.5 * xb[k] - 0.5 * w[k] for k in range(n)]
            fc = F(xc)
            evals += 1
            if fc <= fr:
                V[n], FV[n] = xc, fc
            else:
                shrink = True
        else:
            xcc = [0.5 * xb[k] + 0.5 * w[k] for k in range(n)]
            fcc = F(xcc)
            evals += 1
            if fcc < FV[n]:
                V[n], FV[n] = xcc, fcc
            else:
                shrink = True
        if shrink:
            for j in range(1, n + 1):
                V[j] = [V[0][k] + 0.5 * (V[j][k] - V[0][k]) for k in range(n)]
                FV[j] = F(V[j])
            evals += n
        V, FV = srt()
        iters += 1
    else:
        flag = 0
    return xt(V[0]), FV[0], evals, iters, flag, extra


def euler_roundtrip(x):
    """(euler_deg, rod, quat) of fitted (q1, q2, q3): quat2rod -> rod2angle ZXZ -> degrees in [0, 360)
    -> angle2rod ZXZ -> rod2quat."""
    q = np.array([math.sqrt(1 - x[0] ** 2 - x[1] ** 2 - x[2] ** 2), x[0], x[1], x[2]])
    qn = q / math.sqrt(float(q @ q))
    th = math.acos(qn[0])
    rod = qn[1:] / math.cos(th) if th != 0 else np.zeros(3)
    nr = math.sqrt(float(rod @ rod))
    if nr == 0:
        ang = [0.0, 0.0, 0.0]
    else:
        t = 2 * math.atan(nr)
        sx, sy, sz = rod / nr
        c, s = math.cos(t), math.sin(t)
        a11, a12 = sx * sz * (1 - c) + sy * s, sx * s - sy * sz * (1 - c)
        a21 = min(1.0, max(-1.0, sz ** 2 + (1 - sz ** 2) * c))
        a31, a32 = sx * sz * (1 - c) - sy * s, sy * sz * (1 - c) + sx * s
        ang = [math.atan2(a11, a12), math.acos(a21), math.atan2(a31, a32)]
    ang = [a * 180 / math.pi for a in ang]
    ang = [a + 360 if a < 0 else a for a in ang]
    r1, r2, r3 = (a * math.pi / 180 for a in ang)
    cps, sps, cth, sth, cph, sph = math.cos(r1), math.sin(r1), math.cos(r2), math.sin(r2), math.cos(r3), math.sin(r3)
    tr = cph * cps - sph * cth * sps - sph * sps + cph * cth * cps + cth
    w31, w23 = sth * sps - sph * sth, cph * sth + sth * cps
    w12 = cph * sps + sph * cth * cps + sph * cps + cph * cth * sps
    th2 = math.acos(min(1.0, max(-1.0, (tr - 1) / 2)))
    rod2 = math.tan(th2 / 2) * np.array([w23, w31, w12]) / (2 * math.sin(th2)) if th2 != 0 else np.zeros(3)
    n2 = math.sqrt(float(rod2 @ rod2))
    quat = np.concatenate([[math.cos(math.atan(n2))], rod2 * math.sin(math.atan(n2)) / n2]) if n2 != 0 else np.zeros(4)
    return np.array(ang), rod2, quat


def nm_objective(scene, pos):
    """fit_OR_fun_local: x -> (1 - C, edge count)."""
    def f(x):
        q0 = math.sqrt(1 - (x[0] * x[0] + x[1] * x[1] + x[2] * x[2])) if x[0] * x[0] + x[1] * x[1] + x[2] * x[2] <= 1 \
            else math.nan
        r = scene.score_u(quat_u(q0, x[0], x[1], x[2]), pos)
        val = 1 - r[1] / r[0] if r[0] > 0 else math.nan
        return val, int(r[3])
    return f


def index_seed(scene, pos, q_grid, nr_seed, seed_id=1, fit=True, nr_local=8, grid=0.004, half_width=0.02,
               candidates=None):
    """One seed: (row[18], confident candidate (1-based), edges_seen).  ``candidates`` (k x 4)
    replaces the scan + top step (the re-centring path gives its own 126-orientation scan)."""
    pos = np.asarray(pos, np.float64)
    edges_seen = 0
    if candidates is None:
        out, edges = scene.scan(pos, q_grid)
        sel = top(out, nr_seed)
        edges_seen += int(edges[sel].sum())
        cand = np.asarray(q_grid, np.float64)[sel]
    else:
        cand = np.asarray(candidates, np.float64)
    best = []
    for j, c in enumerate(cand):
        g = ori_local(c, nr_local, grid)
        o, e = scene.scan(pos, g)
        b = first_max(o[:, 2])
        edges_seen += int(e.sum())
        best.append((o[b, 2], g[b], j))
    bc = np.array([b[0] for b in best])
    order = top(np.stack([np.zeros_like(bc), np.zeros_like(bc), bc], 1), len(bc))
    b0 = best[order[0]]
    x0 = b0[1][1:]
    if fit:
        lb = [max(v - half_width, -1.0) for v in x0]
        ub = [min(v + half_width, 1.0) for v in x0]
        x, fval, evals, iters, flag, extra = fminsearchbnd(nm_objective(scene, pos), list(x0), lb, ub)
        edges_seen += sum(extra)
    else:
        x, evals = list(x0), 0
    ang, rod, quat = euler_roundtrip(x)
    r = scene.score_u(quat_u(*quat), pos)
    edges_seen += int(r[3])
    C = r[1] / r[0] if r[0] > 0 else math.nan
    row = np.array([seed_id, *pos, r[0], r[1], C, r[2], *ang, *rod, *quat])
    return row, b0[2] + 1, edges_seen, {"x": np.array(x), "evals": evals}


def pair_spots(scene, U, pos, spots, thr=0.5):
    """forward_comp_pair_spots.m:60-85 for one (U, pos): list of (iw, ih, spot index within the
    projection, dety, detz, exp_y, exp_z, area, energy_kev, dis) and the edge count of the hits.

    ``spots``: per projection an (m x 3) array [dety centroid, detz centroid, area]."""
    rec, _ = O.landings(np.asarray(U, np.float64), np.asarray(pos, np.float64), scene.S9, scene.B9, scene.hkl,
                        scene.dmap, scene.rot, scene.R9, scene.param)
    out, edges = [], 0
    for k in range(len(rec["iw"])):
        if not rec["sel"][k] or not (rec["dis"][k] <= thr):
            continue
        edges += int(rec["edge"][k])
        iw, ih = int(rec["iw"][k]), int(rec["ih"][k])
        dety = float(np.sign(rec["u"][k]) * np.floor(abs(rec["u"][k]) + 0.5))
        detz = float(np.sign(rec["v"][k]) * np.floor(abs(rec["v"][k]) + 0.5))
        sp = np.asarray(spots[iw], np.float64).reshape(-1, 3)
        if len(sp) == 0:
            continue
        d = np.sqrt((sp[:, 0] - dety) ** 2 + (sp[:, 1] - detz) ** 2)
        j = int(np.argmin(d))
        if d[j] < min(math.sqrt(sp[j, 2]), 15.0):
            out.append((iw, ih, j, dety, detz, sp[j, 0], sp[j, 1], sp[j, 2], 12.398 / rec["lam"][k], rec["dis"][k]))
    return out, edges
