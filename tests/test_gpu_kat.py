"""Known-answer cases on the GPU scorer (through the C ABI), single-reflection geometry:
omega = 0, sample at the origin, untilted 1024 x 1024 detector at 11 mm, 0.05 mm pixels.

* Landing pixel against the closed form.  With a map whose value encodes the pixel
  (value = 1 + flat index), dis_median of a one-reflection trial is the value at the landing
  pixel, so it names the pixel the kernel chose.  The spot lies at Lsd*tan(2 theta) from the
  beam centre along the projected G direction (mirror reflection of k_in = x).
* Each filter rejects on its own: wavelength window, beam stop over the landing pixel (and one
  that misses it by a pixel), detector frame; a spot pixel at the landing point is a hit.
Every case is also checked against the FP64 oracle."""
import math

import numpy as np
import pytest

from grainrecon_b200 import geometry as G
from grainrecon_b200._lib import Context
from oracle import oracle as O

pytestmark = pytest.mark.gpu

N = 1024
PX = 0.05


@pytest.fixture(scope="module")
def ctx():
    c = Context(0)
    yield c
    c.close()


def _setup(hkl_row=(-1, 2, 1), lmin=0.05, lmax=5.0):
    geom = G.Geometry(lss=11.0, lsd=11.0, pxy=PX, pxz=PX, detysize=N, detzsize=N, tilt=(0, 0, 0),
                      rot_angles=np.array([0.0]), e_min_kev=G.HC_KEV_A / lmax, e_max_kev=G.HC_KEV_A / lmin)
    B = G.form_b((3.0, 3.0, 3.0, 90, 90, 90))
    hkl = np.array([hkl_row], dtype=np.float64)
    args = (G.flat_rowmajor(np.eye(3)), G.flat_rowmajor(B), G.flat_hkl(hkl))
    return geom, B, hkl, args


def _random_quats(n, seed):
    q = np.random.default_rng(seed).standard_normal((n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    q[q[:, 0] < 0] *= -1
    return q.astype(np.float32)


def _closed_form(q, B9, h, lmin=0.05, lmax=5.0):
    """(selected, u, v) of the single reflection at omega = 0 in FP64 from the float32 inputs."""
    Bm = np.asarray(B9, np.float64).reshape(3, 3)
    sel, us, vs = [], [], []
    for qi in q.astype(np.float64):
        Gv = G.quat_to_u(qi) @ Bm @ h
        g = Gv / np.linalg.norm(Gv)
        lam = 2 * (2 * math.pi / np.linalg.norm(Gv)) * -g[0]  # lambda = 2 d sin(theta), sin(theta) = -cos(beta)
        if not (g[0] < 0 and lmin < lam < lmax):  # beta > 90 deg and inside the wavelength window
            sel.append(False), us.append(np.nan), vs.append(np.nan)
            continue
        two_theta = 2 * (math.acos(g[0]) - math.pi / 2)
        r = 11.0 * math.tan(two_theta)
        ey, ez = g[1] / math.hypot(g[1], g[2]), g[2] / math.hypot(g[1], g[2])
        us.append((N / 2 + 0.5) - r * ey / float(np.float32(PX)))
        vs.append((N / 2 + 0.5) - r * ez / float(np.float32(PX)))
        sel.append(True)
    return np.array(sel), np.array(us), np.array(vs)


def test_landing_pixel_matches_closed_form(ctx):
    geom, B, hkl, (S9, B9, hk) = _setup()
    p = geom.param20(1)
    p[16] = 80.0  # thetamax wide open: the detector frame is the only spatial limit
    # value = 1 + flat index of (dety, detz): map layout detz + (dety-1)*detzsize, 1-based
    dmap = (1.0 + np.arange(N * N, dtype=np.float32)).reshape(1, N, N)
    q = _random_quats(4096, 11)
    out = ctx.forward_comp(np.zeros(3, np.float32), q, S9, B9, hk, dmap.reshape(-1), np.zeros(1, np.float32),
                           G.flat_rowmajor(np.eye(3)), p).reshape(-1, 4)
    ref, _, edges = O.orientation_scan(np.zeros(3, np.float32), q, S9, B9, hk, dmap, np.zeros(1, np.float32),
                                       G.flat_rowmajor(np.eye(3)), p, tight=True)
    ref = ref.reshape(-1, 4)
    sel, u, v = _closed_form(q, B9, hkl[0])
    on = sel & (np.round(u) >= 1) & (np.round(u) <= N) & (np.round(v) >= 1) & (np.round(v) <= N)
    safe = on & (np.abs(u - np.floor(u) - 0.5) > 1e-3) & (np.abs(v - np.floor(v) - 0.5) > 1e-3)
    assert safe.sum() > 500 and (~on).sum() > 500  # both kinds of trial are well represented
    np.testing.assert_array_equal(out[safe, 0], 1)
    flat = (np.round(u[safe]) - 1) * N + (np.round(v[safe]) - 1)
    np.testing.assert_array_equal(out[safe, 3].astype(np.float64), 1 + flat)
    # off the frame or outside the window: nothing simulated, median 2000, completeness NaN
    np.testing.assert_array_equal(out[~on & (edges == 0), 0], 0)
    assert np.all(out[~on & (edges == 0), 3] == 2000) and np.all(np.isnan(out[~on & (edges == 0), 2]))
    clean = edges == 0
    np.testing.assert_array_equal(out[clean, :2], ref[clean, :2])
    np.testing.assert_array_equal(out[clean, 3], ref[clean, 3])


def _one(ctx, q, S9, B9, hk, dmap, p):
    return ctx.forward_comp(np.zeros(3, np.float32), q, S9, B9, hk, dmap.reshape(-1), np.zeros(1, np.float32),
                            G.flat_rowmajor(np.eye(3)), p)


def test_filters_and_hit(ctx):
    geom, B, hkl, (S9, B9, hk) = _setup()
    a = 0.1  # a small rotation; U = I would land within 1e-5 px of a half-pixel tie
    q = np.array([math.cos(a), 0.3 * math.sin(a), 0.5 * math.sin(a), math.sqrt(1 - 0.34) * math.sin(a)], np.float32)
    U = G.quat_to_u(q.astype(np.float64))
    base = geom.param20(1)
    sel, u, v = _closed_form(q[None], B9, hkl[0])
    assert sel[0]
    iu, iv = int(np.round(u[0])), int(np.round(v[0]))
    assert abs(u[0] - np.floor(u[0]) - 0.5) > 1e-3 and abs(v[0] - np.floor(v[0]) - 0.5) > 1e-3
    miss = np.full((1, N, N), 9.0, np.float32)
    hit = miss.copy()
    hit[0, iu - 1, iv - 1] = 0.0  # spot pixel at the landing point
    near = miss.copy()
    near[0, iu - 1, iv] = 0.0  # spot pixel next to it
    cases = {"miss": (miss, base, (1, 0, 0, 9)), "hit": (hit, base, (1, 1, 1, 0)), "near": (near, base, (1, 0, 0, 9))}
    rec, _ = O.landings(U, np.zeros(3), S9, B9, hk, miss, np.zeros(1, np.float32), G.flat_rowmajor(np.eye(3)),
                        base)
    lam = float(rec["lam"][0])
    p = base.copy()
    p[17], p[18] = lam * 1.01, lam * 2  # wavelength window excludes it
    cases["window"] = (hit, p, (0, 0, None, 2000))
    p = base.copy()
    p[12:16] = [iu - 1, iu + 1, iv - 1, iv + 1]  # beam stop over the landing pixel
    cases["beamstop"] = (hit, p, (0, 0, None, 2000))
    p = p.copy()
    p[12:16] = [iu + 1, iu + 3, iv - 1, iv + 1]  # beam stop that misses by one pixel
    cases["beamstop_miss"] = (hit, p, (1, 1, 1, 0))
    p = base.copy()
    p[10] = iu - 1  # detector too narrow: the pixel falls off the frame
    cases["frame"] = (np.zeros((1, iu - 1, N), np.float32), p, (0, 0, None, 2000))
    for name, (dmap, pp, want) in cases.items():
        got = _one(ctx, q, S9, B9, hk, dmap, pp)
        ref = O.forward_comp(U, np.zeros(3), S9, B9, hk, dmap, np.zeros(1, np.float32),
                             G.flat_rowmajor(np.eye(3)), pp)
        assert got[0] == want[0] and got[1] == want[1] and got[3] == want[3], (name, got)
        assert (np.isnan(got[2]) if want[2] is None else got[2] == want[2]), (name, got)
        assert got[0] == ref[0] and got[1] == ref[1] and got[3] == ref[2], (name, got, ref)
