"""ctypes front-end of the FP64 CPU oracle -- TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg import
this module; the product package never does.  Parity status: unpinned (the MATLAB
reference cannot run here and ships no golden vectors); ``grc_oracle.c`` restates
forward_comp.m line by line.

Every entry takes the MEX argument layouts (float32 arrays) and returns numpy
arrays plus the per-trial edge-reflection counts.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libgrc_oracle.so")
_lib = None

_f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")


class Landing(C.Structure):
    _fields_ = [("iw", C.c_int32), ("ih", C.c_int32), ("sel", C.c_int32), ("edge", C.c_int32),
                ("u", C.c_double), ("v", C.c_double), ("lam", C.c_double), ("dis", C.c_double)]


def build() -> str:
    """Compile the oracle with its Makefile (gcc, OpenMP)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        srcs = [os.path.join(_HERE, f) for f in ("grc_oracle.c", "grc_fit_oracle.c")]
        if not os.path.exists(_LIB_PATH) or any(os.path.getmtime(_LIB_PATH) < os.path.getmtime(f) for f in srcs):
            build()
        L = C.CDLL(_LIB_PATH)
        d, i64, i = C.c_double, C.c_int64, C.c_int
        L.oracle_forward_comp.argtypes = [_f64p, _f64p, _f32p, _f32p, _f32p, _f32p, _f32p, _f32p, _f32p,
                                          d, d, d, _f64p]
        L.oracle_landings.argtypes = [_f64p, _f64p, _f32p, _f32p, _f32p, _f32p, _f32p, _f32p, _f32p,
                                      d, d, d, C.POINTER(Landing), _f64p]
        L.oracle_orientation_scan.argtypes = [_f32p, _f32p, i64, _f32p, _f32p, _f32p, _f32p, _f32p, _f32p,
                                              _f32p, d, d, d, i, _f32p, _i32p, _i32p]
        L.oracle_grow.argtypes = [_f32p, i64, _f32p, _f32p, _f32p, _f32p, _f32p, _f32p, _f32p, _f32p,
                                  _f32p, d, d, d, i, C.c_void_p, i, _f32p, _i32p, _i32p]
        L.oracle_compete.argtypes = [_f32p, i64, _f32p, _f32p, _f32p, _f32p, _f32p, _f32p, _f32p, _f32p,
                                     _f32p, _f32p, d, d, d, i, _f32p, _i32p, _i32p]
        L.oracle_max_threads.restype = i
        L.oracle_fit_uv_jac.argtypes = [i, _f64p, _f64p, _f64p, _f64p, _f64p, d, d, d, d, d, _f64p, _f64p, _f64p]
        _lib = L
    return _lib


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32).reshape(-1)


def _defaults(param, dety0, detz0):
    p = _f32(param)
    if dety0 is None:
        dety0 = float(p[10]) / 2 + 0.5
    if detz0 is None:
        detz0 = float(p[11]) / 2 + 0.5
    return p, dety0, detz0


def forward_comp(U, pos, S, B, hkl, proj_bin_bw, rot_angles, RotDet, param, dety0=None, detz0=None, thr=0.5):
    """One trial: (Nr_simu, Nr_intersect, dis_median, n_edge, n_tight_edge) in FP64."""
    p, dety0, detz0 = _defaults(param, dety0, detz0)
    out = np.zeros(5)
    lib().oracle_forward_comp(np.ascontiguousarray(U, np.float64).reshape(9), np.ascontiguousarray(pos, np.float64),
                              _f32(S), _f32(B), _f32(hkl), _f32(proj_bin_bw), _f32(rot_angles), _f32(RotDet), p,
                              dety0, detz0, thr, out)
    return out


def landings(U, pos, S, B, hkl, proj_bin_bw, rot_angles, RotDet, param, dety0=None, detz0=None, thr=0.5):
    """Per-reflection records (omega index, hkl index, selected, edge, u, v, lambda, dis)."""
    p, dety0, detz0 = _defaults(param, dety0, detz0)
    n = int(p[0]) * int(p[1])
    rec = (Landing * n)()
    out = np.zeros(5)
    lib().oracle_landings(np.ascontiguousarray(U, np.float64).reshape(9), np.ascontiguousarray(pos, np.float64),
                          _f32(S), _f32(B), _f32(hkl), _f32(proj_bin_bw), _f32(rot_angles), _f32(RotDet), p,
                          dety0, detz0, thr, rec, out)
    arr = np.ctypeslib.as_array(rec)
    return {k: np.array(arr[k]) for k in ("iw", "ih", "sel", "edge", "u", "v", "lam", "dis")}, out


def orientation_scan(pos, q, S, B, hkl, proj_bin_bw, rot_angles, RotDet, param, dety0=None, detz0=None,
                     thr=0.5, nthreads=0, tight=False):
    """cuda_forward_comp semantics on the CPU: (out[4N] float32, edges[N]), plus the tight-edge
    counts (reflections within 1e-9 px of a rounding boundary or 1e-12 of a window bound) as a
    third value when ``tight``."""
    p, dety0, detz0 = _defaults(param, dety0, detz0)
    q = _f32(q)
    n = q.size // 4
    out = np.zeros(4 * n, np.float32)
    edges = np.zeros(n, np.int32)
    te = np.zeros(n, np.int32)
    rc = lib().oracle_orientation_scan(_f32(pos), q, n, _f32(S), _f32(B), _f32(hkl), _f32(proj_bin_bw),
                                       _f32(rot_angles), _f32(RotDet), p, dety0, detz0, thr, nthreads, out, edges,
                                       te)
    assert rc == 0
    return (out, edges, te) if tight else (out, edges)


def grow(rows6, U, S, B, hkl, proj_bin_bw, rot_angles, RotDet, param, param1, dety0=None, detz0=None,
         thr=0.5, rule=0, ninter=None, nthreads=0, tight=False):
    """cuda_grow_indexed_region semantics on the CPU: (out[7M] float32, edges[M]) (+ tight-edge
    counts when ``tight``)."""
    p, dety0, detz0 = _defaults(param, dety0, detz0)
    rows6 = _f32(rows6)
    m = rows6.size // 6
    out = np.zeros(7 * m, np.float32)
    edges = np.zeros(m, np.int32)
    te = np.zeros(m, np.int32)
    nin = None
    if ninter is not None:
        nin = _f32(ninter)
    rc = lib().oracle_grow(rows6, m, _f32(U), _f32(S), _f32(B), _f32(hkl), _f32(proj_bin_bw), _f32(rot_angles),
                           _f32(RotDet), p, _f32(param1), dety0, detz0, thr, rule,
                           None if nin is None else nin.ctypes.data, nthreads, out, edges, te)
    assert rc == 0
    return (out, edges, te) if tight else (out, edges)


def compete(rows5, id_neigb, euler, S, B, hkl, proj_bin_bw, rot_angles, RotDet, param, param1, dety0=None,
            detz0=None, thr=0.5, nthreads=0, tight=False):
    """cuda_forward_comp_compete semantics on the CPU: (out[8M] float32, edges[M]) (+ tight-edge
    counts when ``tight``)."""
    p, dety0, detz0 = _defaults(param, dety0, detz0)
    rows5 = _f32(rows5)
    m = rows5.size // 5
    out = np.zeros(8 * m, np.float32)
    edges = np.zeros(m, np.int32)
    te = np.zeros(m, np.int32)
    rc = lib().oracle_compete(rows5, m, _f32(id_neigb), _f32(euler), _f32(S), _f32(B), _f32(hkl),
                              _f32(proj_bin_bw), _f32(rot_angles), _f32(RotDet), p, _f32(param1), dety0, detz0,
                              thr, nthreads, out, edges, te)
    assert rc == 0
    return (out, edges, te) if tight else (out, edges)


def max_threads() -> int:
    return int(lib().oracle_max_threads())


def fit_uv_jac(mode, grain6, geo10, S, B, h, omega_deg, pxy, pxz, dety0, detz0):
    """Landing (u, v) and Jacobian rows (ju, jv) of one spot by complex step (FP64).

    mode 0: 6 grain parameters (Rodrigues, centre); mode 1: 10 geometry parameters.
    S, B: 3x3 (row-major), h: (h, k, l)."""
    K = 6 if mode == 0 else 10
    uv, ju, jv = np.zeros(2), np.zeros(K), np.zeros(K)
    f64 = lambda a: np.ascontiguousarray(a, dtype=np.float64).reshape(-1)
    lib().oracle_fit_uv_jac(mode, f64(grain6), f64(geo10), f64(S), f64(B), f64(h), float(omega_deg), float(pxy),
                            float(pxz), float(dety0), float(detz0), uv, ju, jv)
    return uv, ju, jv
