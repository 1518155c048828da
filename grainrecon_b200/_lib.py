"""ctypes binding of libgrainrecon_b200.so (the C ABI of include/grainrecon_b200.h).

There is no fallback: if the shared library is missing or no sm_100 device is
present, every call raises.  Arrays are passed as plain pointers; numpy arrays
are host buffers, objects exposing ``data_ptr()`` (torch CUDA tensors) or
``__cuda_array_interface__`` are device buffers.
"""
from __future__ import annotations

import ctypes as C
import os
import sys

import numpy as np

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "libgrainrecon_b200.so")

GRC_OK, GRC_EINVAL, GRC_ECAPACITY, GRC_ECUDA, GRC_ETIMEOUT, GRC_ENOMASK = 0, 1, 2, 3, 4, 5
STATUS_NAMES = {0: "GRC_OK", 1: "GRC_EINVAL", 2: "GRC_ECAPACITY", 3: "GRC_ECUDA", 4: "GRC_ETIMEOUT",
                5: "GRC_ENOMASK"}

# Every symbol include/grainrecon_b200.h declares.
EXPORTS = [
    "grc_ctx_create", "grc_ctx_destroy", "grc_last_error", "grc_ctx_stream", "grc_sync", "grc_set_options",
    "grc_upload_masks", "grc_upload_masks_device", "grc_set_geometry", "grc_forward_comp",
    "grc_grow_indexed_region", "grc_forward_comp_compete", "grc_forward_comp_device", "grc_grow_device",
    "grc_compete_device", "grc_last_stats", "grc_set_timing", "grc_set_path", "grc_mask_info", "grc_simulate_spots",
    "grc_edt", "grc_forward_comp_noalloc", "grc_batch_create", "grc_batch_set_maps", "grc_batch_run",
    "grc_batch_capture", "grc_batch_replay", "grc_batch_autotune", "grc_batch_info", "grc_batch_destroy",
    "grc_fit_spot_count", "grc_fit_spot_fill", "grc_centroid_residual_adjoint", "grc_fit_grains_lm",
    "grc_fit_grains_nm", "grc_fit_grains_rms", "grc_fit_geometry_lm", "grc_fit_geometry_cost",
    "grc_fit_geometry_rms", "grc_score_trials_device", "grc_fit_orientation_nm", "grc_pair_spots",
    "grc_walk_best_first", "grc_grow_best_first", "grc_score_trials_argmax_device", "grc_forward_comp_argmax_device",
    "grc_set_median", "grc_seed_candidates_device", "grc_seed_refine_device", "grc_local_grid_device",
    "grc_map_key", "grc_upload_masks_if_changed", "grc_upload_spot_masks", "grc_save_packed_masks",
    "grc_load_packed_masks",
]

# grc_walk_score_fn of the C header
WALK_SCORE_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.POINTER(C.c_int32), C.c_int64, C.POINTER(C.c_double))

# grc_spot_pair of the C header
PAIR_DTYPE = np.dtype([("trial", "<i4"), ("iw", "<i4"), ("ih", "<i4"), ("spot", "<i4"), ("dety", "<f8"),
                       ("detz", "<f8"), ("exp_y", "<f8"), ("exp_z", "<f8"), ("area", "<f8"), ("energy_kev", "<f8"),
                       ("dis", "<f8")])
NOALLOC_MAX_ORIENTATIONS = 65536


class GrcError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(code, code)}: {msg}")
        self.code = code


class Stats(C.Structure):
    _fields_ = [("trials", C.c_int64), ("refined", C.c_int64), ("kernel_launches", C.c_int64),
                ("score_ms", C.c_double), ("path", C.c_int64), ("audit_checked", C.c_int64),
                ("audit_mismatch", C.c_int64), ("device_loop", C.c_int64)]


_lib = None


def load(path: str | None = None):
    """Load the library (building it first when sources are newer and nvcc exists)."""
    global _lib
    if _lib is not None:
        return _lib
    p = path or LIB_PATH
    try:
        from . import build as _b
        if _b.needs_build():
            _b.build()
    except RuntimeError:
        if not os.path.exists(p):
            raise
    if not os.path.exists(p):
        raise OSError(f"{p} is missing: build it with `python -m grainrecon_b200.build`")
    L = C.CDLL(p)
    vp, i64, i, d, f = C.c_void_p, C.c_int64, C.c_int, C.c_double, C.c_void_p
    sig = {
        "grc_ctx_create": [C.POINTER(vp), i],
        "grc_ctx_destroy": [vp],
        "grc_last_error": [vp],
        "grc_ctx_stream": [vp],
        "grc_sync": [vp],
        "grc_set_options": [vp, d, d, d],
        "grc_upload_masks": [vp, f, i64, i64, i64],
        "grc_upload_masks_device": [vp, f, i64, i64, i64],
        "grc_set_geometry": [vp, f, f, f, f, f, f],
        "grc_forward_comp": [vp, f, f, i64, f, f, f, f, f, f, f, f],
        "grc_grow_indexed_region": [vp, f, i64, f, f, f, f, f, f, f, f, f, f],
        "grc_forward_comp_compete": [vp, f, i64, f, i64, f, i64, f, f, f, f, f, f, f, f, f],
        "grc_forward_comp_device": [vp, f, i64, f, i64, f],
        "grc_grow_device": [vp, f, i64, f, f, f],
        "grc_compete_device": [vp, f, i64, f, i64, f, i64, f, f, f],
        "grc_last_stats": [vp, C.POINTER(Stats)],
        "grc_set_timing": [vp, i],
        "grc_set_path": [vp, i],
        "grc_mask_info": [vp, C.POINTER(i64), C.POINTER(i), C.POINTER(i64), C.POINTER(i64), C.POINTER(i64)],
        "grc_simulate_spots": [vp, f, f, i64, f],
        "grc_edt": [vp, f, i64, i64, i64, f],
        "grc_forward_comp_noalloc": [vp, f, f, i64, f],
        "grc_batch_create": [vp, f, i64, f, i64, f, i64, f, C.POINTER(vp)],
        "grc_batch_set_maps": [vp, C.POINTER(i64), f, f, f, f, f],
        "grc_batch_run": [vp, f, f],
        "grc_batch_capture": [vp, f],
        "grc_batch_replay": [vp],
        "grc_batch_autotune": [vp, f, i64, C.POINTER(i), C.POINTER(i), C.POINTER(d)],
        "grc_batch_info": [vp, C.POINTER(i64), C.POINTER(i64), C.POINTER(i), C.POINTER(i)],
        "grc_batch_destroy": [vp],
        "grc_fit_spot_count": [vp, f, f, i64, f],
        "grc_fit_spot_fill": [vp, f, f, i64, f, f, f, f, f],
        "grc_centroid_residual_adjoint": [vp, i, f, f, f, f, f, f, i64, f, f],
        "grc_fit_grains_lm": [vp, f, f, i64, f, f, f, f, i64, f, f, i, C.POINTER(i)],
        "grc_fit_grains_nm": [vp, f, f, i64, f, f, f, f, i64, f, f, i, i, f, i],
        "grc_fit_grains_rms": [vp, f, f, f, i64, f, f, f, f, i64, f, f],
        "grc_fit_geometry_lm": [vp, f, i, f, f, f, f, f, i64, f, i, C.POINTER(i)],
        "grc_fit_geometry_cost": [vp, f, i, f, f, f, f, f, i64, f],
        "grc_fit_geometry_rms": [vp, f, i, f, f, f, f, f, f, i64, f],
        "grc_score_trials_device": [vp, f, i64, f, i64, f, f, i64, f],
        "grc_score_trials_argmax_device": [vp, f, i64, f, i64, f, f, i64, i64, f, f, f],
        "grc_forward_comp_argmax_device": [vp, f, i64, f, i64, f, f, f],
        "grc_set_median": [vp, i],
        "grc_seed_candidates_device": [vp, f, i64, f, f, i64, i, f, f, f],
        "grc_seed_refine_device": [vp, f, i64, f, i, i, d, i, f, f, f, f],
        "grc_local_grid_device": [vp, f, i64, i, d, f, f],
        "grc_map_key": [f, i64, i64],
        "grc_upload_spot_masks": [vp, f, i64, i64, i64],
        "grc_save_packed_masks": [vp, C.c_char_p],
        "grc_load_packed_masks": [vp, C.c_char_p],
        "grc_upload_masks_if_changed": [vp, f, i64, i64, i64, i64, C.POINTER(i)],
        "grc_fit_orientation_nm": [vp, f, f, i64, d, i, i, d, d, f, f, f, f, f],
        "grc_pair_spots": [vp, f, f, i64, f, i64, f, f, i64, C.POINTER(i64)],
        "grc_walk_best_first": [WALK_SCORE_FN, vp, i64, i64, i64, f, f, f, f, f, d, d, d, d, f, f, f, f, f, i64,
                                C.POINTER(i64), f, C.POINTER(i)],
        "grc_grow_best_first": [vp, i64, i64, i64, f, f, f, f, f, d, d, d, d, f, f, f, f, f, f, f, f, f, f, f, f,
                                f, f, i64, C.POINTER(i64), f, C.POINTER(i)],
    }
    for name, args in sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = i
    L.grc_last_error.restype = C.c_char_p
    L.grc_map_key.restype = C.c_uint64
    L.grc_ctx_stream.restype = vp
    _lib = L
    return L


def map_key(proj_bin_bw, samples: int = 1 << 20) -> int:
    """grc_map_key of a host float32 map (no GPU needed)."""
    a = f32(proj_bin_bw)
    return int(load().grc_map_key(_ptr(a), a.size, samples))


def _ptr(a):
    """Raw address of a host numpy array, a torch tensor or a CUDA-array-interface object."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        if not a.flags["C_CONTIGUOUS"]:
            raise ValueError("array must be C-contiguous")
        return a.ctypes.data
    if hasattr(a, "data_ptr"):
        if hasattr(a, "is_contiguous") and not a.is_contiguous():
            raise ValueError("tensor must be contiguous")
        return a.data_ptr()
    if hasattr(a, "__cuda_array_interface__"):
        return a.__cuda_array_interface__["data"][0]
    if isinstance(a, int):
        return a
    raise TypeError(f"cannot take the address of {type(a)}")


def _walk_arrays(I, Imask, DisMedian, Ninter):
    """X x Y x Z maps (numpy index order) as MATLAB-order doubles, plus output buffers."""
    I = np.asarray(I, np.float64)
    X, Y, Z = I.shape
    col = lambda a: np.ascontiguousarray(np.asarray(a, np.float64).reshape(X, Y, Z).transpose(2, 1, 0))
    ins = [col(I), col(Imask), col(DisMedian), col(Ninter)]
    outs = [np.empty((Z, Y, X)) for _ in range(3)] + [np.empty((Z, Y, X), np.uint8)]
    cap = int((ins[1] > 0).sum()) + 1
    return (X, Y, Z), ins, outs, np.empty(cap, np.int64), cap


def _walk_result(dims, outs, idx, n, center, rc):
    """(J, Completeness_out, DisMedian_out, Ninter_out, center, replace_center, indexed_indices)."""
    X, Y, Z = dims
    C_out, D_out, N_out, J = (a.transpose(2, 1, 0) for a in outs)
    k = idx[:n] - 1
    ind = np.stack([k % X + 1, (k // X) % Y + 1, k // (X * Y) + 1], 1)
    return J.astype(bool), C_out, D_out, N_out, center, int(rc.value), ind


def walk_best_first(score, I, Imask, DisMedian, Ninter, seed, drop_off, maxD, indexed_comp, maxDmedian):
    """grow_indexed_region.m's region walk in the library with a Python scorer: ``score(vox)``
    maps (k x 3) 1-based voxel indices to (k x 3) [Nr_simu, Nr_intersect, dis_median].  Maps are
    X x Y x Z arrays in numpy index order.  Returns (J, Completeness_out, DisMedian_out,
    Ninter_out, center, replace_center, indexed_indices) as grow_indexed_region.m does."""
    L = load()
    dims, ins, outs, idx, cap = _walk_arrays(I, Imask, DisMedian, Ninter)
    err = []

    def cb(user, vox, n, out):
        try:
            v = np.ctypeslib.as_array(vox, shape=(n * 3,)).reshape(n, 3).astype(np.int64)
            r = np.asarray(score(v), np.float64).reshape(n, 3)
            np.ctypeslib.as_array(out, shape=(n * 3,))[:] = r.reshape(-1)
            return GRC_OK
        except Exception as e:  # noqa: BLE001 -- re-raised after the walk returns
            err.append(e)
            return GRC_EINVAL

    fn = WALK_SCORE_FN(cb)
    sd = np.asarray(seed, np.int32).reshape(3)
    n, center, rc = C.c_int64(), np.zeros(3), C.c_int()
    code = L.grc_walk_best_first(fn, None, *dims, *[_ptr(a) for a in ins], _ptr(sd), float(drop_off), float(maxD),
                                 float(indexed_comp), float(maxDmedian), *[_ptr(a) for a in outs], _ptr(idx), cap,
                                 C.byref(n), _ptr(center), C.byref(rc))
    if err:
        raise err[0]
    if code != GRC_OK:
        raise GrcError(code, "walk_best_first")
    return _walk_result(dims, outs, idx, n.value, center, rc)


def f32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float32).reshape(-1)


class Context:
    """One device context of the scorer (owns the resident distance map and a stream)."""

    def __init__(self, device: int = 0):
        self.L = load()
        self.device = device
        self._ext = None
        h = C.c_void_p()
        rc = self.L.grc_ctx_create(C.byref(h), device)
        if rc != GRC_OK:
            raise GrcError(rc, f"grc_ctx_create(device={device}) failed (no sm_100 GPU visible?)")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.L.grc_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, rc: int):
        if rc != GRC_OK:
            raise GrcError(rc, self.L.grc_last_error(self.h).decode())

    @property
    def stream(self) -> int:
        return int(self.L.grc_ctx_stream(self.h) or 0)

    def _dev(self, fn, *args):
        """Call a C entry that reads or writes device buffers, ordered with torch's current stream.

        The library works on its own non-blocking stream; when torch is in use, that stream first
        waits for the work already queued on torch's current stream (which produced the inputs),
        and torch's stream then waits for the library's work (which produces the outputs).  No host
        synchronisation is added."""
        torch = sys.modules.get("torch")
        cur = ext = None
        if torch is not None and torch.cuda.is_initialized():
            if self._ext is None:
                self._ext = torch.cuda.ExternalStream(self.stream, device=torch.device("cuda", self.device))
            ext = self._ext
            cur = torch.cuda.current_stream(self.device)
            ext.wait_stream(cur)
        self._check(fn(self.h, *args))
        if ext is not None:
            cur.wait_stream(ext)

    def sync(self):
        self._check(self.L.grc_sync(self.h))

    def set_options(self, dety0=float("nan"), detz0=float("nan"), hit_threshold=float("nan")):
        self._check(self.L.grc_set_options(self.h, dety0, detz0, hit_threshold))

    def upload_masks(self, proj_bin_bw, detzsize: int, detysize: int, nrot: int):
        if isinstance(proj_bin_bw, np.ndarray):
            proj_bin_bw = np.ascontiguousarray(proj_bin_bw, dtype=np.float32)
            self._check(self.L.grc_upload_masks(self.h, _ptr(proj_bin_bw), detzsize, detysize, nrot))
        else:  # a device array (torch tensor): ordered with the stream that produced it
            self._dev(self.L.grc_upload_masks, _ptr(proj_bin_bw), detzsize, detysize, nrot)

    def upload_masks_if_changed(self, proj_bin_bw, detzsize: int, detysize: int, nrot: int,
                                samples: int = 1 << 20) -> bool:
        """Upload the map unless its content key and size equal the last keyed upload's."""
        a = f32(proj_bin_bw)
        up = C.c_int(0)
        self._check(self.L.grc_upload_masks_if_changed(self.h, _ptr(a), detzsize, detysize, nrot, samples,
                                                       C.byref(up)))
        return bool(up.value)

    def upload_spot_masks(self, proj_bin, detzsize: int, detysize: int, nrot: int):
        """Binary spot images (nonzero = spot; host array or device tensor) -> device bwdist map."""
        a = proj_bin if hasattr(proj_bin, "data_ptr") else np.ascontiguousarray(proj_bin, dtype=np.uint8).reshape(-1)
        self._dev(self.L.grc_upload_spot_masks, _ptr(a), detzsize, detysize, nrot)

    def save_packed_masks(self, path: str):
        self._check(self.L.grc_save_packed_masks(self.h, os.fsencode(path)))

    def load_packed_masks(self, path: str):
        self._check(self.L.grc_load_packed_masks(self.h, os.fsencode(path)))

    def set_geometry(self, S, B, hkl, rot_angles, RotDet, param):
        keep = [f32(x) for x in (S, B, hkl, rot_angles, RotDet, param)]
        self._check(self.L.grc_set_geometry(self.h, *[_ptr(a) for a in keep]))

    def forward_comp(self, pos, q, S, B, hkl, proj_bin_bw, rot_angles, RotDet, param, out=None):
        """cuda_forward_comp: returns 4*n_q floats [Nr_simu Nr_intersect C dis_median]."""
        q = f32(q)
        n = q.size // 4
        if out is None:
            out = np.empty(4 * n, np.float32)
        pb = None if proj_bin_bw is None else f32(proj_bin_bw)
        keep = [f32(pos), q, f32(S), f32(B), f32(hkl), pb, f32(rot_angles), f32(RotDet), f32(param)]
        p = [_ptr(a) for a in keep]
        self._check(self.L.grc_forward_comp(self.h, p[0], p[1], n, p[2], p[3], p[4], p[5], p[6], p[7], p[8],
                                            _ptr(out)))
        return out

    def grow_best_first(self, I, Imask, DisMedian, Ninter, seed, drop_off, maxD, indexed_comp, maxDmedian, U, S,
                        B, hkl, proj_bin_bw, rot_angles, RotDet, param, param1):
        """grow_indexed_region.m's region walk on the GPU scorer (grc_grow_best_first); returns
        (J, Completeness_out, DisMedian_out, Ninter_out, center, replace_center, indexed_indices)."""
        dims, ins, outs, idx, cap = _walk_arrays(I, Imask, DisMedian, Ninter)
        sd = np.asarray(seed, np.int32).reshape(3)
        pb = None if proj_bin_bw is None else f32(proj_bin_bw)
        keep = [f32(U), f32(S), f32(B), f32(hkl), pb, f32(rot_angles), f32(RotDet), f32(param), f32(param1)]
        n, center, rc = C.c_int64(), np.zeros(3), C.c_int()
        self._check(self.L.grc_grow_best_first(self.h, *dims, *[_ptr(a) for a in ins], _ptr(sd), float(drop_off),
                                               float(maxD), float(indexed_comp), float(maxDmedian),
                                               *[_ptr(a) for a in keep], *[_ptr(a) for a in outs], _ptr(idx), cap,
                                               C.byref(n), _ptr(center), C.byref(rc)))
        return _walk_result(dims, outs, idx, n.value, center, rc)

    def grow_indexed_region(self, rows6, U, S, B, hkl, proj_bin_bw, rot_angles, RotDet, param, param1, out=None):
        """cuda_grow_indexed_region: returns 7*m floats [x y z Nr_simu Nr_intersect dis_median flag]."""
        rows6 = f32(rows6)
        m = rows6.size // 6
        if out is None:
            out = np.empty(7 * m, np.float32)
        pb = None if proj_bin_bw is None else f32(proj_bin_bw)
        keep = [rows6, f32(U), f32(S), f32(B), f32(hkl), pb, f32(rot_angles), f32(RotDet), f32(param), f32(param1)]
        p = [_ptr(a) for a in keep]
        self._check(self.L.grc_grow_indexed_region(self.h, p[0], m, p[1], p[2], p[3], p[4], p[5], p[6], p[7], p[8],
                                                   p[9], _ptr(out)))
        return out

    def forward_comp_compete(self, rows5, id_neigb, euler, S, B, hkl, proj_bin_bw, rot_angles, RotDet, param,
                             param1, out=None):
        """cuda_forward_comp_compete: returns 8*m floats [row phi1 PHI phi2 GrainId C Nr_intersect dis_median]."""
        rows5, idn, eu = f32(rows5), f32(id_neigb), f32(euler)
        m = rows5.size // 5
        if out is None:
            out = np.empty(8 * m, np.float32)
        pb = None if proj_bin_bw is None else f32(proj_bin_bw)
        keep = [rows5, idn, eu, f32(S), f32(B), f32(hkl), pb, f32(rot_angles), f32(RotDet), f32(param), f32(param1)]
        p = [_ptr(a) for a in keep]
        self._check(self.L.grc_forward_comp_compete(self.h, p[0], m, p[1], idn.size, p[2], eu.size // 3, p[3], p[4],
                                                    p[5], p[6], p[7], p[8], p[9], p[10], _ptr(out)))
        return out

    # device-resident entries (torch CUDA tensors / device pointers)
    def forward_comp_device(self, d_pos, n_vox: int, d_q, n_q: int, d_out):
        self._dev(self.L.grc_forward_comp_device, _ptr(d_pos), n_vox, _ptr(d_q), n_q, _ptr(d_out))

    def grow_device(self, d_rows6, m: int, U, param1, d_out):
        u, p1 = f32(U), f32(param1)
        self._dev(self.L.grc_grow_device, _ptr(d_rows6), m, _ptr(u), _ptr(p1), _ptr(d_out))

    def compete_device(self, d_rows5, m: int, d_id, n_neigb: int, d_euler, n_grain: int, param1, d_out,
                       d_trial_out=None):
        p1 = f32(param1)
        self._dev(self.L.grc_compete_device, _ptr(d_rows5), m, _ptr(d_id), n_neigb, _ptr(d_euler),
                                              n_grain, _ptr(p1), _ptr(d_out), _ptr(d_trial_out))

    def score_trials_device(self, d_pos, n_vox: int, d_q, n_q: int, d_trial_voxel, d_trial_orient, n_trials: int,
                            d_out):
        """FP64 trial list: trial t = (voxel d_trial_voxel[t], orientation d_trial_orient[t]); both None
        means trial t = (voxel t, orientation t).  d_pos: 3 doubles per voxel, d_q: 4 doubles per
        orientation, d_out: 4 floats per trial (device buffers)."""
        self._dev(self.L.grc_score_trials_device, _ptr(d_pos), n_vox, _ptr(d_q), n_q, _ptr(d_trial_voxel),
                                                   _ptr(d_trial_orient), n_trials, _ptr(d_out))

    def fit_orientation_nm(self, d_pos, d_x0, n: int, d_x, d_fval, d_evals=None, d_iters=None, d_flag=None,
                           half_width: float = 0.02, max_evals: int = 2000, max_iter: int = 2000,
                           tol_f: float = 1e-10, tol_x: float = 1e-4):
        """Batched fminsearchbnd on 1 - completeness over (q1, q2, q3), one simplex per seed."""
        self._dev(self.L.grc_fit_orientation_nm, _ptr(d_pos), _ptr(d_x0), n, half_width, max_evals, max_iter,
                                                  tol_f, tol_x, _ptr(d_x), _ptr(d_fval), _ptr(d_evals), _ptr(d_iters),
                                                  _ptr(d_flag))

    def pair_spots(self, d_pos, d_q, n: int, d_spots, n_spots: int, d_proj_offsets, max_pairs: int = 0):
        """Spot pairing (see the C header): returns a host structured array of PAIR_DTYPE, in
        (trial, projection, reflection) order.  The device buffer grows when max_pairs is short."""
        import torch
        cap = max(int(max_pairs), 1024)
        while True:
            buf = torch.empty(cap * PAIR_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
            npairs = C.c_int64()
            torch.cuda.current_stream().synchronize()
            rc = self.L.grc_pair_spots(self.h, _ptr(d_pos), _ptr(d_q), n, _ptr(d_spots), n_spots,
                                       _ptr(d_proj_offsets), _ptr(buf), cap, C.byref(npairs))
            if rc == GRC_ECAPACITY and npairs.value > cap:
                cap = int(npairs.value)
                continue
            self._check(rc)
            m = int(npairs.value)
            return buf[: m * PAIR_DTYPE.itemsize].cpu().numpy().view(PAIR_DTYPE).copy()

    def forward_comp_noalloc(self, pos, d_q, n_q: int, d_out):
        """Allocation-free seeding scan: host pos (3 floats), device d_q / d_out; see the C header."""
        p = f32(pos)
        self._dev(self.L.grc_forward_comp_noalloc, _ptr(p), _ptr(d_q), n_q, _ptr(d_out))

    def batch(self, d_rows5, m: int, d_id, n_neigb: int, d_euler, n_grain: int, param1):
        """Plan a batched-grow work list on device buffers (see Batch)."""
        return Batch(self, d_rows5, m, d_id, n_neigb, d_euler, n_grain, param1)

    def simulate_spots(self, d_pos, d_U, n: int, d_mask):
        self._dev(self.L.grc_simulate_spots, _ptr(d_pos), _ptr(d_U), n, _ptr(d_mask))

    def edt(self, d_mask, detzsize: int, detysize: int, nrot: int, d_map):
        self._dev(self.L.grc_edt, _ptr(d_mask), detzsize, detysize, nrot, _ptr(d_map))

    def set_median(self, enable: bool):
        """False: seeding scans count from the bit-packed hit mask and leave column 4 NaN."""
        self._check(self.L.grc_set_median(self.h, 1 if enable else 0))

    def forward_comp_argmax_device(self, d_pos, n_vox: int, d_q, n_q: int, d_out, d_best, d_best_c):
        """Seeding scan plus the first maximum of completeness per voxel (d_out may be None)."""
        self._dev(self.L.grc_forward_comp_argmax_device, _ptr(d_pos), n_vox, _ptr(d_q), n_q, _ptr(d_out),
                  _ptr(d_best), _ptr(d_best_c))

    def score_trials_argmax_device(self, d_pos, n_vox: int, d_q, n_q: int, d_trial_voxel, d_trial_orient,
                                   n_trials: int, group_size: int, d_out, d_best, d_best_c):
        """FP64 trial list plus the first maximum per group of ``group_size`` trials."""
        self._dev(self.L.grc_score_trials_argmax_device, _ptr(d_pos), n_vox, _ptr(d_q), n_q, _ptr(d_trial_voxel),
                  _ptr(d_trial_orient), n_trials, group_size, _ptr(d_out), _ptr(d_best), _ptr(d_best_c))

    def seed_candidates_device(self, d_pos, n: int, d_q, n_q: int, n_top: int, d_idx, d_cand=None, d_out=None,
                               d_q64=None):
        """Seeding scan (completeness only) and the top ``n_top`` rows per seed."""
        self._dev(self.L.grc_seed_candidates_device, _ptr(d_pos), n, _ptr(d_q), _ptr(d_q64), n_q, n_top, _ptr(d_idx),
                  _ptr(d_cand), _ptr(d_out))

    def seed_refine_device(self, d_pos, n: int, d_cand, k: int, nr: int, gridsize: float, d_best_q, d_best_c,
                           d_order, n_x0: int = 0, d_x0=None):
        """Local refine of every candidate: grid maxima in per-seed sortrows order (+ fit start points)."""
        self._dev(self.L.grc_seed_refine_device, _ptr(d_pos), n, _ptr(d_cand), k, nr, gridsize, n_x0, _ptr(d_best_q),
                  _ptr(d_best_c), _ptr(d_order), _ptr(d_x0))

    def local_grid_device(self, d_cand, n_cand: int, nr: int, gridsize: float, d_rows, d_rows_f32=None):
        """ori_local_sampling grids of n_cand quaternions in unique(q,'rows') order."""
        self._dev(self.L.grc_local_grid_device, _ptr(d_cand), n_cand, nr, gridsize, _ptr(d_rows), _ptr(d_rows_f32))

    def set_timing(self, enable: bool):
        self._check(self.L.grc_set_timing(self.h, int(bool(enable))))

    def set_path(self, path: int):
        """0 = by size, 1 = per-trial kernel, 2 = CTA sweep, 3 = warp scan."""
        self._check(self.L.grc_set_path(self.h, int(path)))

    def last_stats(self) -> dict:
        s = Stats()
        self._check(self.L.grc_last_stats(self.h, C.byref(s)))
        return {"trials": s.trials, "refined": s.refined, "kernel_launches": s.kernel_launches,
                "score_ms": s.score_ms, "path": s.path, "audit_checked": s.audit_checked,
                "audit_mismatch": s.audit_mismatch, "device_loop": s.device_loop}

    def mask_info(self) -> dict:
        nd, nz, ny, nr = C.c_int64(), C.c_int64(), C.c_int64(), C.c_int64()
        bits = C.c_int()
        self._check(self.L.grc_mask_info(self.h, C.byref(nd), C.byref(bits), C.byref(nz), C.byref(ny), C.byref(nr)))
        return {"n_distinct": nd.value, "code_bits": bits.value, "detzsize": nz.value, "detysize": ny.value,
                "nrot": nr.value}


class Batch:
    """A planned batched-grow iteration (grc_batch_*): run, capture into a CUDA graph, replay, autotune."""

    def __init__(self, ctx: Context, d_rows5, m, d_id, n_neigb, d_euler, n_grain, param1):
        self.ctx, self.L = ctx, ctx.L
        self._keep = (d_rows5, d_id, d_euler)  # borrowed device arrays must outlive the batch
        p1 = f32(param1)
        h = C.c_void_p()
        ctx._dev(lambda _h, *a: self.L.grc_batch_create(ctx.h, *a), _ptr(d_rows5), m, _ptr(d_id), n_neigb,
                 _ptr(d_euler), n_grain, _ptr(p1), C.byref(h))
        self.h = h

    def info(self) -> dict:
        m, T = C.c_int64(), C.c_int64()
        p, s = C.c_int(), C.c_int()
        self.ctx._check(self.L.grc_batch_info(self.h, C.byref(m), C.byref(T), C.byref(p), C.byref(s)))
        return {"voxels": m.value, "trials": T.value, "path": p.value, "slots": s.value}

    def set_maps(self, dims, completeness=None, grain_id=None, dismedian=None, ninter=None, visitflag=None):
        d = (C.c_int64 * 3)(*[int(x) for x in dims])
        self._maps = (completeness, grain_id, dismedian, ninter, visitflag)
        self.ctx._dev(lambda _h, *a: self.L.grc_batch_set_maps(self.h, *a), d, *[_ptr(x) for x in self._maps])

    def run(self, d_out8, d_trial_out=None):
        self.ctx._dev(lambda _h, *a: self.L.grc_batch_run(self.h, *a), _ptr(d_out8), _ptr(d_trial_out))

    def capture(self, d_out8):
        self._graph_out = d_out8
        self.ctx._dev(lambda _h, *a: self.L.grc_batch_capture(self.h, *a), _ptr(d_out8))

    def replay(self):
        self.ctx._dev(lambda _h: self.L.grc_batch_replay(self.h))

    def autotune(self, d_out8, max_voxels: int = 0) -> dict:
        p, s, ms = C.c_int(), C.c_int(), C.c_double()
        self.ctx._dev(lambda _h, *a: self.L.grc_batch_autotune(self.h, *a), _ptr(d_out8), max_voxels, C.byref(p), C.byref(s),
                                                  C.byref(ms))
        return {"path": p.value, "slots": s.value, "ms": ms.value}

    def close(self):
        if getattr(self, "h", None):
            self.L.grc_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
