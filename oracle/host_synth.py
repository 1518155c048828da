"""Host-only synthesis of the benchmark inputs -- TEST AND BENCHMARK INFRASTRUCTURE ONLY.

The CPU reference arm of ``bench.py`` must build its sample and distance map without a GPU and
without the product library.  These helpers do that with the C code of ``grc_synth_host.c``
(OpenMP on the host cores):

* ``make_sample_host(kind, seed)``: ``synth.make_sample`` with the grain-id volume computed by
  ``host_power_voronoi`` (the sites and weights of ``synth.voronoi_sites``);
* ``distance_map_host(sample)``: the spot masks of the ground-truth grains
  (``host_simulate_mask``, every voxel with its grain's orientation) and their exact EDT
  (``host_edt``), as float32 (nrot, dety, detz) -- the layout of
  ``reshape(proj_bin_bw,1,[])``.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import oracle as O

_f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")
_bound = False


def _lib():
    global _bound
    L = O.lib()
    if not _bound:
        i, i64, d = C.c_int, C.c_int64, C.c_double
        L.host_power_voronoi.argtypes = [i, _f64p, _f64p, i, i, _i32p]
        L.host_simulate_mask.argtypes = [_f32p, _f32p, _f32p, _f32p, _f32p, _f32p, d, d, _f64p, _i32p, i64, _f64p,
                                         i64, i, _u8p]
        L.host_edt.argtypes = [_u8p, i64, i64, i64, i, _f32p]
        _bound = True
    return L


def power_voronoi(dim: int, n_grains: int, seed: int, sigma: float, nthreads: int = 0) -> np.ndarray:
    """Grain ids (dim^3 int32) of ``synth.voronoi_cylinder`` computed on the host cores in C."""
    from grainrecon_b200 import synth
    sites, w2 = synth.voronoi_sites(dim, n_grains, seed, sigma)
    gid = np.zeros(dim * dim * dim, np.int32)
    rc = _lib().host_power_voronoi(int(dim), np.ascontiguousarray(sites, np.float64),
                                   np.ascontiguousarray(w2, np.float64), int(n_grains), int(nthreads), gid)
    assert rc == 0
    return gid.reshape(dim, dim, dim)


def make_sample_host(kind: str, seed: int = 1, nthreads: int = 0):
    from grainrecon_b200 import synth
    return synth.make_sample(kind, seed=seed, voronoi=lambda d, n, s, g: power_voronoi(d, n, s, g, nthreads))


def spot_mask_host(sample, nthreads: int = 0) -> np.ndarray:
    """Boolean-as-uint8 spot masks (nrot, dety, detz) of every voxel of the sample."""
    from grainrecon_b200 import geometry as G
    g = sample.geom
    S9, B9, hkl, rot, R9, p = sample.mex_arrays()
    idx = sample.voxel_indices()
    gid = np.ascontiguousarray(sample.grain_id[idx[:, 0] - 1, idx[:, 1] - 1, idx[:, 2] - 1], np.int32)
    # positions rounded to float32 as the product's synthesiser receives them
    pos = np.ascontiguousarray(sample.vol.pos_of_index(idx).astype(np.float32), np.float64).reshape(-1)
    Ug = np.ascontiguousarray(np.stack([G.flat_rowmajor(G.quat_to_u(q)) for q in sample.grain_q]), np.float64)
    mask = np.zeros(g.nrot * g.detysize * g.detzsize, np.uint8)
    rc = _lib().host_simulate_mask(S9, B9, hkl, rot, R9, p, g.detysize / 2 + 0.5, g.detzsize / 2 + 0.5, pos, gid,
                                   len(gid), Ug.reshape(-1), len(sample.grain_q), int(nthreads), mask)
    assert rc == 0
    return mask.reshape(g.nrot, g.detysize, g.detzsize)


def edt_host(mask: np.ndarray, nthreads: int = 0) -> np.ndarray:
    """bwdist of every projection of ``mask`` (nrot, dety, detz) as float32."""
    m = np.ascontiguousarray(mask, np.uint8)
    out = np.empty(m.shape, np.float32)
    rc = _lib().host_edt(m.reshape(-1), m.shape[0], m.shape[1], m.shape[2], int(nthreads), out.reshape(-1))
    assert rc == 0
    return out


def distance_map_host(sample, nthreads: int = 0) -> np.ndarray:
    return edt_host(spot_mask_host(sample, nthreads), nthreads)
