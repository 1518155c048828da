"""Host-side mirror of GrainRecon's GPU wrappers, backed by the C ABI.

Same function names, argument order and meaning as the MATLAB files they mirror;
arrays follow MATLAB's index order (``proj_bin_bw`` is detz x dety x nrot, voxel
indices are 1-based).  Every scorer call goes through libgrainrecon_b200.so --
there is no CPU path here.

The reference re-uploads the whole distance map on every MEX call and resets the
device afterwards (ForwardCalc_OR_space_comp_cuda.m:22,42).  Here a module-level
context keeps the rank-coded map resident and re-uploads only when a different
array (by identity, shape and a content sample) is passed.
"""
from __future__ import annotations

import math

import numpy as np

from . import geometry as G
from ._lib import Context

_ctx: Context | None = None
_map_key = None


def context() -> Context:
    global _ctx
    if _ctx is None:
        _ctx = Context(0)
    return _ctx


def reset_masks():
    """Forget the resident map (call after modifying a map array in place)."""
    global _map_key
    _map_key = None


def _flat_map(proj_bin_bw) -> np.ndarray:
    """reshape(proj_bin_bw,1,[]) of a detz x dety x nrot array (column-major flatten)."""
    a = np.asarray(proj_bin_bw)
    if a.ndim == 3:
        a = a.ravel(order="F")
    return np.ascontiguousarray(a, dtype=np.float32)


def _map_for_call(proj_bin_bw):
    """The flat map when it must be (re)uploaded, else None (resident map is reused)."""
    global _map_key
    a = np.asarray(proj_bin_bw)
    # every (size/4096)-th element in C order, gathered by index: reshape(-1) of a transposed
    # view would copy the whole map on every call
    at = np.arange(0, a.size, max(1, a.size // 4096))
    sample = a[np.unravel_index(at, a.shape)] if a.ndim > 1 else a.reshape(-1)[at]
    key = (id(proj_bin_bw), a.shape, a.dtype.str, hash(np.asarray(sample, np.float32).tobytes()))
    if key == _map_key:
        return None
    _map_key = key
    return _flat_map(a)


def _param(nr_hkl, nr_rot, Lsam2sou, Lsam2det, P0y, P0z, dety00, detz00, pixelysize, pixelzsize, detysize,
           detzsize, BeamStopY, BeamStopZ, thetamax, lambda_min, lambda_max, RotAxisOffset):
    # ForwardCalc_OR_space_comp_cuda.m:25-27
    return np.array([nr_hkl, nr_rot, Lsam2sou, Lsam2det, P0y, P0z, dety00, detz00, pixelysize, pixelzsize,
                     detysize, detzsize, *np.ravel(BeamStopY)[:2], *np.ravel(BeamStopZ)[:2], thetamax,
                     lambda_min, lambda_max, RotAxisOffset], dtype=np.float32)


def _hkl(Ahkl, nrhkl):
    return np.asarray(Ahkl, dtype=np.float64)[:nrhkl, :3]


def ForwardCalc_OR_space_comp_cuda(pos, OR_q, S, B, Ahkl, nrhkl, proj_bin_bw, rot_angles, RotDet, Lsam2sou,
                                   Lsam2det, P0y, P0z, RotAxisOffset, dety00, detz00, pixelysize, pixelzsize,
                                   detysize, detzsize, BeamStopY, BeamStopZ, thetamax, lambda_min, lambda_max):
    """ForwardCalc_OR_space_comp_cuda.m:7-43.

    Returns Output (N x 8) = [Nr_simu Nr_intersect completeness dis_median q0 q1 q2 q3].
    The reference's ``nr_rot*nr_hkl > 181*80`` capacity error (:28-29) does not apply.
    """
    hkl = _hkl(Ahkl, nrhkl)
    q = np.asarray(OR_q, dtype=np.float64).reshape(-1, 4)
    param = _param(hkl.shape[0], len(rot_angles), Lsam2sou, Lsam2det, P0y, P0z, dety00, detz00, pixelysize,
                   pixelzsize, detysize, detzsize, BeamStopY, BeamStopZ, thetamax, lambda_min, lambda_max,
                   RotAxisOffset)
    out = context().forward_comp(np.asarray(pos, np.float32), q.astype(np.float32), G.flat_rowmajor(S),
                                 G.flat_rowmajor(B), G.flat_hkl(hkl), _map_for_call(proj_bin_bw),
                                 np.asarray(rot_angles, np.float32), G.flat_rowmajor(RotDet), param)
    Output = np.zeros((q.shape[0], 8))
    Output[:, :4] = out.reshape(-1, 4)
    Output[:, 4:] = q
    return Output


def _voxel_rows(I, Imask, DisMedian, vox):
    """Rows [x y z I mask DisMedian] of 1-based voxel indices (grow_indexed_region_cuda.m:71-77)."""
    v = np.asarray(vox, dtype=np.int64)
    rows = np.zeros((len(v), 6))
    rows[:, :3] = v
    ix = (v[:, 0] - 1, v[:, 1] - 1, v[:, 2] - 1)
    rows[:, 3] = np.asarray(I)[ix]
    rows[:, 4] = np.asarray(Imask)[ix]
    rows[:, 5] = np.asarray(DisMedian)[ix]
    return rows


def grow_indexed_region_cuda(I, Imask, DisMedian, Ninter, pos_indices, Spot_L, drop_off, maxD, indexed_comp, UU,
                             proj_bin_bw, rot_angles, S, B, Ahkl, nrhkl, RotDet, thetamax, lambda_min, lambda_max,
                             Lsam2sou, Lsam2det, dety00, detz00, P0y, P0z, RotAxisOffset, pixelysize, pixelzsize,
                             detysize, detzsize, BeamStopY, BeamStopZ, RecVolumePixel, tomo_scale, VoxSize,
                             simap_data_flag, maxDmedian):
    """grow_indexed_region_cuda.m:3-153.

    ``tomo_scale`` is a dict with 'Center' and 'Dimension' (3 each); ``RecVolumePixel``
    a 3 x 2 array whose first column is used.  Returns (J, Completeness_out,
    DisMedian_out, Ninter_out, center, replace_center, indexed_indices).
    """
    I = np.array(I, dtype=np.float64, copy=True)
    x, y, z = (int(p) for p in pos_indices)
    I[x - 1, y - 1, z - 1] = indexed_comp                                            # :32
    J = np.zeros(I.shape)
    J[x - 1, y - 1, z - 1] = 2
    Completeness_out = I.copy()
    DisMedian_out = np.array(DisMedian, dtype=np.float64, copy=True)
    Ninter_out = np.array(Ninter, dtype=np.float64, copy=True)
    seed_comp = I[x - 1, y - 1, z - 1]                                               # :39
    csum = seed_comp
    cpos = seed_comp * np.array([x, y, z], dtype=np.float64)
    center0 = cpos / csum
    Box_L = math.ceil(Spot_L * np.mean([pixelysize, pixelzsize]) / ((Lsam2det / Lsam2sou) * VoxSize))  # :44
    box = np.zeros((3, 2), dtype=np.int64)
    for i, p in enumerate((x, y, z)):                                                # :46-57
        box[i, 0] = p - Box_L if p - Box_L > 0 else 1
        box[i, 1] = p + Box_L if p + Box_L < I.shape[i] else I.shape[i]
    # meshgrid(x,y,z) order: y varies fastest along the first dimension
    xg, yg, zg = np.meshgrid(np.arange(box[0, 0], box[0, 1] + 1), np.arange(box[1, 0], box[1, 1] + 1),
                             np.arange(box[2, 0], box[2, 1] + 1))
    vox = np.stack([xg.ravel(order="F"), yg.ravel(order="F"), zg.ravel(order="F")], 1)  # :58-59
    cp = G.mround(box[:, 1] - box[:, 0]) / 2 + box[:, 0]                             # :61
    dis = np.sqrt(((vox - cp[None, :]) ** 2).sum(1))
    vox = vox[dis <= Box_L]                                                          # :66
    rows = _voxel_rows(I, Imask, DisMedian, vox)
    hkl = _hkl(Ahkl, nrhkl)
    param = _param(hkl.shape[0], len(rot_angles), Lsam2sou, Lsam2det, P0y, P0z, dety00, detz00, pixelysize,
                   pixelzsize, detysize, detzsize, BeamStopY, BeamStopZ, thetamax, lambda_min, lambda_max,
                   RotAxisOffset)
    param1 = np.array([*np.asarray(RecVolumePixel)[:, 0], simap_data_flag, VoxSize, *tomo_scale["Center"],
                       *tomo_scale["Dimension"], seed_comp, drop_off, maxDmedian], dtype=np.float32)  # :94-95
    out = context().grow_indexed_region(rows, G.flat_rowmajor(UU), G.flat_rowmajor(S), G.flat_rowmajor(B),
                                        G.flat_hkl(hkl), _map_for_call(proj_bin_bw),
                                        np.asarray(rot_angles, np.float32), G.flat_rowmajor(RotDet), param,
                                        param1).reshape(-1, 7)
    acc = out[out[:, 6] == 1]                                                        # :117
    ix = tuple(acc[:, :3].astype(np.int64).T - 1)                                    # :118-128
    J[ix] = 2
    Completeness_out[ix] = acc[:, 4] / acc[:, 3]
    DisMedian_out[ix] = acc[:, 5]
    Ninter_out[ix] = acc[:, 4]
    J = J > 1                                                                        # :131
    idx = np.argwhere(np.asfortranarray(J).transpose(2, 1, 0)).astype(np.int64)[:, ::-1] + 1  # ind2sub(find(J)) order
    if len(idx) > 1:                                                                 # :134-142
        c = Completeness_out[tuple((idx - 1).T)]
        # running sums in find() order (add.accumulate adds one term at a time, as the loop does)
        csum = np.add.accumulate(np.concatenate([[csum], c]))[-1]
        cpos = np.add.accumulate(np.concatenate([cpos[None], c[:, None] * idx]), axis=0)[-1]
    center1 = cpos / csum                                                            # :144
    if np.sqrt(((center1 - center0) ** 2).sum()) > max(maxD, maxD / 10000 * len(idx)):
        center, replace_center = G.mround(center1), 1
    else:
        center, replace_center = center0, 0
    return J, Completeness_out, DisMedian_out, Ninter_out, center, replace_center, idx


def Forward_calc_comp_allvoxel_cuda(I, Imask, DisMedian, Ninter, voxel_waiting_growth0, maxD, UU, proj_bin_bw,
                                    rot_angles, S, B, Ahkl, nrhkl, RotDet, thetamax, lambda_min, lambda_max,
                                    Lsam2sou, Lsam2det, dety00, detz00, P0y, P0z, RotAxisOffset, pixelysize,
                                    pixelzsize, detysize, detzsize, BeamStopY, BeamStopZ, RecVolumePixel,
                                    tomo_scale, VoxSize, simap_data_flag, maxDmedian):
    """Forward_calc_comp_allvoxel_cuda.m:3-78: score every listed voxel with one U."""
    Completeness_out = np.array(I, dtype=np.float64, copy=True)
    DisMedian_out = np.array(DisMedian, dtype=np.float64, copy=True)
    Ninter_out = np.array(Ninter, dtype=np.float64, copy=True)
    rows = _voxel_rows(I, Imask, DisMedian, voxel_waiting_growth0)
    hkl = _hkl(Ahkl, nrhkl)
    param = _param(hkl.shape[0], len(rot_angles), Lsam2sou, Lsam2det, P0y, P0z, dety00, detz00, pixelysize,
                   pixelzsize, detysize, detzsize, BeamStopY, BeamStopZ, thetamax, lambda_min, lambda_max,
                   RotAxisOffset)
    param1 = np.array([*np.asarray(RecVolumePixel)[:, 0], simap_data_flag, VoxSize, *tomo_scale["Center"],
                       *tomo_scale["Dimension"], 0, 0, maxDmedian], dtype=np.float32)  # :46-47
    out = context().grow_indexed_region(rows, G.flat_rowmajor(UU), G.flat_rowmajor(S), G.flat_rowmajor(B),
                                        G.flat_hkl(hkl), _map_for_call(proj_bin_bw),
                                        np.asarray(rot_angles, np.float32), G.flat_rowmajor(RotDet), param,
                                        param1).reshape(-1, 7)
    with np.errstate(invalid="ignore", divide="ignore"):
        ix = tuple(out[:, :3].astype(np.int64).T - 1)                                # :69-76
        Completeness_out[ix] = out[:, 4] / out[:, 3]
        DisMedian_out[ix] = out[:, 5]
        Ninter_out[ix] = out[:, 4]
        Comp_max = np.nanmax(out[:, 4] / out[:, 3]) if len(out) else np.nan          # :77
    return Completeness_out, DisMedian_out, Ninter_out, Comp_max


def grow_unindexed_compete_comp_cuda(DS_in, wait_revising_voxels, id_neigb_all, id_neigb_ind, proj_bin_bw,
                                     rot_angles, S, B, Ahkl, nrhkl, RotDet, thetamax, lambda_min, lambda_max,
                                     Lsam2sou, Lsam2det, dety00, detz00, P0y, P0z, RotAxisOffset, pixelysize,
                                     pixelzsize, detysize, detzsize, BeamStopY, BeamStopZ, RecVolumePixel,
                                     tomo_scale, VoxSize, simap_data_flag):
    """grow_unindexed_compete_comp_cuda.m:3-65.

    ``DS_in`` is a dict with 'EulerAngle' (n_grain x 3, degrees) and the maps
    'Completeness', 'GrainId', 'Dismedian', 'Ninter', 'VisitFlag' (updated copies
    are returned).  ``id_neigb_ind`` holds the 1-based [first last] range per voxel.
    """
    DS_out = {k: (np.array(v, copy=True) if isinstance(v, np.ndarray) else v) for k, v in DS_in.items()}
    rows5 = np.concatenate([np.asarray(wait_revising_voxels, np.float64),
                            np.asarray(id_neigb_ind, np.float64)], axis=1)            # :12
    hkl = _hkl(Ahkl, nrhkl)
    param = _param(hkl.shape[0], len(rot_angles), Lsam2sou, Lsam2det, P0y, P0z, dety00, detz00, pixelysize,
                   pixelzsize, detysize, detzsize, BeamStopY, BeamStopZ, thetamax, lambda_min, lambda_max,
                   RotAxisOffset)
    param1 = np.array([*np.asarray(RecVolumePixel)[:, 0], simap_data_flag, VoxSize, *tomo_scale["Center"],
                       *tomo_scale["Dimension"]], dtype=np.float32)                    # :29
    out = context().forward_comp_compete(rows5, np.asarray(id_neigb_all, np.float32),
                                         np.asarray(DS_in["EulerAngle"], np.float32), G.flat_rowmajor(S),
                                         G.flat_rowmajor(B), G.flat_hkl(hkl), _map_for_call(proj_bin_bw),
                                         np.asarray(rot_angles, np.float32), G.flat_rowmajor(RotDet), param,
                                         param1).reshape(-1, 8)
    ix = tuple(np.asarray(wait_revising_voxels, np.int64).T - 1)                      # :51-64
    DS_out["Completeness"][ix] = out[:, 5]
    DS_out["GrainId"][ix] = out[:, 4]
    DS_out["Dismedian"][ix] = out[:, 7]
    DS_out["Ninter"][ix] = out[:, 6]
    DS_out["VisitFlag"][ix] = 0.5
    return DS_out, out


def grow_indexed_region(I, Imask, DisMedian, Ninter, pos_indices, drop_off, maxD, indexed_comp, UU, proj_bin_bw,
                        rot_angles, S, B, Ahkl, nrhkl, RotDet, thetamax, lambda_min, lambda_max, Lsam2sou, Lsam2det,
                        minEucDis, dety00, detz00, P0y, P0z, RotAxisOffset, pixelysize, pixelzsize, dety0, detz0,
                        detysize, detzsize, BeamStopY, BeamStopZ, RecVolumePixel, tomo_scale, VoxSize,
                        simap_data_flag, maxDmedian):
    """grow_indexed_region.m:1-145: best-first growth from the seed voxel in the library's native
    walk (grc_grow_best_first), its voxels scored on the GPU a block at a time.  ``minEucDis``,
    ``dety0`` and ``detz0`` must equal the scorer's options (0.5 px threshold, detector centre).
    Returns (J, Completeness_out, DisMedian_out, Ninter_out, center, replace_center,
    indexed_indices)."""
    hkl = _hkl(Ahkl, nrhkl)
    param = _param(hkl.shape[0], len(rot_angles), Lsam2sou, Lsam2det, P0y, P0z, dety00, detz00, pixelysize,
                   pixelzsize, detysize, detzsize, BeamStopY, BeamStopZ, thetamax, lambda_min, lambda_max,
                   RotAxisOffset)
    param1 = np.array([*np.asarray(RecVolumePixel)[:, 0], simap_data_flag, VoxSize, *tomo_scale["Center"],
                       *tomo_scale["Dimension"], 0, 0, maxDmedian], dtype=np.float32)
    return context().grow_best_first(I, Imask, DisMedian, Ninter, pos_indices, drop_off, maxD, indexed_comp,
                                     maxDmedian, G.flat_rowmajor(UU), G.flat_rowmajor(S), G.flat_rowmajor(B),
                                     G.flat_hkl(hkl), _map_for_call(proj_bin_bw), np.asarray(rot_angles, np.float32),
                                     G.flat_rowmajor(RotDet), param, param1)
