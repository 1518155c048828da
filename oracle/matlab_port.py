"""Line-by-line numpy transliteration of forward_comp.m -- TEST INFRASTRUCTURE ONLY.

A second, independent restatement of the reference scorer, written to mirror the
MATLAB text statement by statement (vectorised over reflections as the .m file is),
so that the C oracle (grc_oracle.c) can be checked against it and golden vectors
can be produced without MATLAB.  Parity status: unpinned (no MATLAB here).

Used only by tests/ and tests/golden/make_golden.py.
"""
from __future__ import annotations

import numpy as np


def _mround(x):
    """MATLAB round(): half away from zero."""
    return np.sign(x) * np.floor(np.abs(x) + 0.5)


def forward_comp(U, proj_bin_bw, pos, rot_angles, S, B, Ahkl, nrhkl, RotDet, thetamax, lambda_min, lambda_max,
                 Lsam2sou, Lsam2det, minEucDis, dety00, detz00, P0y, P0z, RotAxisOffset, pixelysize, pixelzsize,
                 dety0, detz0, detysize, detzsize, BeamStopY, BeamStopZ, edge_px=1e-4):
    """forward_comp.m:4-90.  ``proj_bin_bw`` is indexed (detz, dety, omega), 1-based in MATLAB.

    Returns (Nr_simu, Nr_intersect, dis_median, n_edge); n_edge counts reflections inside
    the wavelength/Bragg window whose unrounded pixel coordinate lies within ``edge_px``
    of a rounding boundary, or whose wavelength lies within 1e-9 (relative) of the window.
    """
    n_edge = 0
    L = Lsam2sou + Lsam2det                                                     # :8
    Nr_simu = 0                                                                 # :9
    Nr_intersect = 0                                                            # :10
    SimuSpots = []                                                              # :13
    hkl = np.asarray(Ahkl, dtype=np.float64)[:nrhkl, 0:3].T                     # :15
    Gw = S @ U @ B @ hkl                                                        # :16
    pos = np.array(pos, dtype=np.float64).reshape(1, 3)
    pos[:, 1] = pos[:, 1] - RotAxisOffset                                       # :17
    for i in range(len(rot_angles)):                                            # :18
        omega = rot_angles[i] * np.pi / 180                                     # :19
        Omega = np.array([[np.cos(omega), -np.sin(omega), 0], [np.sin(omega), np.cos(omega), 0], [0, 0, 1]])
        SamposW = Omega @ S @ pos.T                                             # :22
        SamposW = SamposW[:, 0]
        center = np.array([L, (SamposW[1] - P0y + RotAxisOffset) * L / (Lsam2sou + SamposW[0]),
                           (SamposW[2] - P0z) * L / (Lsam2sou + SamposW[0])])   # :23-24
        alpha = np.arctan(np.sqrt((SamposW[1] - P0y + RotAxisOffset) ** 2 + (SamposW[2] - P0z) ** 2)
                          / (Lsam2sou + SamposW[0]))                            # :25
        grainpos = np.array([Lsam2sou + SamposW[0], SamposW[1] - P0y + RotAxisOffset, SamposW[2] - P0z])  # :26
        Gt = Omega @ Gw                                                         # :28
        v1 = np.vstack([np.zeros(hkl.shape[1]), Gt[1, :], Gt[2, :]])            # :29
        Glen = (Gt[0, :] ** 2 + Gt[1, :] ** 2 + Gt[2, :] ** 2) ** 0.5           # :30
        gpn = grainpos / np.linalg.norm(grainpos)
        beta = np.arccos(np.clip((gpn[:, None] * (Gt / Glen)).sum(0), -1, 1))  # :31
        theta = beta - np.pi / 2                                                # :33
        sintth = np.sin(2 * theta)                                              # :34
        d = 1.0 / Glen * 2 * np.pi                                              # :36
        lambdahkl = 2 * d * np.sin(theta)                                       # :37
        v1n = v1 / np.sqrt(v1[0, :] ** 2 + v1[1, :] ** 2 + v1[2, :] ** 2)
        cn = center / np.linalg.norm(center)
        with np.errstate(invalid="ignore", divide="ignore"):
            phix = np.arccos(np.clip((v1n * cn[:, None]).sum(0), -1, 1))      # :40
            phiy = phix - 2 * theta                                             # :41
            L2 = (Lsam2det - SamposW[0]) / np.cos(alpha)                        # :42
            diffvec = L2 * sintth / np.sin(phiy)                                # :43
            konst = np.sqrt(Gt[1, :] ** 2 + Gt[2, :] ** 2)                      # :44
            dety22 = center[1] + diffvec * Gt[1, :] / konst                     # :46
            detz22 = center[2] + diffvec * Gt[2, :] / konst                     # :47
            K = np.vstack([np.full(hkl.shape[1], Lsam2det), dety22, detz22]) - SamposW[:, None]
            K_out_unit = K / ((Lsam2det - SamposW[0]) ** 2 + (dety22 - SamposW[1]) ** 2
                              + (detz22 - SamposW[2]) ** 2) ** 0.5              # :49-50
            t = ((RotDet[0, 0] * (Lsam2det - SamposW[0]) + RotDet[1, 0] * (dety00 - RotAxisOffset - SamposW[1])
                  + RotDet[2, 0] * (detz00 - SamposW[2]))
                 / (RotDet[0, 0] * K_out_unit[0, :] + RotDet[1, 0] * K_out_unit[1, :]
                    + RotDet[2, 0] * K_out_unit[2, :]))                         # :51-52
            off = np.array([SamposW[0] - Lsam2det, SamposW[1] - dety00 + RotAxisOffset, SamposW[2] - detz00])
            vv = t * K_out_unit + off[:, None]
            dety22 = np.array([RotDet[0, 1], RotDet[1, 1], RotDet[2, 1]]) @ vv  # :54
            detz22 = np.array([RotDet[0, 2], RotDet[1, 2], RotDet[2, 2]]) @ vv  # :55
            dety = _mround(-dety22 / pixelysize + dety0)                        # :58
            detz = _mround(-detz22 / pixelzsize + detz0)                        # :59
            select3 = np.nonzero((beta > np.pi / 2) & (beta < (90 + thetamax * 4) / 180 * np.pi)
                                 & (lambdahkl > lambda_min) & (lambdahkl < lambda_max)
                                 & (dety >= 1) & (dety <= detysize) & (detz >= 1) & (detz <= detzsize)
                                 & ~((dety >= BeamStopY[0]) & (dety <= BeamStopY[1])
                                     & (detz >= BeamStopZ[0]) & (detz <= BeamStopZ[1])))[0]  # :61-65
            u = -dety22 / pixelysize + dety0
            v = -detz22 / pixelzsize + detz0
            inwin = (beta > np.pi / 2) & (beta < (90 + thetamax * 4) / 180 * np.pi) & \
                (lambdahkl > lambda_min) & (lambdahkl < lambda_max)
            lam_edge = (np.abs(lambdahkl - lambda_min) <= 1e-9 * lambda_min) | \
                (np.abs(lambdahkl - lambda_max) <= 1e-9 * lambda_max)
            near = np.isfinite(u) & np.isfinite(v) & (u > -2) & (v > -2) & (u < detysize + 3) & (v < detzsize + 3)
            pix_edge = near & ((np.abs(u - np.floor(u) - 0.5) < edge_px) | (np.abs(v - np.floor(v) - 0.5) < edge_px))
            n_edge += int(((inwin | lam_edge) & pix_edge | lam_edge).sum())
        if select3.size:                                                        # :66
            Nr_simu = Nr_simu + len(select3)                                    # :67
            for j in select3:                                                   # :68
                dis = float(proj_bin_bw[int(detz[j]) - 1, int(dety[j]) - 1, i])  # :69
                if dis <= minEucDis / np.mean([pixelysize, pixelzsize]):        # :71
                    Nr_intersect = Nr_intersect + 1                             # :72
                SimuSpots.append(dis)                                           # :79-80 (column 8)
    if SimuSpots:                                                               # :86
        s = np.sort(np.array(SimuSpots))
        n = s.size
        dis_median = s[n // 2] if n % 2 else (s[n // 2 - 1] + s[n // 2]) / 2   # :87 (MATLAB median)
    else:
        dis_median = 2000.0                                                     # :89
    return Nr_simu, Nr_intersect, dis_median, n_edge


def forward_comp_mex_args(U, pos, S9, B9, hkl_flat, proj_flat, rot_angles, R9, param, dety0=None, detz0=None,
                          thr=0.5):
    """forward_comp on the MEX argument layouts (float32 inputs promoted to double)."""
    p = np.asarray(param, dtype=np.float32).astype(np.float64)
    nhkl, nrot = int(p[0]), int(p[1])
    detysize, detzsize = int(p[10]), int(p[11])
    if dety0 is None:
        dety0 = detysize / 2 + 0.5
    if detz0 is None:
        detz0 = detzsize / 2 + 0.5
    f64 = lambda a: np.asarray(a, dtype=np.float32).astype(np.float64)
    S = f64(S9).reshape(3, 3)
    B = f64(B9).reshape(3, 3)
    R = f64(R9).reshape(3, 3)
    Ahkl = f64(hkl_flat).reshape(-1, 3)
    proj = np.asarray(proj_flat, dtype=np.float32).reshape(nrot, detysize, detzsize).transpose(2, 1, 0)
    pxy, pxz = p[8], p[9]
    return forward_comp(np.asarray(U, np.float64).reshape(3, 3), proj, f64(pos), f64(rot_angles), S, B, Ahkl, nhkl,
                        R, p[16], p[17], p[18], p[2], p[3], thr * (pxy + pxz) / 2, p[6], p[7], p[4], p[5], p[19],
                        pxy, pxz, dety0, detz0, detysize, detzsize, p[12:14], p[14:16])
