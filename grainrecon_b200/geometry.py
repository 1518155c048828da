"""Crystallography and detector-geometry helpers for the completeness scorer.

These build the plain arrays that the reference MATLAB code passes to its CUDA MEX
functions (``S``, ``B``, ``hkl``, ``RotDet``, ``rot_angles`` and the 20-float
``param`` / 14-float ``param1`` vectors).  Each helper cites the reference function
it restates; all arithmetic is float64 and the arrays handed to the library are
rounded to float32 exactly as the MATLAB wrappers do with ``single(...)``.
"""
from __future__ import annotations

import dataclasses
import math
from typing import Sequence

import numpy as np

# Energy (keV) <-> wavelength (Angstrom) constant used by setup_hkl.m:21-22.
HC_KEV_A = 12.39818746


def form_b(cell: Sequence[float]) -> np.ndarray:
    """Reciprocal-lattice B matrix with the 2*pi convention (FormB.m:15-52)."""
    a, b, c = (float(x) for x in cell[:3])
    ca, cb, cg = (math.cos(math.radians(x)) for x in cell[3:6])
    sa, sb, sg = (math.sin(math.radians(x)) for x in cell[3:6])
    vol = a * b * c * math.sqrt(1 - ca * ca - cb * cb - cg * cg + 2 * ca * cb * cg)
    ast = 2 * math.pi * b * c * sa / vol
    bst = 2 * math.pi * a * c * sb / vol
    cst = 2 * math.pi * a * b * sg / vol
    sbst = vol / (a * b * c * sa * sg)
    sgst = vol / (a * b * c * sa * sb)
    cbst = (ca * cg - cb) / (sa * sg)
    cgst = (ca * cb - cg) / (sa * sb)
    bm = np.zeros((3, 3))
    bm[0, 0] = ast
    bm[0, 1] = bst * cgst
    bm[0, 2] = cst * cbst
    bm[1, 1] = bst * sgst
    bm[1, 2] = -cst * sbst * ca
    bm[2, 2] = cst * sbst * sa
    return bm


# Systematic-absence condition vectors (23 entries, meaning as in sysabs.m:13-36)
# for the two lattices the benchmark samples use: F-centred Fm-3m (Al, #225) and
# I-centred Im-3m (Fe, #229).
SYSCOND = {
    225: [0, 0, 0, 2] + [0] * 19,
    229: [0, 0, 0, 0, 2] + [0] * 18,
}


def sysabs(hkl: Sequence[int], cond: Sequence[int]) -> bool:
    """True when reflection ``hkl`` is systematically absent (sysabs.m:37-...)."""
    h, k, l = (int(x) for x in hkl)

    def bad(val, x):
        return x != 0 and abs(val) % x != 0

    absent = False
    if bad(h + k, cond[0]) or bad(h + l, cond[1]) or bad(k + l, cond[2]):
        absent = True
    if cond[3] != 0:
        x = cond[3]
        if not (abs(h + k) % x == 0 and abs(h + l) % x == 0 and abs(k + l) % x == 0):
            absent = True
    if bad(h + k + l, cond[4]) or bad(-h + k + l, cond[5]):
        absent = True
    if h == k and (bad(h, cond[6]) or bad(l, cond[7]) or bad(h + l, cond[8]) or bad(2 * h + l, cond[9])):
        absent = True
    if h == 0 and (bad(k, cond[10]) or bad(l, cond[11]) or bad(k + l, cond[12])):
        absent = True
    if k == 0 and (bad(h, cond[13]) or bad(l, cond[14]) or bad(h + l, cond[15])):
        absent = True
    if l == 0 and (bad(h, cond[16]) or bad(k, cond[17]) or bad(h + k, cond[18])):
        absent = True
    if l == 0 and h == k and bad(h, cond[19]):
        absent = True
    if abs(k) + abs(l) == 0 and bad(h, cond[20]):
        absent = True
    if abs(h) + abs(l) == 0 and bad(k, cond[21]):
        absent = True
    if abs(h) + abs(k) == 0 and bad(l, cond[22]):
        absent = True
    return absent


def gen_hkl(space_group: int, hkl_number: int, hmax: int = 8) -> np.ndarray:
    """Reflections of the first ``hkl_number`` families, Friedel mates included.

    Restates setup_hkl.m:46-60: keep every allowed (h,k,l) whose h^2+k^2+l^2 does not
    exceed the ``hkl_number``-th smallest allowed value.  The order here is by
    h^2+k^2+l^2, then lexicographic (descending) -- the reference's order comes from
    genhkl.m's segment walk; scores do not depend on reflection order.
    """
    cond = SYSCOND[space_group]
    cand = []
    rng = range(-hmax, hmax + 1)
    for h in rng:
        for k in rng:
            for l in rng:
                if h == k == l == 0 or sysabs((h, k, l), cond):
                    continue
                cand.append((h * h + k * k + l * l, h, k, l))
    sq = sorted({c[0] for c in cand})
    hkl2_max = sq[min(hkl_number, len(sq)) - 1]
    sel = sorted([c for c in cand if c[0] <= hkl2_max], key=lambda c: (c[0], -c[1], -c[2], -c[3]))
    return np.array([c[1:] for c in sel], dtype=np.float64)


def det_rot(tilt_x: float, tilt_y: float, tilt_z: float) -> np.ndarray:
    """Detector rotation RotDet = Rz*Ry*Rx, tilts in degrees (get_det_R.m:1-7)."""
    cx, sx = math.cos(math.radians(tilt_x)), math.sin(math.radians(tilt_x))
    cy, sy = math.cos(math.radians(tilt_y)), math.sin(math.radians(tilt_y))
    cz, sz = math.cos(math.radians(tilt_z)), math.sin(math.radians(tilt_z))
    rx = np.array([[1, 0, 0], [0, cx, -sx], [0, sx, cx]])
    ry = np.array([[cy, 0, sy], [0, 1, 0], [-sy, 0, cy]])
    rz = np.array([[cz, -sz, 0], [sz, cz, 0], [0, 0, 1]])
    return rz @ ry @ rx


def theta_max_deg(lsd, detysize, pxy, detzsize, pxz) -> float:
    """Half of the largest two-theta seen by the detector corner (setup_hkl.m:17-20)."""
    v = np.array([lsd, 0.5 * detysize * pxy, 0.5 * detzsize * pxz])
    c = lsd / np.linalg.norm(v)
    return math.degrees(math.acos(c)) / 2.0


def mround(x):
    """MATLAB ``round``: halves away from zero (numpy's ``round`` takes them to even)."""
    x = np.asarray(x, np.float64)
    return np.sign(x) * np.floor(np.abs(x) + 0.5)


def quat_to_u(q: Sequence[float]) -> np.ndarray:
    """Active rotation matrix from a quaternion (q0,q1,q2,q3) (quaternion2U.m:3-28)."""
    q0, q1, q2, q3 = (float(x) for x in q)
    return np.array([
        [2 * (q0 * q0 + q1 * q1) - 1, 2 * (q1 * q2 - q0 * q3), 2 * (q1 * q3 + q0 * q2)],
        [2 * (q1 * q2 + q0 * q3), 2 * (q0 * q0 + q2 * q2) - 1, 2 * (q2 * q3 - q0 * q1)],
        [2 * (q1 * q3 - q0 * q2), 2 * (q2 * q3 + q0 * q1), 2 * (q0 * q0 + q3 * q3) - 1]])


def euler_to_u(phi1: float, phi: float, phi2: float) -> np.ndarray:
    """U from Bunge Euler angles in radians (euler2u.m:5-)."""
    c1, s1 = math.cos(phi1), math.sin(phi1)
    c, s = math.cos(phi), math.sin(phi)
    c2, s2 = math.cos(phi2), math.sin(phi2)
    return np.array([
        [c1 * c2 - s1 * s2 * c, -c1 * s2 - s1 * c2 * c, s1 * s],
        [s1 * c2 + c1 * s2 * c, -s1 * s2 + c1 * c2 * c, -c1 * s],
        [s2 * s, c2 * s, c]])


def u_to_euler(u: np.ndarray) -> np.ndarray:
    """Bunge (phi1, PHI, phi2) in radians of U, the inverse of euler_to_u (euler2u.m)."""
    m = np.asarray(u, dtype=np.float64)
    phi = math.acos(max(-1.0, min(1.0, m[2, 2])))
    if abs(math.sin(phi)) < 1e-12:
        return np.array([math.atan2(m[1, 0], m[0, 0]), phi, 0.0])
    return np.array([math.atan2(m[0, 2], -m[1, 2]), phi, math.atan2(m[2, 0], m[2, 1])])


def u_to_quat(u: np.ndarray) -> np.ndarray:
    """Unit quaternion (q0 >= 0) of a rotation matrix (Shepperd's method)."""
    m = np.asarray(u, dtype=np.float64)
    tr = m[0, 0] + m[1, 1] + m[2, 2]
    cands = [tr, m[0, 0], m[1, 1], m[2, 2]]
    i = int(np.argmax(cands))
    if i == 0:
        w = math.sqrt(1 + tr) / 2
        q = [w, (m[2, 1] - m[1, 2]) / (4 * w), (m[0, 2] - m[2, 0]) / (4 * w), (m[1, 0] - m[0, 1]) / (4 * w)]
    elif i == 1:
        x = math.sqrt(1 + 2 * m[0, 0] - tr) / 2
        q = [(m[2, 1] - m[1, 2]) / (4 * x), x, (m[0, 1] + m[1, 0]) / (4 * x), (m[0, 2] + m[2, 0]) / (4 * x)]
    elif i == 2:
        y = math.sqrt(1 + 2 * m[1, 1] - tr) / 2
        q = [(m[0, 2] - m[2, 0]) / (4 * y), (m[0, 1] + m[1, 0]) / (4 * y), y, (m[1, 2] + m[2, 1]) / (4 * y)]
    else:
        z = math.sqrt(1 + 2 * m[2, 2] - tr) / 2
        q = [(m[1, 0] - m[0, 1]) / (4 * z), (m[0, 2] + m[2, 0]) / (4 * z), (m[1, 2] + m[2, 1]) / (4 * z), z]
    q = np.array(q)
    if q[0] < 0:
        q = -q
    return q / np.linalg.norm(q)


def _cubic_ops() -> np.ndarray:
    """The 24 proper rotations of the cubic point group 432 as unit quaternions."""
    ops = []
    for perm in ([0, 1, 2], [1, 2, 0], [2, 0, 1], [1, 0, 2], [0, 2, 1], [2, 1, 0]):
        for signs in np.ndindex(2, 2, 2):
            m = np.zeros((3, 3))
            for r, c in enumerate(perm):
                m[r, c] = -1.0 if signs[r] else 1.0
            if abs(np.linalg.det(m) - 1.0) < 1e-9:
                ops.append(u_to_quat(m))
    return np.array(ops)


def _qmul(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    w1, x1, y1, z1 = np.moveaxis(a, -1, 0)
    w2, x2, y2, z2 = np.moveaxis(b, -1, 0)
    return np.stack([w1 * w2 - x1 * x2 - y1 * y2 - z1 * z2,
                     w1 * x2 + x1 * w2 + y1 * z2 - z1 * y2,
                     w1 * y2 - x1 * z2 + y1 * w2 + z1 * x2,
                     w1 * z2 + x1 * y2 - y1 * x2 + z1 * w2], axis=-1)


def cubic_fz_orientations(n: int, seed: int) -> np.ndarray:
    """``n`` seeded, uniformly distributed orientations reduced to the cubic FZ.

    Stand-in for the Oh hyperspherical grids read by get_ori_set.m:10-18
    (``Ori_Oh_3deg.txt`` = 9,218 rows, ``Ori_Oh_2deg.txt`` = 32,768 rows): same count
    and the same row layout ``[q0 q1 q2 q3]`` with q0 >= 0.  Each random quaternion is
    replaced by its symmetry-equivalent with the largest scalar part.
    """
    rng = np.random.default_rng(seed)
    u1, u2, u3 = rng.random((3, n))
    q = np.stack([np.sqrt(1 - u1) * np.sin(2 * np.pi * u2), np.sqrt(1 - u1) * np.cos(2 * np.pi * u2),
                  np.sqrt(u1) * np.sin(2 * np.pi * u3), np.sqrt(u1) * np.cos(2 * np.pi * u3)], axis=1)
    ops = _cubic_ops()
    eq = _qmul(q[:, None, :], ops[None, :, :])
    best = np.argmax(np.abs(eq[:, :, 0]), axis=1)
    out = eq[np.arange(n), best]
    out[out[:, 0] < 0] *= -1
    return out


def ori_local_sampling(q: Sequence[float], nr: int, gridsize: float = 0.004) -> np.ndarray:
    """Cartesian (b,c,d) grid around ``q`` with q0 = sqrt(1-b^2-c^2-d^2).

    Restates ori_local_sampling.m:12-34: (nr+1)^3 grid points plus the centre,
    then ``unique(q,'rows')`` (sorted, duplicate rows removed).
    """
    q = np.asarray(q, dtype=np.float64)
    if q.size == 3:
        q = np.concatenate([[math.sqrt(1 - float(q @ q))], q])
    steps = np.arange(nr + 1) * gridsize - gridsize * nr / 2
    rows = [q]
    for b in q[1] + steps:
        for c in q[2] + steps:
            for d in q[3] + steps:
                rows.append(np.array([math.sqrt(1 - (b * b + c * c + d * d)), b, c, d]))
    return np.unique(np.array(rows), axis=0)


@dataclasses.dataclass
class Geometry:
    """Source/sample/detector set-up; field names follow setup_exp.m and the MEX ``param``."""

    lss: float = 11.0            # Lsam2sou [mm]
    lsd: float = 11.0            # Lsam2det [mm]
    p0y: float = 0.0
    p0z: float = 0.0
    dety00: float = 0.0
    detz00: float = 0.0
    pxy: float = 0.0672          # pixelysize [mm]
    pxz: float = 0.0672          # pixelzsize [mm]
    detysize: int = 1024
    detzsize: int = 1024
    beamstop_y: tuple = (0.0, 0.0)   # BeamStopY(1:2) [pixel]; (0,0) excludes nothing
    beamstop_z: tuple = (0.0, 0.0)
    tilt: tuple = (0.0, 0.0, 0.0)    # tilt_x/y/z [deg]
    rot_axis_offset: float = 0.0
    e_min_kev: float = 10.0
    e_max_kev: float = 70.0
    rot_angles: np.ndarray = dataclasses.field(default_factory=lambda: np.arange(0, 361, 2.0))

    @property
    def lambda_min(self) -> float:
        return HC_KEV_A / self.e_max_kev

    @property
    def lambda_max(self) -> float:
        return HC_KEV_A / self.e_min_kev

    @property
    def theta_max(self) -> float:
        return theta_max_deg(self.lsd, self.detysize, self.pxy, self.detzsize, self.pxz)

    @property
    def rot_det(self) -> np.ndarray:
        return det_rot(*self.tilt)

    @property
    def nrot(self) -> int:
        return int(len(self.rot_angles))

    def param20(self, nhkl: int) -> np.ndarray:
        """The 20-float ``param`` vector (ForwardCalc_OR_space_comp_cuda.m:25-27)."""
        return np.array([nhkl, self.nrot, self.lss, self.lsd, self.p0y, self.p0z, self.dety00,
                         self.detz00, self.pxy, self.pxz, self.detysize, self.detzsize,
                         self.beamstop_y[0], self.beamstop_y[1], self.beamstop_z[0], self.beamstop_z[1],
                         self.theta_max, self.lambda_min, self.lambda_max, self.rot_axis_offset],
                        dtype=np.float32)


@dataclasses.dataclass
class Volume:
    """Reconstruction-volume frame used to turn voxel indices into mm (param1)."""

    rec_volume_pixel: tuple = (1, 1, 1)   # RecVolumePixel(:,1)'
    simap: int = 1                        # simap_data_flag
    vox_size: float = 0.005               # VoxSize [mm]
    center: tuple = (0.0, 0.0, 0.0)       # tomo_scale.Center' [mm]
    dimension: tuple = (20, 20, 20)       # tomo_scale.Dimension

    def param14(self, seed_comp: float, drop_off: float, max_dmedian: float) -> np.ndarray:
        """The 14-float ``param1`` vector (grow_indexed_region_cuda.m:94-95)."""
        return np.array([*self.rec_volume_pixel, self.simap, self.vox_size, *self.center,
                         *self.dimension, seed_comp, drop_off, max_dmedian], dtype=np.float32)

    def pos_of_index(self, idx: np.ndarray) -> np.ndarray:
        """Voxel centre [mm] of 1-based indices (grow_indexed_region_parallel.m:70-74)."""
        idx = np.asarray(idx, dtype=np.float64)
        pos = ((idx + np.asarray(self.rec_volume_pixel, dtype=np.float64) - 1)
               - np.asarray(self.dimension, dtype=np.float64) / 2) * self.vox_size + np.asarray(self.center)
        if self.simap == 1:
            pos = pos.copy()
            pos[..., 0] = -pos[..., 0]
            pos[..., 1] = -pos[..., 1]
        return pos


def flat_rowmajor(m: np.ndarray) -> np.ndarray:
    """``single(reshape(M',1,9))``: a 3x3 matrix flattened row by row as float32."""
    return np.ascontiguousarray(np.asarray(m, dtype=np.float64).reshape(3, 3), dtype=np.float32).reshape(9)


def flat_hkl(hkl: np.ndarray) -> np.ndarray:
    """``single(reshape(hkl,1,[]))`` for a 3 x nhkl matrix: [h1 k1 l1 h2 k2 l2 ...]."""
    return np.ascontiguousarray(np.asarray(hkl, dtype=np.float32).reshape(-1, 3)).reshape(-1)
