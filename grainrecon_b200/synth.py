"""Seeded synthetic samples, spot masks and distance maps.

The reference's example data (spot .mat files, ground-truth h5, 1-degree grids) is
not available, so benchmarks and tests run on synthetic samples with the shapes of
the reference's configurations:

* a cylinder of voxels split into grains by a seeded (power-weighted) Voronoi
  tessellation, one uniformly random orientation per grain;
* spot masks forward-simulated from that ground truth with the point-voxel model
  of forward_comp.m (a pixel is a spot pixel when some voxel of some grain lands a
  selected reflection on it);
* the distance map ``proj_bin_bw = bwdist(mask)`` of GrainMapping_fun.m:73-75, i.e.
  the Euclidean distance of every pixel to the nearest spot pixel (0 on spots).

Small samples are synthesised with host-side numpy; large volumes use the library's
device-side spot simulator and EDT instead (``device_maps``).
"""
from __future__ import annotations

import dataclasses

import numpy as np

from . import geometry as G


@dataclasses.dataclass
class Sample:
    geom: G.Geometry
    vol: G.Volume
    cell: tuple
    space_group: int
    B: np.ndarray                 # 3x3
    hkl: np.ndarray               # nhkl x 3
    S: np.ndarray                 # 3x3
    grain_id: np.ndarray          # Dim int32 (0 = outside the cylinder)
    grain_q: np.ndarray           # ngrain x 4 ground-truth quaternions (row g-1 = grain g)
    seed: int = 0

    @property
    def nhkl(self) -> int:
        return int(self.hkl.shape[0])

    def voxel_indices(self) -> np.ndarray:
        """1-based (x,y,z) indices of every voxel inside the sample, in C order."""
        idx = np.argwhere(self.grain_id > 0) + 1
        return idx.astype(np.int64)

    def mex_arrays(self):
        """(S9, B9, hkl_flat, rot_angles, RotDet9, param20) as the MATLAB wrappers build them."""
        return (G.flat_rowmajor(self.S), G.flat_rowmajor(self.B), G.flat_hkl(self.hkl),
                np.asarray(self.geom.rot_angles, np.float32), G.flat_rowmajor(self.geom.rot_det),
                self.geom.param20(self.nhkl))


def voronoi_sites(dim: int, n_grains: int, seed: int, lognormal_sigma: float = 0.0):
    """Seeded sites (n x 3, inside the cylinder) and squared weights (n) of the power diagram
    that ``voronoi_cylinder`` and ``voronoi_cylinder_torch`` partition the volume with."""
    rng = np.random.default_rng(seed)
    r = dim / 2.0
    sites = []
    while len(sites) < n_grains:
        p = rng.random(3) * dim
        if (p[0] - r) ** 2 + (p[1] - r) ** 2 <= r * r:
            sites.append(p)
    sites = np.array(sites)
    mean_d = dim / max(n_grains, 1) ** (1 / 3)
    w2 = np.zeros(n_grains)
    if lognormal_sigma > 0:
        w = rng.lognormal(mean=0.0, sigma=lognormal_sigma, size=n_grains) * mean_d * 0.5
        w2 = w * w
    return sites, w2


def voronoi_cylinder(dim: int, n_grains: int, seed: int, lognormal_sigma: float = 0.0) -> np.ndarray:
    """Grain-id volume (dim^3, int32) of a cylinder along z split by a seeded Voronoi.

    With ``lognormal_sigma > 0`` each site gets a log-normal weight and voxels go to
    the site minimising |x-c|^2 - w^2 (a power diagram), which spreads grain sizes.
    """
    r = dim / 2.0
    ax = np.arange(dim) + 0.5
    X, Y, Z = np.meshgrid(ax, ax, ax, indexing="ij")
    inside = (X - r) ** 2 + (Y - r) ** 2 <= r * r
    sites, w2 = voronoi_sites(dim, n_grains, seed, lognormal_sigma)
    pts = np.stack([X[inside], Y[inside], Z[inside]], axis=1)
    best = np.zeros(len(pts), np.int32)
    chunk = 1 << 16
    for s in range(0, len(pts), chunk):
        p = pts[s:s + chunk]
        d = ((p[:, None, :] - sites[None, :, :]) ** 2).sum(-1) - w2[None, :]
        best[s:s + chunk] = np.argmin(d, axis=1).astype(np.int32) + 1
    gid = np.zeros((dim, dim, dim), np.int32)
    gid[inside] = best
    return gid


def named_setup(kind: str, seed: int = 1, **over):
    """Geometry, lattice and grid of a named sample: (geom, cell, space_group, hkl, dim, n_grains,
    voxel_mm, lognormal_sigma).  The volume itself is not built."""
    rng = np.random.default_rng(seed + 1000)
    tilt = tuple(rng.uniform(-0.5, 0.5, 3))
    if kind in ("fe6", "fe_small", "fe_tiny"):
        cell = (2.8665, 2.8665, 2.8665, 90, 90, 90)
        sg = 229
        if kind == "fe6":
            dim, ng, det, px, rot = 20, 6, 1024, 0.0672, np.arange(0, 361, 2.0)
        elif kind == "fe_small":
            dim, ng, det, px, rot = 12, 6, 256, 0.2688, np.arange(0, 361, 10.0)
        else:
            dim, ng, det, px, rot = 8, 3, 128, 0.5376, np.arange(0, 361, 30.0)
        vox = 0.1 / dim
        sigma = 0.0
    elif kind in ("al400", "al_small"):
        cell = (4.0495, 4.0495, 4.0495, 90, 90, 90)
        sg = 225
        if kind == "al400":
            dim, ng, det, px, rot = 160, 400, 2048, 0.0336, np.arange(0, 361, 1.0)
        else:
            dim, ng, det, px, rot = 24, 20, 512, 0.1344, np.arange(0, 361, 5.0)
        vox = 0.4 / dim
        sigma = 0.4
    else:
        raise ValueError(kind)
    geom = G.Geometry(pxy=px, pxz=px, detysize=det, detzsize=det, tilt=tilt, rot_angles=rot)
    for k, v in over.items():
        setattr(geom, k, v)
    return geom, cell, sg, G.gen_hkl(sg, 6), dim, ng, vox, sigma


def make_sample(kind: str = "fe_small", seed: int = 1, voronoi=None, **over) -> Sample:
    """Named synthetic samples.

    ``fe6``   : BCC Fe a=2.8665, 6 grains, 100 um cylinder at 5 um (20^3 grid, ~6.3k voxels),
                6 families (86 reflections), 1024^2 detector at 0.0672 mm, Lss=Lsd=11 mm,
                tilts U(-0.5,0.5) deg, 181 projections 0:2:360, E 10-70 keV.
    ``al400`` : FCC Al a=4.0495, 400 grains log-normal (sigma 0.4), 400 um cylinder at 2.5 um
                (160^3 grid, ~3.2M voxels), 6 families (64 reflections), 2048^2 detector at
                0.0336 mm, 361 projections 0:1:360.
    ``fe_small``: the fe6 set-up shrunk for fast CPU tests (12^3 grid, 256^2 detector at
                0.2688 mm, 37 projections 0:10:360).

    ``voronoi(dim, n_grains, seed, sigma)`` replaces the grain-id generator (by default numpy,
    or torch on a GPU for grids of 64^3 and more; all take the sites of ``voronoi_sites``).
    """
    geom, cell, sg, hkl, dim, ng, vox, sigma = named_setup(kind, seed, **over)
    vol = G.Volume(rec_volume_pixel=(1, 1, 1), simap=1, vox_size=vox, center=(0.0, 0.0, 0.0),
                   dimension=(dim, dim, dim))
    if voronoi is not None:
        use_torch = False
    elif dim >= 64:
        try:
            import torch
            use_torch = torch.cuda.is_available()
        except ImportError:
            use_torch = False
    else:
        use_torch = False
    if voronoi is not None:
        gid = np.asarray(voronoi(dim, ng, seed, sigma), np.int32)
    elif use_torch:
        gid = voronoi_cylinder_torch(dim, ng, seed, sigma).cpu().numpy()
    else:
        gid = voronoi_cylinder(dim, ng, seed, sigma)
    q = G.cubic_fz_orientations(ng, seed + 7)
    return Sample(geom=geom, vol=vol, cell=cell, space_group=sg, B=G.form_b(cell), hkl=hkl, S=np.eye(3),
                  grain_id=gid, grain_q=q, seed=seed)


def landing_pixels(sample: Sample, pos: np.ndarray, U: np.ndarray, dety0=None, detz0=None):
    """Selected landing pixels of many (pos, U) trials -- algebraic form, float64.

    ``pos``: n x 3 [mm]; ``U``: n x 3 x 3.  Returns (iw, dety, detz) int arrays (1-based
    pixel indices) of every selected reflection.  Used only to synthesise masks.
    """
    g = sample.geom
    f = lambda a: np.asarray(np.asarray(a, np.float32), np.float64)
    S = f(G.flat_rowmajor(sample.S)).reshape(3, 3)
    B = f(G.flat_rowmajor(sample.B)).reshape(3, 3)
    R = f(G.flat_rowmajor(g.rot_det)).reshape(3, 3)
    p = f(g.param20(sample.nhkl))
    lss, lsd, p0y, p0z, y00, z00, pxy, pxz = p[2:10]
    ny, nz = int(p[10]), int(p[11])
    bs = p[12:16]
    tmax, lmin, lmax, rao = p[16:20]
    dety0 = ny / 2 + 0.5 if dety0 is None else dety0
    detz0 = nz / 2 + 0.5 if detz0 is None else detz0
    hkl = f(sample.hkl)
    pos = f(pos).copy()
    pos[:, 1] -= rao
    Sp = pos @ S.T
    Gw = np.einsum("ij,njk,kl,hl->nhi", S, f(U), B, hkl)          # n x nhkl x 3
    Glen = np.linalg.norm(Gw, axis=-1)
    cbmax = np.cos(np.radians(90 + 4 * tmax)) if 90 + 4 * tmax < 180 else -2.0
    out = []
    for iw, w in enumerate(f(g.rot_angles)):
        c, s = np.cos(np.radians(w)), np.sin(np.radians(w))
        SW = np.stack([c * Sp[:, 0] - s * Sp[:, 1], s * Sp[:, 0] + c * Sp[:, 1], Sp[:, 2]], 1)
        gp = np.stack([lss + SW[:, 0], SW[:, 1] - p0y + rao, SW[:, 2] - p0z], 1)
        ngp = np.linalg.norm(gp, axis=1)
        k = gp / ngp[:, None]
        L2 = (lsd - SW[:, 0]) * ngp / gp[:, 0]
        L = lss + lsd
        a = np.stack([lsd - SW[:, 0], gp[:, 1] * L / gp[:, 0] - SW[:, 1], gp[:, 2] * L / gp[:, 0] - SW[:, 2]], 1)
        dv = np.stack([SW[:, 0] - lsd, SW[:, 1] - y00 + rao, SW[:, 2] - z00], 1)
        num = -(dv @ R[:, 0])
        Gt = np.stack([c * Gw[..., 0] - s * Gw[..., 1], s * Gw[..., 0] + c * Gw[..., 1], Gw[..., 2]], -1)
        x = np.einsum("ni,nhi->nh", k, Gt) / Glen
        lam = -2 * (2 * np.pi / Glen) * x
        ok = (x < 0) & (x > cbmax) & (lam > lmin) & (lam < lmax)
        if not ok.any():
            continue
        ni, hi = np.nonzero(ok)
        xs = x[ni, hi]
        st = -xs
        ct = np.sqrt(1 - xs * xs)
        s2, c2 = 2 * st * ct, 1 - 2 * st * st
        gt = Gt[ni, hi]
        konst = np.hypot(gt[:, 1], gt[:, 2])
        gy, gz = gt[:, 1] / konst, gt[:, 2] / konst
        kk = k[ni]
        cphx = gy * kk[:, 1] + gz * kk[:, 2]
        sphx = np.sqrt(np.maximum(0, 1 - cphx * cphx))
        with np.errstate(divide="ignore", invalid="ignore"):
            diff = L2[ni] * s2 / (sphx * c2 - cphx * s2)
            K = a[ni] + np.stack([np.zeros_like(diff), diff * gy, diff * gz], 1)
            fK = num[ni] / (K @ R[:, 0])
            y2 = fK * (K @ R[:, 1]) + dv[ni] @ R[:, 1]
            z2 = fK * (K @ R[:, 2]) + dv[ni] @ R[:, 2]
            u = dety0 - y2 / pxy
            v = detz0 - z2 / pxz
        iu, iv = np.floor(u + 0.5), np.floor(v + 0.5)
        sel = (iu >= 1) & (iu <= ny) & (iv >= 1) & (iv <= nz) & ~(
            (iu >= bs[0]) & (iu <= bs[1]) & (iv >= bs[2]) & (iv <= bs[3]))
        out.append((np.full(int(sel.sum()), iw), iu[sel].astype(np.int64), iv[sel].astype(np.int64)))
    if not out:
        z = np.zeros(0, np.int64)
        return z, z, z
    return tuple(np.concatenate([o[i] for o in out]) for i in range(3))


def simulate_mask(sample: Sample, stride: int = 1, chunk: int = 2048) -> np.ndarray:
    """Boolean spot mask (nrot, detysize, detzsize) from the ground-truth grains."""
    g = sample.geom
    mask = np.zeros((g.nrot, g.detysize, g.detzsize), bool)
    idx = sample.voxel_indices()[::stride]
    gid = sample.grain_id[idx[:, 0] - 1, idx[:, 1] - 1, idx[:, 2] - 1]
    pos = sample.vol.pos_of_index(idx)
    Us = np.stack([G.quat_to_u(q) for q in sample.grain_q])[gid - 1]
    for s in range(0, len(idx), chunk):
        iw, iy, iz = landing_pixels(sample, pos[s:s + chunk], Us[s:s + chunk])
        mask[iw, iy - 1, iz - 1] = True
    return mask


def distance_map(mask: np.ndarray) -> np.ndarray:
    """bwdist per projection: Euclidean distance to the nearest spot pixel (float32).

    Layout (nrot, dety, detz) in C order, which is the MATLAB (detz, dety, nrot)
    column-major array flattened by ``reshape(proj_bin_bw,1,[])``.  A projection
    with no spot pixel is all +Inf, as bwdist returns.
    """
    from scipy.ndimage import distance_transform_edt

    out = np.empty(mask.shape, np.float32)
    for i in range(mask.shape[0]):
        if mask[i].any():
            out[i] = distance_transform_edt(~mask[i]).astype(np.float32)
        else:
            out[i] = np.inf
    return out


def voronoi_cylinder_torch(dim: int, n_grains: int, seed: int, lognormal_sigma: float = 0.0, device="cuda"):
    """``voronoi_cylinder`` evaluated with torch on ``device`` (same sites and weights)."""
    import torch

    r = dim / 2.0
    s_np, w_np = voronoi_sites(dim, n_grains, seed, lognormal_sigma)
    sites = torch.tensor(s_np, dtype=torch.float64, device=device)
    w2 = torch.tensor(w_np, dtype=torch.float64, device=device)
    ax = torch.arange(dim, dtype=torch.float64, device=device) + 0.5
    gid = torch.zeros((dim, dim, dim), dtype=torch.int32, device=device)
    for ix in range(dim):
        Y, Z = torch.meshgrid(ax, ax, indexing="ij")
        X = torch.full_like(Y, float(ax[ix]))
        inside = (X - r) ** 2 + (Y - r) ** 2 <= r * r
        pts = torch.stack([X[inside], Y[inside], Z[inside]], 1)
        if pts.shape[0] == 0:
            continue
        d = ((pts[:, None, :] - sites[None, :, :]) ** 2).sum(-1) - w2[None, :]
        sl = gid[ix]
        sl[inside] = (torch.argmin(d, dim=1) + 1).to(torch.int32)
    return gid


def device_maps(sample: Sample, ctx, keep_host_map: bool = False):
    """Simulate the spot masks and their distance map on the GPU and make the map resident.

    Uses the library's device spot simulator (the same point-voxel model as
    ``simulate_mask``) and exact EDT, then ``grc_upload_masks_device``.  Returns the
    host float32 map (nrot, dety, detz) when ``keep_host_map``, else None.
    """
    import torch

    g = sample.geom
    S9, B9, hkl, rot, R9, p = sample.mex_arrays()
    ctx.set_geometry(S9, B9, hkl, rot, R9, p)
    idx = sample.voxel_indices()
    gid = sample.grain_id[idx[:, 0] - 1, idx[:, 1] - 1, idx[:, 2] - 1]
    pos = sample.vol.pos_of_index(idx).astype(np.float32)
    Ug = np.stack([G.flat_rowmajor(G.quat_to_u(q)) for q in sample.grain_q])
    d_U = torch.from_numpy(Ug).cuda()[torch.from_numpy(gid - 1).long().cuda()].reshape(-1).contiguous()
    n = g.nrot * g.detysize * g.detzsize
    d_mask = torch.zeros(n, dtype=torch.uint8, device="cuda")
    ctx.simulate_spots(torch.from_numpy(pos.reshape(-1)).cuda(), d_U, len(idx), d_mask)
    del d_U
    d_map = torch.empty(n, dtype=torch.float32, device="cuda")
    ctx.edt(d_mask, g.detzsize, g.detysize, g.nrot, d_map)
    del d_mask
    ctx.upload_masks(d_map, g.detzsize, g.detysize, g.nrot)
    host = d_map.cpu().numpy().reshape(g.nrot, g.detysize, g.detzsize) if keep_host_map else None
    del d_map
    torch.cuda.empty_cache()
    return host


def _rot_small(rng, n, sigma_deg):
    """n random rotations with Gaussian angle (sigma_deg) about uniformly random axes."""
    ax = rng.normal(size=(n, 3))
    ax /= np.linalg.norm(ax, axis=1, keepdims=True)
    ang = np.radians(rng.normal(0.0, sigma_deg, n))
    K = np.zeros((n, 3, 3))
    K[:, 0, 1], K[:, 0, 2], K[:, 1, 2] = -ax[:, 2], ax[:, 1], -ax[:, 0]
    K[:, 1, 0], K[:, 2, 0], K[:, 2, 1] = ax[:, 2], -ax[:, 1], ax[:, 0]
    s, c = np.sin(ang)[:, None, None], np.cos(ang)[:, None, None]
    return np.eye(3)[None] + s * K + (1 - c) * (K @ K)


def compete_worklist(sample: Sample, seed: int = 0, p: float = 0.15, kmax: int = 64, n_variants: int = 32,
                     sigma_deg: float = 0.5, voxels: np.ndarray | None = None):
    """Uneven candidate lists for the batched grower (cuda_forward_comp_compete layout).

    Every voxel gets k ~ Geometric(p) candidates truncated to [1, kmax]; each candidate is
    the orientation of the voxel's own grain or of a face-neighbour's grain, either exact
    or one of ``n_variants`` copies perturbed by a Gaussian ``sigma_deg`` rotation.
    Returns (rows5 [m x 5: x y z first last], id_neigb [1-based rows of euler], euler
    [n_entries x 3, degrees]) as float32 arrays.
    """
    rng = np.random.default_rng(seed)
    gid = sample.grain_id
    idx = sample.voxel_indices() if voxels is None else np.asarray(voxels, np.int64)
    m = len(idx)
    ng = len(sample.grain_q)
    # Euler table: grain g (1-based), variant v (0 = exact) -> row (g-1)*(n_variants+1)+v
    Ug = np.stack([G.quat_to_u(q) for q in sample.grain_q])
    rows = []
    for g in range(ng):
        R = _rot_small(rng, n_variants, sigma_deg)
        rows.append(np.concatenate([Ug[g][None], R @ Ug[g]], 0))
    Uall = np.concatenate(rows, 0)
    euler = (np.degrees(np.stack([G.u_to_euler(u) for u in Uall])) % 360).astype(np.float32)
    k = np.minimum(rng.geometric(p, m), kmax)
    off = np.concatenate([[0], np.cumsum(k)])
    n = int(off[-1])
    vox_of = np.repeat(np.arange(m), k)
    shifts = np.array([[0, 0, 0], [1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1]])
    sh = shifts[rng.integers(0, len(shifts), n)]
    nb = np.clip(idx[vox_of] - 1 + sh, 0, np.array(gid.shape) - 1)
    g_nb = gid[nb[:, 0], nb[:, 1], nb[:, 2]]
    g_own = gid[idx[vox_of, 0] - 1, idx[vox_of, 1] - 1, idx[vox_of, 2] - 1]
    g = np.where(g_nb > 0, g_nb, g_own).astype(np.int64)
    var = rng.integers(0, n_variants + 1, n)
    id_neigb = ((g - 1) * (n_variants + 1) + var + 1).astype(np.float32)
    rows5 = np.zeros((m, 5), np.float32)
    rows5[:, :3] = idx
    rows5[:, 3] = off[:-1] + 1
    rows5[:, 4] = off[1:]
    return rows5, id_neigb, euler
