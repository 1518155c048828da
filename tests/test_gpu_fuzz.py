"""Seeded random geometries against the FP64 oracle, on every kernel and both output modes.

Each case draws a geometry the benchmark samples never reach: a non-square detector with
offsets, tilts up to 8 degrees, a beam stop, a rotation-axis offset, non-uniform projection
angles, an energy window, and a reflection list of 12 to 128 rows (one to four reflection slots
per lane in the window kernels); six more push to 1-2 reflections, 1-12 projections, 20-degree
tilts and a beam stop over the detector centre.  Odd seeds use a distance map with a few
distinct values (8-bit codes), even seeds one with millions (32-bit codes and the radix refine
of the median).  On the per-trial kernel, the CTA sweep and the warp scan, with and without the median,
every trial without a tight edge reflection equals the oracle in every column it returns.  Seven of
the geometries also run the grow and compete entries against the oracle's grow and compete, and
six run the spot pairing against the oracle's forward_comp_pair_spots."""
import numpy as np
import pytest

from grainrecon_b200 import geometry as G
from grainrecon_b200._lib import Context
from oracle import oracle as O

pytestmark = pytest.mark.gpu

CASES = [(101, 12, False), (102, 40, False), (103, 64, False), (104, 100, False), (105, 128, False),
         (106, 27, False), (107, 90, False), (108, 128, False),
         # extremes: 1-2 reflections, few projections, 20-degree tilts, a centred beam stop
         (115, 1, True), (110, 2, True), (111, 33, True), (112, 65, True), (113, 97, True), (114, 128, True)]


def _case(seed, nhkl, extreme=False):
    rng = np.random.default_rng(seed)
    sg, cell = (229, (2.8665,) * 3 + (90,) * 3) if seed % 2 else (225, (4.0495,) * 3 + (90,) * 3)
    hkl = G.gen_hkl(sg, 40, hmax=8)[:nhkl].astype(np.float64)
    assert len(hkl) == nhkl
    nrot = int(rng.integers(1, 13)) if extreme else int(rng.integers(37, 182))
    rot = np.sort(rng.uniform(0.0, 360.0, nrot))
    dety, detz = (int(x) for x in rng.integers(200, 641, 2))
    px = float(rng.uniform(0.05, 0.15))
    if extreme:  # a beam stop around the detector centre, 10-30 % of each side
        hy, hz = dety * rng.uniform(0.05, 0.15), detz * rng.uniform(0.05, 0.15)
        by, bz = (dety / 2 - hy, dety / 2 + hy), (detz / 2 - hz, detz / 2 + hz)
    else:
        by = sorted(rng.uniform(0, dety, 2)) if rng.random() < 0.7 else (0.0, 0.0)
        bz = sorted(rng.uniform(0, detz, 2)) if rng.random() < 0.7 else (0.0, 0.0)
    tilt = 20.0 if extreme else 8.0
    geom = G.Geometry(lss=float(rng.uniform(8, 14)), lsd=float(rng.uniform(6, 14)),
                      p0y=float(rng.uniform(-0.05, 0.05)), p0z=float(rng.uniform(-0.05, 0.05)),
                      dety00=float(rng.uniform(-1, 1)), detz00=float(rng.uniform(-1, 1)),
                      pxy=px, pxz=px * float(rng.uniform(0.8, 1.25)), detysize=dety, detzsize=detz,
                      beamstop_y=tuple(by), beamstop_z=tuple(bz), tilt=tuple(rng.uniform(-tilt, tilt, 3)),
                      rot_axis_offset=float(rng.uniform(-0.1, 0.1) if extreme else rng.uniform(-0.03, 0.03)),
                      e_min_kev=float(rng.uniform(8, 20)), e_max_kev=float(rng.uniform(40, 90)),
                      rot_angles=rot)
    shape = (nrot, dety, detz)
    if seed % 2:  # a few distinct values: 8-bit codes, medians from the histogram
        levels = np.array([0.0, 1.0, 1.4142135, 2.0, 2.236068, 3.0, 5.0, 8.0], np.float32)
        dmap = levels[rng.choice(len(levels), size=shape, p=[0.15, 0.2, 0.15, 0.15, 0.1, 0.1, 0.1, 0.05])]
    else:  # thousands of distinct values: 16-bit codes, medians from the radix refine
        dmap = (1.0 + rng.random(shape, dtype=np.float32) * 300.0).astype(np.float32)
        dmap[rng.random(shape) < 0.12] = 0.0
    B = G.form_b(cell)
    S = G.flat_rowmajor(np.eye(3))
    args = (S, G.flat_rowmajor(B), G.flat_hkl(hkl), np.asarray(rot, np.float32), G.flat_rowmajor(geom.rot_det),
            geom.param20(nhkl))
    pos = rng.uniform(-0.15, 0.15, (2, 3)).astype(np.float32)
    q = G.cubic_fz_orientations(1500, seed).astype(np.float32)
    return geom, dmap, args, pos, q


@pytest.mark.parametrize("seed,nhkl,extreme", CASES)
def test_random_geometry_matches_oracle(seed, nhkl, extreme):
    geom, dmap, (S9, B9, hk, rot, R9, p), pos, q = _case(seed, nhkl, extreme)
    with Context(0) as ctx:
        ctx.set_geometry(S9, B9, hk, rot, R9, p)
        ctx.upload_masks(dmap, geom.detzsize, geom.detysize, geom.nrot)
        for v in range(len(pos)):
            ref, _, tight = O.orientation_scan(pos[v], q, S9, B9, hk, dmap, rot, R9, p, tight=True)
            ref = ref.reshape(-1, 4)
            ok = tight == 0
            assert ok.sum() >= len(q) - 15
            # the geometry lands reflections on the detector
            assert (ref[:, 0] > 0).sum() > (len(q) // 50 if extreme else len(q) // 4)
            for path in (1, 2, 3):
                ctx.set_path(path)
                for median in (True, False):
                    ctx.set_median(median)
                    gpu = ctx.forward_comp(pos[v], q, S9, B9, hk, None, rot, R9, p).reshape(-1, 4)
                    assert ctx.last_stats()["path"] == path
                    cols = 4 if median else 3
                    np.testing.assert_array_equal(gpu[ok, :cols], ref[ok, :cols],
                                                  err_msg=f"seed {seed} voxel {v} path {path} median {median}")
                    if not median:
                        assert np.isnan(gpu[:, 3]).all()
        ctx.set_path(0)
        ctx.set_median(True)


def _volume_param1(rng, simap, dim=60):
    """param1[:11] of a dim^3 volume of 5 um voxels around a random centre (the positions span
    about +-0.15 mm, like the seed positions above); simap 1 flips x and y."""
    centre = rng.uniform(-0.02, 0.02, 3)
    return np.array([1, 1, 1, simap, 0.005, *centre, dim, dim, dim, 0, 0, 0], np.float32), dim


@pytest.mark.parametrize("seed,nhkl,extreme", [CASES[i] for i in (0, 1, 4, 5, 8, 9, 12)])
def test_random_geometry_grow_and_compete_match_oracle(seed, nhkl, extreme):
    """cuda_grow_indexed_region and cuda_forward_comp_compete on the same random geometries, on
    every kernel: trials without a tight edge reflection equal the oracle in every column
    (dis_median to float32 rounding, as in the fixed-geometry parity tests)."""
    geom, dmap, (S9, B9, hk, rot, R9, p), _, q = _case(seed, nhkl, extreme)
    rng = np.random.default_rng(seed + 1000)
    p1, dim = _volume_param1(rng, seed % 2)
    m = 256
    idx = rng.integers(1, dim + 1, (m, 3)).astype(np.float32)
    # grow rows [x y z I mask dmed]; about 0.12-0.15 of the random map's pixels are hits
    rows6 = np.zeros((m, 6), np.float32)
    rows6[:, :3] = idx
    rows6[:, 3] = rng.uniform(0, 0.3, m)
    rows6[:, 4] = rng.random(m) > 0.2
    rows6[:, 5] = rng.uniform(0, 10, m)
    p1g = p1.copy()
    p1g[11:14] = (0.15, 0.1, 6.0)  # flag: C >= 0.135, about the random map's hit fraction
    U = G.flat_rowmajor(G.quat_to_u(q[0]))
    g_ref, _, g_tight = O.grow(rows6, U, S9, B9, hk, dmap, rot, R9, p, p1g, tight=True)
    g_ref = g_ref.reshape(-1, 7)
    g_ok = g_tight == 0
    assert g_ok.sum() >= m - 8
    # compete: 1-16 candidates per voxel among 40 orientations, one voxel without any
    ng = 40
    eul = (np.degrees([G.u_to_euler(G.quat_to_u(x)) for x in q[:ng]]) % 360).astype(np.float32)
    counts = np.minimum(rng.geometric(0.3, m), 16)
    counts[7] = 0
    ids, rows5 = [], np.zeros((m, 5), np.float32)
    rows5[:, :3] = idx
    for i, c in enumerate(counts):
        rows5[i, 3] = len(ids) + 1
        ids.extend(rng.integers(1, ng + 1, c).tolist())
        rows5[i, 4] = len(ids)
    ids = np.array(ids, np.float32)
    c_ref, _, c_tight = O.compete(rows5, ids, eul, S9, B9, hk, dmap, rot, R9, p, p1, tight=True)
    c_ref = c_ref.reshape(-1, 8)
    c_ok = c_tight == 0
    assert c_ok.sum() >= m - 16
    with Context(0) as ctx:
        ctx.set_geometry(S9, B9, hk, rot, R9, p)
        ctx.upload_masks(dmap, geom.detzsize, geom.detysize, geom.nrot)
        for path in (1, 2, 3):
            ctx.set_path(path)
            msg = f"seed {seed} path {path}"
            gg = ctx.grow_indexed_region(rows6, U, S9, B9, hk, None, rot, R9, p, p1g).reshape(-1, 7)
            assert ctx.last_stats()["path"] == path
            np.testing.assert_array_equal(gg[g_ok][:, [0, 1, 2, 3, 4, 6]], g_ref[g_ok][:, [0, 1, 2, 3, 4, 6]],
                                          err_msg=msg + " grow")
            np.testing.assert_allclose(gg[g_ok, 5], g_ref[g_ok, 5], rtol=1e-6, err_msg=msg + " grow median")
            gc = ctx.forward_comp_compete(rows5, ids, eul, S9, B9, hk, None, rot, R9, p, p1).reshape(-1, 8)
            assert ctx.last_stats()["path"] == path
            np.testing.assert_array_equal(gc[c_ok][:, :7], c_ref[c_ok][:, :7], err_msg=msg + " compete")
            np.testing.assert_allclose(gc[c_ok, 7], c_ref[c_ok, 7], rtol=1e-6, err_msg=msg + " compete median")
            assert gc[7, 4] == 0 and gc[7, 7] == 2000
        ctx.set_path(0)


def _pairing_spots(rng, geom, trials, S9, B9, hk, dmap, rot, R9, p):
    """Measured spots of a random geometry: the landings of the given (U, pos) trials with 0.4 px
    centroid noise and random areas, plus 10 spurious spots per projection."""
    per = [[] for _ in range(geom.nrot)]
    for U, pos in trials:
        rec, _ = O.landings(U, pos, S9, B9, hk, dmap, rot, R9, p)
        for j in np.nonzero(rec["sel"])[0]:
            per[rec["iw"][j]].append((rec["u"][j] + rng.normal(0, 0.4), rec["v"][j] + rng.normal(0, 0.4),
                                      rng.uniform(4, 40)))
    for iw in range(geom.nrot):
        for _ in range(10):
            per[iw].append((rng.uniform(1, geom.detysize), rng.uniform(1, geom.detzsize), 10.0))
    return [np.array(a, np.float64).reshape(-1, 3) for a in per]


@pytest.mark.parametrize("seed,nhkl,extreme", [CASES[i] for i in (0, 1, 4, 5, 10, 12)])
def test_random_geometry_pairing_matches_oracle(seed, nhkl, extreme):
    """grc_pair_spots on random geometries against the oracle's forward_comp_pair_spots.m: six
    trials, three of them with their own noisy spots in the list; every trial whose hits carry
    no edge reflection has the oracle's pair list (projection, reflection, spot, pixel, centroid,
    area and distance exact, energy to 1e-12)."""
    from grainrecon_b200 import seeding as S
    from oracle import seed_oracle as SO
    geom, dmap, (S9, B9, hk, rot, R9, p), pos, q = _case(seed, nhkl, extreme)
    rng = np.random.default_rng(seed + 2000)
    tp = pos[[0, 1, 0, 1, 0, 1]].astype(np.float64)
    tq = q[:6].astype(np.float64)
    Us = [G.quat_to_u(x) for x in tq]
    spots = _pairing_spots(rng, geom, [(Us[t], tp[t]) for t in range(3)], S9, B9, hk, dmap, rot, R9, p)
    off = np.concatenate([[0], np.cumsum([len(a) for a in spots])])
    sc = SO.Scene(S9, B9, hk, rot, R9, p, dmap)
    with Context(0) as ctx:
        ctx.set_geometry(S9, B9, hk, rot, R9, p)
        ctx.upload_masks(dmap, geom.detzsize, geom.detysize, geom.nrot)
        pairs = S.pair_spots(ctx, tp, tq, spots, geom.nrot)
    n_clean = n_pairs = 0
    for t in range(len(tp)):
        ref, edges = SO.pair_spots(sc, Us[t], tp[t], spots)
        if edges:
            continue
        n_clean += 1
        got = pairs[pairs["trial"] == t]
        assert len(got) == len(ref), (seed, t, len(got), len(ref))
        n_pairs += len(ref)
        for a, r in zip(got, ref):
            iw, ih, j, dety, detz, ey, ez, area, ekev, dis = r
            assert (a["iw"], a["ih"], a["spot"]) == (iw, ih, off[iw] + j)
            assert (a["dety"], a["detz"], a["exp_y"], a["exp_z"], a["area"]) == (dety, detz, ey, ez, area)
            assert a["dis"] == np.float32(dis)
            np.testing.assert_allclose(a["energy_kev"], ekev, rtol=1e-12)
    assert n_clean >= 4 and n_pairs > 0
