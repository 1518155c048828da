"""The scorer's inputs pinned to the reference's crystallography (CPU).

The oracle and the GPU both consume ``geometry.py``'s reflection list, wavelength window, theta_max
and B matrix, so a mistake there would pass every parity test.  These checks restate the
reference's definitions independently:

* setup_hkl.m:46-60 keeps every allowed reflection whose h^2+k^2+l^2 does not exceed the
  hklnumber-th smallest allowed value, Friedel mates included.  With the lattice-centring rules
  (FCC: h, k, l all odd or all even; BCC: h+k+l even) and six families this is 64 reflections for
  FCC Al and 86 for BCC Fe;
* setup_hkl.m:21-22: lambda_max = 12.39818746/E_min, lambda_min = 12.39818746/E_max, so a
  10-70 keV source gives [0.17712, 1.23982] A;
* setup_hkl.m:17-20: theta_max is half the two-theta of the detector corner, acos of the angle
  between the beam and [Lsam2det, detysize*pixelysize/2, detzsize*pixelzsize/2];
* FormB.m:15-52: B (2*pi convention) with |B h| = 2*pi/d_hkl for any cell, d from the metric
  tensor, and B = 2*pi/a * I for a cubic cell.
"""
import itertools
import math

import numpy as np
import pytest

from grainrecon_b200 import geometry as G
from grainrecon_b200 import synth


def _allowed(space_group, h, k, l):
    if space_group == 225:  # F-centred: unmixed parity
        return len({h % 2, k % 2, l % 2}) == 1
    if space_group == 229:  # I-centred
        return (h + k + l) % 2 == 0
    raise ValueError(space_group)


def _families(space_group, n_families, hmax=8):
    """All allowed (h, k, l) != 0 of the first n_families values of h^2+k^2+l^2."""
    refl = [(h, k, l) for h, k, l in itertools.product(range(-hmax, hmax + 1), repeat=3)
            if (h, k, l) != (0, 0, 0) and _allowed(space_group, h, k, l)]
    sq = sorted({h * h + k * k + l * l for h, k, l in refl})[:n_families]
    return {r for r in refl if r[0] ** 2 + r[1] ** 2 + r[2] ** 2 <= sq[-1]}, sq


@pytest.mark.parametrize("sg,n_expected,squares", [
    (225, 64, [3, 4, 8, 11, 12, 16]),    # {111} {200} {220} {311} {222} {400}: 8+6+12+24+8+6
    (229, 86, [2, 4, 6, 8, 10, 12]),     # {110} {200} {211} {220} {310} {222}: 12+6+24+12+24+8
])
def test_reflection_lists(sg, n_expected, squares):
    got = G.gen_hkl(sg, 6)
    ref, sq = _families(sg, 6)
    assert sq == squares
    assert len(ref) == n_expected
    assert got.shape == (n_expected, 3)
    assert {tuple(int(x) for x in r) for r in got} == ref
    assert {tuple(-int(x) for x in r) for r in got} == ref  # Friedel mates included


def test_benchmark_samples_carry_the_reference_inputs():
    for kind, n_hkl, det, px, nrot in (("fe6", 86, 1024, 0.0672, 181), ("al400", 64, 2048, 0.0336, 361)):
        geom, cell, sg, hkl, *_ = synth.named_setup(kind, seed=1)
        p = geom.param20(len(hkl))
        assert int(p[0]) == n_hkl and int(p[1]) == nrot
        assert int(p[10]) == int(p[11]) == det and p[8] == np.float32(px)
        # lambda window of a 10-70 keV source
        assert p[17] == np.float32(12.39818746 / 70) and p[18] == np.float32(12.39818746 / 10)
        assert abs(float(p[17]) - 0.17712) < 5e-6 and abs(float(p[18]) - 1.23982) < 5e-6
        # theta_max from the detector corner, restated with atan2 instead of acos
        half_diag = math.hypot(0.5 * det * px, 0.5 * det * px)
        tmax = math.degrees(math.atan2(half_diag, geom.lsd)) / 2
        assert abs(float(p[16]) - tmax) < 1e-4
        assert abs(geom.theta_max - tmax) < 1e-10
        # B of a cubic cell
        np.testing.assert_allclose(G.form_b(cell), 2 * math.pi / cell[0] * np.eye(3), atol=1e-14)


@pytest.mark.parametrize("cell", [
    (4.0495, 4.0495, 4.0495, 90, 90, 90),
    (3.1, 4.7, 5.3, 90, 90, 90),
    (5.1, 5.1, 8.2, 90, 90, 120),
    (4.2, 5.3, 6.1, 81.0, 97.0, 104.0),
])
def test_form_b_gives_reciprocal_lengths(cell):
    """|B h| = 2 pi / d_hkl with d from the direct metric tensor; B upper triangular (FormB.m)."""
    a, b, c = cell[:3]
    al, be, ga = (math.radians(x) for x in cell[3:])
    Gm = np.array([[a * a, a * b * math.cos(ga), a * c * math.cos(be)],
                   [a * b * math.cos(ga), b * b, b * c * math.cos(al)],
                   [a * c * math.cos(be), b * c * math.cos(al), c * c]])
    Ginv = np.linalg.inv(Gm)
    B = G.form_b(cell)
    assert np.allclose(np.tril(B, -1), 0)
    for h in itertools.product(range(-3, 4), repeat=3):
        if h == (0, 0, 0):
            continue
        h = np.array(h, float)
        d = 1.0 / math.sqrt(h @ Ginv @ h)
        assert abs(np.linalg.norm(B @ h) - 2 * math.pi / d) < 1e-12 * (2 * math.pi / d)
