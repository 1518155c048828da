"""Device mask preparation: spot images to the resident map, and the packed spot-mask file.

* grc_upload_spot_masks (binary spot images, the device bwdist) scores exactly as the host
  bwdist map uploaded with grc_upload_masks;
* grc_save_packed_masks writes the documented layout (checked here by decoding the file with
  numpy alone), and grc_load_packed_masks restores a context that scores identically;
* a truncated, lengthened, altered or foreign file, or a header announcing more pixels per
  projection than a map may hold, is refused with GRC_EINVAL before anything is allocated."""
import numpy as np
import pytest

from grainrecon_b200 import geometry as G
from grainrecon_b200 import synth
from grainrecon_b200._lib import Context, GrcError, GRC_EINVAL

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def sample():
    s = synth.make_sample("al_small", seed=3)
    mask = synth.simulate_mask(s, stride=2)
    return s, mask, synth.distance_map(mask)


def _scan(ctx, s, n=800):
    S9, B9, hkl, rot, R9, p = s.mex_arrays()
    ctx.set_geometry(S9, B9, hkl, rot, R9, p)
    idx = s.voxel_indices()
    q = np.concatenate([s.grain_q, G.cubic_fz_orientations(n, 8)]).astype(np.float32)
    outs = [ctx.forward_comp(s.vol.pos_of_index(v).astype(np.float32), q, S9, B9, hkl, None, rot, R9, p)
            for v in idx[[3, len(idx) // 2]]]
    return np.concatenate(outs)


def test_spot_masks_score_as_host_bwdist(sample):
    s, mask, dmap = sample
    g = s.geom
    with Context(0) as a, Context(0) as b:
        a.upload_masks(dmap, g.detzsize, g.detysize, g.nrot)
        b.upload_spot_masks(mask.astype(np.uint8), g.detzsize, g.detysize, g.nrot)
        assert a.mask_info()["n_distinct"] == b.mask_info()["n_distinct"]
        np.testing.assert_array_equal(_scan(a, s), _scan(b, s))


def test_packed_mask_file_round_trip(sample, tmp_path):
    s, mask, dmap = sample
    g = s.geom
    path = str(tmp_path / "al_small.grcmask")
    with Context(0) as a:
        a.upload_masks(dmap, g.detzsize, g.detysize, g.nrot)
        ref = _scan(a, s)
        a.save_packed_masks(path)
    raw = open(path, "rb").read()
    plane = g.detzsize * g.detysize
    pw = (plane + 127) // 128 * 4
    assert raw[:8] == b"GRCMASK1" and len(raw) == 80 + 4 * pw * g.nrot
    hdr = np.frombuffer(raw[8:16], "<u4")
    dims = np.frombuffer(raw[16:48], "<i8")
    assert list(hdr) == [1, 80] and list(dims) == [g.detzsize, g.detysize, g.nrot, pw]
    words = np.frombuffer(raw[80:], "<u4").reshape(g.nrot, pw)
    bits = np.unpackbits(words.view(np.uint8), axis=1, bitorder="little")[:, :plane]
    np.testing.assert_array_equal(bits.reshape(mask.shape).astype(bool), mask)
    with Context(0) as b:
        b.load_packed_masks(path)
        np.testing.assert_array_equal(_scan(b, s), ref)
        big = bytearray(raw[:80])  # a consistent header announcing 10^6 x 10^6 pixels per projection
        big[16:48] = np.array([10**6, 10**6, g.nrot, (10**12 + 127) // 128 * 4], "<i8").tobytes()
        for bad in (raw[:-4], raw + b"\0\0\0\0", raw[:100] + bytes([raw[100] ^ 1]) + raw[101:],
                    b"NOTAMASK" + raw[8:], bytes(big) + raw[80:]):
            p2 = str(tmp_path / "bad.grcmask")
            open(p2, "wb").write(bad)
            with pytest.raises(GrcError) as e:
                b.load_packed_masks(p2)
            assert e.value.code == GRC_EINVAL
        np.testing.assert_array_equal(_scan(b, s), ref)  # a refused file leaves the resident map
