"""The allocation-free seeding scan against the regular drop-in entry and the oracle.

grc_forward_comp_noalloc exists for callers that cannot allocate GPU memory while
they score (a MEX shim inside MATLAB's gpuArray memory manager, a framework whose
caching allocator owns the device, a per-seed loop where cudaMalloc would
synchronise the device).  Its scratch is a fixed device array shared by every call,
so calls in a row must each give the regular entry's answer: nothing may leak from
one call into the next, on either kernel it takes.  The buffers below are allocated by the test, not by
the entry point.  This file is collected last on purpose.
"""
import numpy as np
import pytest

from grainrecon_b200 import geometry as G
from grainrecon_b200 import synth
from grainrecon_b200._lib import NOALLOC_MAX_ORIENTATIONS, Context, GrcError, GRC_ECAPACITY, GRC_EINVAL
from oracle import oracle as O

pytestmark = pytest.mark.gpu
MED_RTOL = 1e-6  # dis_median tolerance used by the other parity tests


def test_noalloc_matches_drop_in_entry_twice():
    import torch

    s = synth.make_sample("fe_small", seed=1)
    dmap = synth.distance_map(synth.simulate_mask(s))
    S9, B9, hkl, rot, R9, p = s.mex_arrays()
    idx = s.voxel_indices()
    with Context(0) as ctx:
        cases = []
        # 706 and 1,006 orientations take the per-trial kernel, 4,006 the warp scan (from 1/16 of
        # a round), as the regular entry would
        for k, (v, n) in enumerate(((idx[7], 700), (idx[len(idx) // 2], 1000), (idx[3], 4000))):
            pos = s.vol.pos_of_index(v).astype(np.float32)
            q = np.concatenate([s.grain_q, G.cubic_fz_orientations(n, 40 + k)]).astype(np.float32)
            ref = ctx.forward_comp(pos, q, S9, B9, hkl, dmap if k == 0 else None, rot, R9, p).reshape(-1, 4)
            orc, _, tight = O.orientation_scan(pos, q, S9, B9, hkl, dmap, rot, R9, p, tight=True)
            cases.append((pos, q, ref, orc.reshape(-1, 4), tight == 0))
        # calls in a row, different sizes: none may see an earlier call's leftovers
        for (pos, q, ref, orc, exact), path in zip(cases, (1, 1, 3)):
            d_q = torch.from_numpy(q.reshape(-1)).cuda()
            d_out = torch.full((q.shape[0] * 4,), -7.0, dtype=torch.float32, device="cuda")
            torch.cuda.synchronize()
            ctx.forward_comp_noalloc(pos, d_q, q.shape[0], d_out)
            assert ctx.last_stats()["path"] == path
            got = d_out.cpu().numpy().reshape(-1, 4)
            np.testing.assert_array_equal(got[:, :3], ref[:, :3])
            np.testing.assert_allclose(got[:, 3], ref[:, 3], rtol=MED_RTOL)
            # and the FP64 oracle, on every trial without a reflection within 1e-9 px of a boundary
            assert exact.sum() >= len(q) - 2
            np.testing.assert_array_equal(got[exact, :3], orc[exact, :3])
            np.testing.assert_allclose(got[exact, 3], orc[exact, 3], rtol=MED_RTOL)
        with pytest.raises(GrcError) as e:
            ctx.forward_comp_noalloc(cases[0][0], d_q, NOALLOC_MAX_ORIENTATIONS + 1, d_out)
        assert e.value.code == GRC_ECAPACITY
        # host buffers are refused before any kernel sees them
        host_q = torch.from_numpy(cases[0][1].reshape(-1).copy())
        with pytest.raises(GrcError) as e:
            ctx.forward_comp_noalloc(cases[0][0], host_q, cases[0][1].shape[0], d_out)
        assert e.value.code == GRC_EINVAL
