"""The two routes that synthesise benchmark inputs agree.

The GPU benchmark arm builds its sample with torch (grain ids of grids of 64^3 and more) and its
spot masks and distance map with the library's device kernels; the CPU reference arm builds the
same inputs on the host cores (oracle/grc_synth_host.c).  Both arms must time the same workload,
so the grain ids, masks and maps must be the same."""
import numpy as np
import pytest

from grainrecon_b200 import synth
from grainrecon_b200._lib import Context
from oracle import host_synth as H

pytestmark = pytest.mark.gpu


def test_fe6_map_host_equals_device():
    s = synth.make_sample("fe6", seed=1)
    sh = H.make_sample_host("fe6", seed=1)
    assert np.array_equal(s.grain_id, sh.grain_id)
    with Context(0) as ctx:
        dev = synth.device_maps(s, ctx, keep_host_map=True)
    host = H.distance_map_host(sh)
    assert dev.shape == host.shape
    assert np.array_equal(dev, host)


def test_al400_grain_ids_host_equal_torch():
    dim, ng, sigma = 160, 400, 0.4
    g_torch = synth.voronoi_cylinder_torch(dim, ng, 1, sigma).cpu().numpy()
    g_host = H.power_voronoi(dim, ng, 1, sigma)
    assert np.array_equal(g_torch, g_host)
