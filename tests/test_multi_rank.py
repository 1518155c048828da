"""Multi-rank plumbing of bench.py on CPU (gloo, world_size 2): every rank scores its own
disjoint seed shard per step and the job time is the max over ranks."""
import os
import socket

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import sys

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        shards = [bench.seed_range(step, rank, world, 8) for step in range(5)]
        t = bench.max_over_ranks(1.0 + rank)  # rank 1 is the slow one
        out[rank] = (shards, t)
    finally:
        dist.destroy_process_group()


def test_seed_sharding_and_max_time_over_ranks():
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.start_processes(_worker, args=(world, port, out), nprocs=world, start_method="spawn", join=True)
        res = dict(out)
    seen = []
    for rank in range(world):
        shards, t = res[rank]
        assert t == pytest.approx(2.0)  # every rank reports the slowest rank's time
        seen.extend(range(a, z) for a, z in shards)
    rows = [r for rng in seen for r in rng]
    assert len(rows) == len(set(rows)) == world * 5 * 8  # disjoint, complete
    assert sorted(rows) == list(range(world * 5 * 8))


def test_single_process_time_is_identity():
    import sys
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.5) == 3.5
    assert bench.seed_range(2, 0, 1, 64) == (128, 192)


def test_workload_note_says_whether_the_read_array_exceeds_l2():
    """The timing rule for the bench line: inputs larger than L2 between timed steps, or the
    line says they are not.  The Al seeding scan reads a 189 MB hit mask (and 1.51 GB of 8-bit
    codes with the four columns); the Fe mask (24 MB) stays in L2 and the note says so."""
    import sys
    from types import SimpleNamespace as NS

    import numpy as np
    sys.path.insert(0, ROOT)
    import bench

    def sample(nrot, n, sg, ngr, nhkl):
        return NS(geom=NS(nrot=nrot, detysize=n, detzsize=n), space_group=sg, grain_q=[0] * ngr, nhkl=nhkl,
                  grain_id=np.ones(4))

    al = sample(361, 2048, 225, 400, 64)
    fe = sample(181, 1024, 229, 6, 86)
    assert bench.workload_desc(al, 64)["l2"].startswith("inputs larger than L2 (126 MB): the packed hit mask (189 MB")
    assert "(1.51 GB)" in bench.workload_desc(al, 64, "full")["l2"]
    assert "fits in L2" in bench.workload_desc(fe, 64)["l2"]
    assert bench.workload_desc(fe, 64, "full")["l2"].startswith("inputs larger than L2")
    assert bench.workload_desc(al, 64)["trials_per_step_per_gpu"] == 64 * bench.N_ORIENT
