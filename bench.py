#!/usr/bin/env python
"""Benchmark of the completeness scorer on its production seeding workload.

Workload (default ``--config al400``): the seeding stage of the plain GPU scorer --
FCC Al (a = 4.0495 A, 6 families = 64 reflections), 400 grains with log-normal
sizes in a 400 um x 400 um cylinder at 2.5 um (~3.2M voxels), 361 projections,
2048 x 2048 detector at 0.0336 mm, every seed voxel scored against a 32,768-
orientation cubic grid.  Seeded synthetic inputs stand in for the reference's
data (spot masks forward-simulated from the ground truth, distance map = exact
EDT); the orientation set is a seeded uniform sample of the cubic fundamental
zone with the Oh 2-degree grid's size.

A step = ``--seeds`` seed voxels x 32,768 orientations per GPU (weak scaling: each
rank scores its own seeds, no data-path collective).  ``value`` is device-resident
trials/s (CUDA events on the library's stream, max over ranks); ``e2e`` calls the
drop-in C-ABI entry ``grc_forward_comp`` once per seed voxel with pinned host
buffers, copies included.  ``--impl reference`` times the FP64 CPU oracle (the
restated reference CPU scorer) on the host cores on a bounded sample.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "voxel·orientation trials/s"
N_ORIENT = 32768
N_SEEDS = 20000


def seed_range(step: int, rank: int, world: int, per_rank: int):
    """Seed rows [start, stop) that ``rank`` scores in ``step`` (weak scaling, disjoint shards)."""
    base = (step * world + rank) * per_rank
    return base, base + per_rank


def max_over_ranks(seconds: float, device=None) -> float:
    """Max of a per-rank time over all ranks (the job's time); identity without a process group."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(seconds)
    t = torch.tensor([seconds], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def env_rank():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled every 200 ms while running."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if len(r) > 5 + i and r[5 + i] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def build_problem(config: str, seed: int, sample=None):
    from grainrecon_b200 import geometry as G
    from grainrecon_b200 import synth
    s = sample if sample is not None else synth.make_sample(config, seed=seed)
    idx = s.voxel_indices()
    rng = np.random.default_rng(seed + 99)
    seeds = idx[rng.choice(len(idx), min(N_SEEDS, len(idx)), replace=False)]
    pos = s.vol.pos_of_index(seeds).astype(np.float32)
    q = G.cubic_fz_orientations(N_ORIENT, seed + 5).astype(np.float32)
    return s, pos, q


def workload_desc(s, seeds_per_step, output="completeness"):
    g = s.geom
    npx = g.nrot * g.detysize * g.detzsize
    read = (f"the packed hit mask ({npx / 8 / 1e6:.0f} MB, one bit per pixel)" if output == "completeness"
            else f"the distance map as 8-bit rank codes ({npx / 1e9:.2f} GB)")
    big = (npx / 8 if output == "completeness" else npx) > 126e6
    return {"workload": (f"seeding scan: {'FCC Al' if s.space_group == 225 else 'BCC Fe'} "
                         f"{len(s.grain_q)} grains, {int((s.grain_id > 0).sum())} voxels, "
                         f"{g.detysize}x{g.detzsize} detector, {g.nrot} projections, {s.nhkl} reflections; "
                         f"{seeds_per_step} seed voxels x {N_ORIENT} orientations per step per GPU"),
            "trials_per_step_per_gpu": seeds_per_step * N_ORIENT,
            "reflections_per_trial": g.nrot * s.nhkl,
            "l2": (f"inputs larger than L2 (126 MB): {read} is read by every step" if big else
                   f"{read} fits in L2 (126 MB) and stays resident across steps (no flush)"),
            "parallelism": "replicas: seeds sharded across ranks, no collective on the data path"}


def cpu_baseline(s, host_map, pos, q, n_trials):
    """The FP64 oracle on all host cores (OpenMP) and on one thread, on a bounded sample."""
    from oracle import oracle as O
    S9, B9, hkl, rot, R9, p = s.mex_arrays()
    t0 = time.perf_counter()
    O.orientation_scan(pos[0], q[:n_trials], S9, B9, hkl, host_map, rot, R9, p)
    dt = time.perf_counter() - t0
    n1 = max(64, n_trials // 16)
    t0 = time.perf_counter()
    O.orientation_scan(pos[1], q[:n1], S9, B9, hkl, host_map, rot, R9, p, nthreads=1)
    dt1 = time.perf_counter() - t0
    return {"value": n_trials / dt, "unit": "trials/s", "cores": O.max_threads(), "kind": "port",
            "sample": f"1 seed voxel x {n_trials} orientations of the same workload (FP64 oracle, OpenMP)",
            "seconds": dt,
            "one_thread": {"value": n1 / dt1, "unit": "trials/s", "cores": 1,
                           "sample": f"1 seed voxel x {n1} orientations on one thread"}}


def run_reference(args):
    """The FP64 CPU oracle (the restated reference scorer) on the host cores.  Nothing here touches
    a GPU or the product library: the sample's grain ids, its spot masks (every voxel with its
    grain's orientation) and their distance map are built on the host by the oracle's C helpers
    (oracle/grc_synth_host.c), from the same seeds as the GPU arm's device synthesis."""
    rank, world, local = env_rank()
    if rank != 0:
        return 0
    from oracle import host_synth as H
    from oracle import oracle as O
    t0 = time.perf_counter()
    sample = H.make_sample_host(args.config, args.seed)
    s, pos, q = build_problem(args.config, args.seed, sample)
    host_map = H.distance_map_host(s)
    setup_s = time.perf_counter() - t0
    S9, B9, hkl, rot, R9, p = s.mex_arrays()
    n = args.ref_trials
    for i in range(args.warmup):
        O.orientation_scan(pos[i % len(pos)], q[:n], S9, B9, hkl, host_map, rot, R9, p)
    t0 = time.perf_counter()
    for i in range(args.steps):
        O.orientation_scan(pos[(args.warmup + i) % len(pos)], q[i * n % N_ORIENT:][:n], S9, B9, hkl, host_map, rot,
                           R9, p)
    dt = time.perf_counter() - t0
    val = args.steps * n / dt
    n1 = max(64, n // 16)
    t1 = time.perf_counter()
    O.orientation_scan(pos[0], q[:n1], S9, B9, hkl, host_map, rot, R9, p, nthreads=1)
    dt1 = time.perf_counter() - t1
    cfg = workload_desc(s, args.seeds)
    cfg["l2"] = "host memory: the FP64 oracle reads the float32 distance map"
    line = {"impl": "reference", "metric": METRIC, "value": val, "unit": "trials/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": cfg,
            "cpu_baseline": {"value": val, "unit": "trials/s", "cores": O.max_threads(), "kind": "port",
                             "sample": f"each step: 1 seed voxel x {n} orientations of the same workload",
                             "one_thread": {"value": n1 / dt1, "unit": "trials/s", "cores": 1,
                                            "sample": f"1 seed voxel x {n1} orientations on one thread"}},
            "e2e": {"value": val, "unit": "trials/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "setup_s": setup_s,
            "setup": "sample, spot masks and distance map synthesised on the host cores (no GPU)"}
    print(json.dumps(line), flush=True)
    return 0


SCORER_DTYPE = "f32+f64"  # FP32 landing chain, FP64 for every landing within 0.006 px of a pixel edge


def run_ours(args):
    import torch
    import torch.distributed as dist
    from grainrecon_b200 import synth
    from grainrecon_b200._lib import Context

    rank, world, local = env_rank()
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    s, pos, q = build_problem(args.config, args.seed)
    ctx = Context(local)
    want_cpu = rank == 0 and world == 1 and not args.no_cpu_baseline and not args.profile
    t0 = time.perf_counter()
    host_map = synth.device_maps(s, ctx, keep_host_map=want_cpu)
    setup_s = time.perf_counter() - t0
    S9, B9, hkl, rot, R9, p = s.mex_arrays()
    ctx.set_geometry(S9, B9, hkl, rot, R9, p)
    comp = args.output == "completeness"
    ctx.set_median(not comp)
    ctx.set_path(args.path)
    S = args.seeds
    K, W = args.steps, args.warmup
    need = (K + W) * S * world
    seeds = np.resize(pos, (max(need, len(pos)), 3))
    d_pos = torch.from_numpy(seeds.reshape(-1).copy()).cuda()
    d_q = torch.from_numpy(q.reshape(-1)).cuda()
    d_out = torch.empty((K, S * N_ORIENT * 4), dtype=torch.float32, device="cuda")
    d_best = torch.empty((K, S), dtype=torch.int32, device="cuda")
    d_best_c = torch.empty((K, S), dtype=torch.float32, device="cuda")
    d_tmp = torch.empty(S * N_ORIENT * 4, dtype=torch.float32, device="cuda")
    d_tb = torch.empty(S, dtype=torch.int32, device="cuda")
    d_tc = torch.empty(S, dtype=torch.float32, device="cuda")
    stream = torch.cuda.ExternalStream(ctx.stream)

    def seed_slice(step):
        a, z = seed_range(step, rank, world, S)
        return d_pos[3 * a: 3 * z]

    # one step: the seeding scan of S seeds x N_ORIENT orientations and each seed's first maximum
    ctx.set_timing(True)
    for i in range(W):
        ctx.forward_comp_argmax_device(seed_slice(i), S, d_q, N_ORIENT, d_tmp, d_tb, d_tc)
        ctx.last_stats()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    score_ms = []
    launches = 0
    path = 0
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        ev0.record(stream)
        for i in range(K):
            ctx.forward_comp_argmax_device(seed_slice(W + i), S, d_q, N_ORIENT, d_out[i], d_best[i], d_best_c[i])
            st = ctx.last_stats()  # reads the scoring kernels' CUDA events of this step
            score_ms.append(st["score_ms"])
            launches += st["kernel_launches"]
            path = st["path"]
        ev1.record(stream)
        torch.cuda.synchronize()
    total_ms = ev0.elapsed_time(ev1)
    if args.profile:
        # selected reflections (map lookups) per trial of the profiled steps: turns an ncu
        # capture's DRAM bytes per launch into bytes per lookup
        simu = d_out.view(K, -1, 4)[:, :, 0].double()
        print(json.dumps({"profile": args.config, "output": args.output, "lookups_per_trial": float(simu.mean()),
                          "trials_per_step": S * N_ORIENT, "kernel_launches": launches}), flush=True)
        ctx.close()
        return 0
    max_ms = max_over_ranks(total_ms, device="cuda")
    trials = K * S * N_ORIENT * world
    value = trials / (max_ms / 1e3)
    lookups = d_out.view(K, -1, 4)[:, :, 0].double().sum(dim=1).cpu().numpy()  # selected reflections per launch
    achieved = float(np.mean(lookups * 32.0 / (np.array(score_ms) / 1e3))) / 1e9
    # the first maximum of each seed against the step's own completeness column
    c = d_out.view(K, S, N_ORIENT, 4)[..., 2].cpu().numpy()
    cm = np.where(np.isnan(c), -np.inf, c)
    argmax_ok = bool(np.array_equal(cm.argmax(axis=2), d_best.cpu().numpy()))

    # the other output mode on the same steps (device-resident), for comparison
    ctx.set_median(comp)
    for i in range(2):
        ctx.forward_comp_argmax_device(seed_slice(i), S, d_q, N_ORIENT, d_tmp, d_tb, d_tc)
    torch.cuda.synchronize()
    ev0.record(stream)
    n_other = max(1, min(K, 5))
    for i in range(n_other):
        ctx.forward_comp_argmax_device(seed_slice(W + i), S, d_q, N_ORIENT, d_tmp, d_tb, d_tc)
    ev1.record(stream)
    torch.cuda.synchronize()
    other_val = n_other * S * N_ORIENT * world / (max_over_ranks(ev0.elapsed_time(ev1), device="cuda") / 1e3)
    ctx.set_median(not comp)

    # end to end through the drop-in entry, one call per seed voxel, pinned host buffers
    q_host = torch.from_numpy(q.reshape(-1)).pin_memory().numpy()
    out_host = torch.empty(N_ORIENT * 4, dtype=torch.float32).pin_memory().numpy()
    pos_host = torch.from_numpy(seeds.reshape(-1, 3).copy()).pin_memory().numpy()
    ctx.set_timing(False)
    e2e_steps = max(1, min(K, args.e2e_steps))
    for i in range(1):
        ctx.forward_comp(pos_host[0], q_host, S9, B9, hkl, None, rot, R9, p, out=out_host)
    if world > 1:
        dist.barrier()
    t0 = time.perf_counter()
    for i in range(e2e_steps):
        a, z = seed_range(W + i, rank, world, S)
        for j in range(a, z):
            ctx.forward_comp(pos_host[j], q_host, S9, B9, hkl, None, rot, R9, p, out=out_host)
    e2e_s = max_over_ranks(time.perf_counter() - t0, device="cuda")
    e2e_val = e2e_steps * S * N_ORIENT * world / e2e_s

    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except OSError:
        pass
    peak = peaks.get("hbm_gbs")
    peak_note = "measured hbm_gbs (MEASURED_PEAKS.json)" if peak else "fallback 6650 GB/s"
    peak = peak or 6650.0
    kernel = "sweep_kernel" if path == 2 else ("scan_kernel" if path == 3 else "score_kernel")
    traffic = None
    issue = None
    clocks = clk.summary()
    try:
        # DRAM bytes per selected reflection and warp instructions per trial measured by ncu on
        # the same kernel, workload and output mode (profiles/); absent for one not captured
        prof = json.load(open(os.path.join(ROOT, "profiles", f"{kernel}_dram.json")))["workloads"][
            f"{args.config}-{args.output}"]
        traffic = float(np.mean(lookups)) * prof["dram_bytes_per_lookup"]
        if "warp_instructions_per_trial" in prof:
            # issue roofline: one warp instruction per scheduler per clock, 4 schedulers per SM
            sm_mhz = clocks.get("sm_mhz") or 1965.0
            nsm = torch.cuda.get_device_properties(local).multi_processor_count
            peak_issue = nsm * 4 * sm_mhz * 1e6
            ach_issue = value / world * prof["warp_instructions_per_trial"]
            issue = {"achieved": ach_issue, "peak": peak_issue, "unit": "warp instructions/s",
                     "frac": ach_issue / peak_issue, "instructions_per_trial": prof["warp_instructions_per_trial"],
                     "peak_source": f"{nsm} SMs x 4 schedulers x {sm_mhz:.0f} MHz (sampled under load)",
                     "instructions_source": f"stored ncu capture profiles/{kernel}_dram.json"}
    except (OSError, KeyError, ValueError):
        pass
    cpu = None
    if want_cpu:
        torch.cuda.synchronize()
        cpu = cpu_baseline(s, host_map, seeds, q, args.cpu_trials)
    if rank == 0:
        cfg = workload_desc(s, S, args.output)
        cfg["output"] = (("completeness only: Nr_simu, Nr_intersect and completeness from the bit-packed hit "
                          "mask (column 4 NaN), and each seed's first maximum over its orientations; the "
                          "seeding engine reads column 3 only (GrainMapping_engine_gpu_comp.m:103)") if comp else
                         "the reference's four columns (exact dis_median from the 8-bit rank codes) and each "
                         "seed's first maximum over its orientations")
        line = {"metric": METRIC, "value": value, "unit": "trials/s", "n_gpus": world, "steps": K, "warmup": W,
                "ms_per_step": max_ms / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": SCORER_DTYPE, "data": "synthetic", "config": cfg,
                "clocks": clocks,
                "e2e": {"value": e2e_val, "unit": "trials/s",
                        "h2d_bytes_per_step": S * (12 + N_ORIENT * 16), "d2h_bytes_per_step": S * N_ORIENT * 16,
                        "note": (f"{e2e_steps} steps of {S} grc_forward_comp calls (one per seed voxel), "
                                 f"median {'off (grc_set_median(ctx, 0))' if comp else 'on'}")},
                "gpu_launches": launches,
                "argmax_matches_output": argmax_ok,
                ("full_output" if comp else "completeness_only"): {
                    "value": other_val, "unit": "trials/s", "steps": n_other,
                    "note": "the same steps in the other output mode, device-resident"},
                "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                             "frac": achieved / peak, "traffic": traffic,
                             "traffic_source": "stored ncu capture (profiles/), DRAM bytes per lookup x lookups",
                             "kernel": kernel, "peak_source": peak_note,
                             "algorithmic_bytes": "32 B (one sector) per selected reflection's map lookup",
                             "lookups_per_launch": float(np.mean(lookups)),
                             "score_ms_per_launch": float(np.mean(score_ms)),
                             "issue": issue},
                "cpu_baseline": cpu, "setup_s": setup_s}
        print(json.dumps(line), flush=True)
    ctx.close()
    if world > 1:
        dist.destroy_process_group()
    return 0


def run_grow(args):
    """Batched grower (uneven candidate sets) against one scorer call per voxel."""
    import torch
    from grainrecon_b200 import synth
    from grainrecon_b200._lib import Context

    rank, world, local = env_rank()
    torch.cuda.set_device(local)
    s = synth.make_sample("al400", seed=args.seed)
    ctx = Context(local)
    synth.device_maps(s, ctx)
    idx = s.voxel_indices()
    rng = np.random.default_rng(args.seed + 7)
    vox = idx[np.sort(rng.choice(len(idx), min(args.grow_voxels, len(idx)), replace=False))]
    rows5, ids, eul = synth.compete_worklist(s, seed=args.seed, voxels=vox)
    m = len(rows5)
    d_rows5 = torch.from_numpy(rows5.reshape(-1).copy()).cuda()
    d_ids = torch.from_numpy(ids).cuda()
    d_eul = torch.from_numpy(eul.reshape(-1).copy()).cuda()
    param1 = s.vol.param14(0, 0, 0)[:11]
    out = torch.empty(8 * m, dtype=torch.float32, device="cuda")
    b = ctx.batch(d_rows5, m, d_ids, ids.size, d_eul, len(eul), param1)
    T = b.info()["trials"]
    tune = b.autotune(out, max_voxels=min(m, 30000))
    stream = torch.cuda.ExternalStream(ctx.stream)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    # plain launches of the planned batch (no graph)
    for _ in range(args.warmup):
        b.run(out)
    ctx.sync()
    ev0.record(stream)
    for _ in range(args.steps):
        b.run(out)
    ev1.record(stream)
    ctx.sync()
    direct_ms = ev0.elapsed_time(ev1) / args.steps
    # the same iteration replayed from a CUDA graph
    b.capture(out)
    for _ in range(args.warmup):
        b.replay()
    ctx.sync()
    with ClockSampler(local) as clk:
        ev0.record(stream)
        for _ in range(args.steps):
            b.replay()
        ev1.record(stream)
        ctx.sync()
    graph_ms = ev0.elapsed_time(ev1) / args.steps
    batched = T / (graph_ms / 1e3)
    # the reference's own batching of this work: one compete call per 30,000 waiting voxels
    # (revise_all_unindexed_voxel_cuda.m:77), each call planning its CSR list and copying nothing
    # else (the device-buffer entry grc_compete_device, timed with CUDA events)
    chunk = 30000
    for _ in range(max(1, args.warmup)):
        for c0 in range(0, m, chunk):
            c1 = min(m, c0 + chunk)
            ctx.compete_device(d_rows5[5 * c0:5 * c1], c1 - c0, d_ids, ids.size, d_eul, len(eul), param1,
                               out[8 * c0:8 * c1])
    ctx.sync()
    ev0.record(stream)
    for _ in range(args.steps):
        for c0 in range(0, m, chunk):
            c1 = min(m, c0 + chunk)
            ctx.compete_device(d_rows5[5 * c0:5 * c1], c1 - c0, d_ids, ids.size, d_eul, len(eul), param1,
                               out[8 * c0:8 * c1])
    ev1.record(stream)
    ctx.sync()
    chunked_ms = ev0.elapsed_time(ev1) / args.steps
    # the same chunks through the MEX-shaped host entry (cuda_forward_comp_compete): host rows, the
    # full neighbour and Euler arrays and the geometry every call, host output; the resident map
    # stands for the shim's content-keyed upload.  Wall clock, copies included.
    S9, B9, hkl, rot, R9, p = s.mex_arrays()
    rows5_h = np.ascontiguousarray(rows5, np.float32)
    ids_h = np.ascontiguousarray(ids, np.float32)
    eul_h = np.ascontiguousarray(eul, np.float32).reshape(-1)
    out_h = np.empty(8 * m, np.float32)
    p1_14 = s.vol.param14(0, 0, 0)
    for c0 in range(0, min(m, chunk), chunk):
        ctx.forward_comp_compete(rows5_h[c0:c0 + chunk], ids_h, eul_h, S9, B9, hkl, None, rot, R9, p, p1_14,
                                 out=out_h[8 * c0:8 * (c0 + chunk)])
    t0 = time.perf_counter()
    for c0 in range(0, m, chunk):
        c1 = min(m, c0 + chunk)
        ctx.forward_comp_compete(rows5_h[c0:c1], ids_h, eul_h, S9, B9, hkl, None, rot, R9, p, p1_14,
                                 out=out_h[8 * c0:8 * c1])
    host_chunked_ms = (time.perf_counter() - t0) * 1e3
    # one scorer call per voxel (the launch-bound extreme)
    nb = min(args.plain_voxels, m)
    one = torch.empty(8, dtype=torch.float32, device="cuda")
    for i in range(min(20, nb)):
        ctx.compete_device(d_rows5[5 * i:5 * i + 5], 1, d_ids, ids.size, d_eul, len(eul), param1, one)
    ctx.sync()
    t0 = time.perf_counter()
    for i in range(nb):
        ctx.compete_device(d_rows5[5 * i:5 * i + 5], 1, d_ids, ids.size, d_eul, len(eul), param1, one)
    ctx.sync()
    plain_s = time.perf_counter() - t0
    plain = float(rows5[:nb, 4].max() - rows5[0, 3] + 1) / plain_s
    line = {"metric": METRIC, "value": batched, "unit": "trials/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": graph_ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": SCORER_DTYPE, "data": "synthetic",
            "config": {"workload": (f"batched grow: FCC Al 400 grains, {m} voxels with 1-64 candidates "
                                    f"(Geometric p=0.15, neighbour grains + 0.5 deg perturbations), {T} trials "
                                    f"per iteration"),
                       "l2": "inputs larger than L2: resident map read every iteration"},
            "clocks": clk.summary(),
            "batched_graph": {"trials_per_s": batched, "ms_per_iteration": graph_ms},
            "batched_direct": {"trials_per_s": T / (direct_ms / 1e3), "ms_per_iteration": direct_ms},
            "graph_gain": direct_ms / graph_ms,
            "reference_chunks": {"trials_per_s": T / (chunked_ms / 1e3), "ms_per_iteration": chunked_ms,
                                 "note": (f"one grc_compete_device call per {chunk} voxels "
                                          "(revise_all_unindexed_voxel_cuda.m:77), CSR planned per call")},
            "speedup_vs_reference_chunks": chunked_ms / graph_ms,
            "reference_chunks_host": {"trials_per_s": T / (host_chunked_ms / 1e3), "ms_per_iteration": host_chunked_ms,
                                      "note": (f"one grc_forward_comp_compete call per {chunk} voxels with host "
                                               "buffers (the MEX entry), wall clock, one iteration")},
            "plain_per_voxel": {"trials_per_s": plain, "voxels_sampled": nb,
                                "note": "one grc_compete_device call (one scoring launch set) per voxel"},
            "speedup_vs_plain": batched / plain, "autotune": tune}
    print(json.dumps(line), flush=True)
    b.close()
    ctx.close()
    return 0


def seed_cpu_baseline(s, host_map, pos, q, nr_seed, evals_per_seed, n_scan=2048, nm_evals=300):
    """Oracle time per seed for the same indexing work: the scan and local-refine trials at the
    oracle's multi-core rate (a sample of ``n_scan`` orientations), the Nelder-Mead evaluations at
    its one-core rate (a sample of ``nm_evals`` evaluations: fminsearchbnd is sequential)."""
    from oracle import oracle as O
    from oracle import seed_oracle as SO
    S9, B9, hkl, rot, R9, p = s.mex_arrays()
    sc = SO.Scene(S9, B9, hkl, rot, R9, p, host_map)
    t0 = time.perf_counter()
    sc.scan(pos[0], q[:n_scan])
    t_trial = (time.perf_counter() - t0) / n_scan
    f = SO.nm_objective(sc, pos[0].astype(np.float64))
    x = np.asarray(q[0], np.float64)[1:]
    t0 = time.perf_counter()
    for k in range(nm_evals):
        f(x + 1e-5 * k)
    t_eval = (time.perf_counter() - t0) / nm_evals
    trials = len(q) + nr_seed * 730 + 1
    per_seed = trials * t_trial + evals_per_seed * t_eval
    return {"value": 1.0 / per_seed, "unit": "seeds/s", "cores": O.max_threads(), "kind": "port",
            "sample": (f"{n_scan} scan trials on {O.max_threads()} threads ({1 / t_trial:.0f} trials/s) and "
                       f"{nm_evals} Nelder-Mead evaluations on one thread ({1 / t_eval:.0f} evals/s), scaled to "
                       f"{trials} trials + {evals_per_seed:.0f} evaluations per seed"),
            "seconds_per_seed": per_seed}


def run_seed(args):
    """Seeding stage per seed: scan of the 32,768-orientation grid, top Nr_seed, local refine of
    every candidate (730 orientations each), batched fminsearchbnd, final scoring."""
    import torch
    from grainrecon_b200 import seeding as SD
    from grainrecon_b200 import synth
    from grainrecon_b200._lib import Context

    rank, world, local = env_rank()
    torch.cuda.set_device(local)
    s, pos, q = build_problem("al400", args.seed)
    ctx = Context(local)
    want_cpu = rank == 0 and not args.no_cpu_baseline
    host_map = synth.device_maps(s, ctx, keep_host_map=want_cpu)
    ix = SD.SeedIndexer(ctx, q, nr_seed=args.nr_seed)
    n = args.seed_batch
    pos64 = pos.astype(np.float64)

    def batch(k):
        lo = (k * n) % (len(pos64) - n)
        return list(range(lo + 1, lo + n + 1)), pos64[lo:lo + n]

    for k in range(args.warmup):
        ix.index(*batch(k))
    torch.cuda.synchronize()
    # phase split of one batch (separately synchronised, untimed)
    ids, p = batch(args.warmup)
    ph = {}
    t0 = time.perf_counter()
    cand = ix.candidates(p)
    torch.cuda.synchronize()
    ph["scan_top_s"] = time.perf_counter() - t0
    t0 = time.perf_counter()
    _, _, _, x0 = ix.refine(p, cand, 1)
    torch.cuda.synchronize()
    ph["local_refine_s"] = time.perf_counter() - t0
    t0 = time.perf_counter()
    x, fval, ev, it, fl = ix.fit_nm(p, x0)
    torch.cuda.synchronize()
    ph["nelder_mead_s"] = time.perf_counter() - t0
    t0 = time.perf_counter()
    ix.final(p, x)
    torch.cuda.synchronize()
    ph["final_s"] = time.perf_counter() - t0
    evals = ev.double().mean().item()
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        rows = None
        for k in range(args.steps):
            rows, _ = ix.index(*batch(args.warmup + 1 + k))
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
    dt = max_over_ranks(dt, torch.device("cuda", local))
    seeds = n * args.steps * world
    line = {"metric": "seeds indexed/s", "value": seeds / dt, "unit": "seeds/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": SCORER_DTYPE, "data": "synthetic",
            "config": {"workload": (f"seeding stage: FCC Al 400 grains, 2048x2048 detector, 361 projections; "
                                    f"{n} seeds per step x ({N_ORIENT} scan + {args.nr_seed} x 730 local-refine "
                                    f"trials + fminsearchbnd (<= 2000 evaluations) + 1 final)"),
                       "nr_seed": args.nr_seed, "seeds_per_step": n,
                       "l2": "inputs larger than L2: the resident map is read by every step"},
            "clocks": clk.summary(),
            "e2e": {"value": seeds / dt, "unit": "seeds/s", "h2d_bytes_per_step": n * 3 * 8,
                    "d2h_bytes_per_step": n * 18 * 8,
                    "note": "host seed positions in, host indexing rows out: the timed steps are end to end"},
            "phases_one_batch_s": ph, "nm_mean_evaluations": evals, "nm_converged": float((fl == 1).double().mean()),
            "mean_C": float(np.nanmean(rows[:, 6])) if rows is not None else None,
            "trials_per_seed": N_ORIENT + args.nr_seed * 730 + 1 + evals}
    if want_cpu:
        line["cpu_baseline"] = seed_cpu_baseline(s, host_map, pos, q, args.nr_seed, evals)
    if rank == 0:
        print(json.dumps(line), flush=True)
    ctx.close()
    return 0


def run_walk(args):
    """Best-first region growth (grow_indexed_region.m:32-137) of the three largest grains of the FCC
    Al sample, through grc_grow_best_first with host arrays: the native walk, its voxels scored
    on the GPU a block at a time."""
    import torch
    from grainrecon_b200 import geometry as G
    from grainrecon_b200 import synth
    from grainrecon_b200._lib import Context

    rank, world, local = env_rank()
    torch.cuda.set_device(local)
    s = synth.make_sample("al400", seed=args.seed)
    ctx = Context(local)
    host = synth.device_maps(s, ctx, keep_host_map=not args.no_cpu_baseline)
    S9, B9, hkl, rot, R9, p = s.mex_arrays()
    dims = s.grain_id.shape
    Imask = (s.grain_id > 0).astype(np.float64)
    idx = s.voxel_indices()
    gid = s.grain_id[tuple((idx - 1).T)]
    sizes = np.bincount(gid)
    grains = np.argsort(sizes)[::-1][:3]
    p1 = s.vol.param14(0, 0, 10)
    zeros, twenty = np.zeros(dims), np.zeros(dims) + 20
    cases = []
    for g in grains:
        members = idx[gid == g]
        cases.append((members[len(members) // 2], G.flat_rowmajor(G.quat_to_u(s.grain_q[g - 1]))))
    walk = lambda seed, U: ctx.grow_best_first(zeros, Imask, twenty, zeros, seed, 0.05, 3, 0.95, 10, U, S9, B9,
                                               hkl, None, rot, R9, p, p1)
    walk(*cases[0])  # warm-up
    with ClockSampler(local) as clk:
        t0 = time.perf_counter()
        grown = [len(walk(*c)[6]) for c in cases]
        dt = time.perf_counter() - t0
    line = {"metric": "best-first grown voxels/s", "value": sum(grown) / dt, "unit": "voxels/s", "n_gpus": 1,
            "higher_is_better": True, "dtype": SCORER_DTYPE, "data": "synthetic",
            "config": {"workload": (f"grow_indexed_region walk from the centre voxel of the 3 largest grains "
                                    f"({', '.join(str(int(sizes[g])) for g in grains)} voxels) of FCC Al 400 grains, "
                                    f"{int(Imask.sum())} voxels, 2048x2048 detector, 361 projections, drop_off 0.05")},
            "clocks": clk.summary(), "grown": grown, "seconds": dt}
    if rank == 0 and not args.no_cpu_baseline:
        # the oracle walk with the FP64 oracle scorer: its first 300 grown voxels of the first case
        from oracle import oracle as O
        from oracle import walk_oracle as WO
        seed, U = cases[0]

        def score(vox):
            rows6 = np.zeros((len(vox), 6), np.float32)
            rows6[:, :3] = vox
            out, _ = O.grow(rows6, U, S9, B9, hkl, host, rot, R9, p, p1)
            return out.reshape(-1, 7)[:, 3:6]

        n_grow = 300
        t0 = time.perf_counter()
        WO.best_first_growth(score, zeros, Imask, twenty, zeros, seed, 0.05, 3, 0.95, 10, stop_after=n_grow)
        per_voxel = (time.perf_counter() - t0) / n_grow
        line["cpu_baseline"] = {"value": 1.0 / per_voxel, "unit": "voxels/s", "cores": O.max_threads(),
                                "kind": "port", "sample": (f"oracle walk + FP64 oracle scorer: the first {n_grow} "
                                                           f"grown voxels of the first grain")}
    ctx.close()
    if rank == 0:
        print(json.dumps(line, default=float), flush=True)
    return 0


def run_map(args):
    """Whole mapping run of the BCC Fe sample (6 grains, 6,320 voxels, 1024x1024 detector, 181
    projections): GrainMapping_fun's iteration on the GPU engine from the masks alone."""
    import torch
    from grainrecon_b200 import forward as FW
    from grainrecon_b200 import geometry as G
    from grainrecon_b200 import mapping as M
    from grainrecon_b200 import synth

    rank, world, local = env_rank()
    torch.cuda.set_device(local)
    s = synth.make_sample("fe6", seed=args.seed)
    g = s.geom
    dims = s.grain_id.shape
    host = synth.device_maps(s, FW.context(), keep_host_map=True)
    FW.reset_masks()
    q_grid = G.cubic_fz_orientations(N_ORIENT, args.seed + 5).astype(np.float32)
    ts = {"Center": np.array(s.vol.center), "Dimension": np.array(s.vol.dimension)}
    rvp = np.array([[1, dims[0]], [1, dims[1]], [1, dims[2]]])
    mask = (s.grain_id > 0).astype(np.float64)
    pbb = host.transpose(2, 1, 0)
    # untimed: one wrapper call makes the map resident in the wrappers' context
    FW.ForwardCalc_OR_space_comp_cuda(s.vol.pos_of_index(s.voxel_indices()[0]), q_grid[:8], s.S, s.B, s.hkl,
                                      len(s.hkl), pbb, g.rot_angles, g.rot_det, g.lss, g.lsd, g.p0y, g.p0z,
                                      g.rot_axis_offset, g.dety00, g.detz00, g.pxy, g.pxz, g.detysize, g.detzsize,
                                      g.beamstop_y, g.beamstop_z, g.theta_max, g.lambda_min, g.lambda_max)
    call = lambda: M.GrainMapping_iterate(
        mask, {"q": q_grid}, g.rot_det, None, pbb, g.rot_angles, s.S, s.B, s.hkl, len(s.hkl), g.theta_max,
        g.lambda_min, g.lambda_max, g.lss, g.lsd, 0.85, 0.5, 0.5 * g.pxy, g.dety00, g.detz00, g.p0y, g.p0z,
        g.rot_axis_offset, g.pxy, g.pxz, g.detysize / 2 + 0.5, g.detzsize / 2 + 0.5, g.detysize, g.detzsize,
        g.beamstop_y, g.beamstop_z, 0.05, 3, ts, s.vol.vox_size, rvp, s.vol.simap, 10, iter_end=args.map_iters,
        seed=args.seed, batch=64, max_iter=args.map_iters)
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        t0 = time.perf_counter()
        DS, rows, seeds, nvox, frac = call()
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
    got = DS["GrainId"] > 0
    ops = [G.quat_to_u(o) for o in G._cubic_ops()]
    Ug = [G.quat_to_u(q) for q in s.grain_q]
    true_gid = s.grain_id[got]
    eul = DS["EulerZXZ"][:, got]
    good = 0
    for k in range(eul.shape[1]):
        Uf = G.euler_to_u(*np.radians(eul[:, k]))
        U0 = Ug[true_gid[k] - 1]
        c = max((np.trace(U0.T @ Uf @ C) - 1) / 2 for C in ops)
        good += np.degrees(np.arccos(np.clip(c, -1, 1))) < 1.0
    n_seeds = int(sum(len(r) for r in rows))
    tried = int(sum((r[:, 6] > 0).sum() for r in rows))  # seeds that were indexed (not skipped)
    line = {"metric": "sample mapping time", "value": dt, "unit": "s", "n_gpus": 1, "higher_is_better": False,
            "dtype": SCORER_DTYPE, "data": "synthetic",
            "config": {"workload": (f"GrainMapping iteration on BCC Fe 6 grains, {int(mask.sum())} voxels, "
                                    f"1024x1024 detector, 181 projections, {N_ORIENT}-orientation grid, "
                                    f"Nr_seed 400, up to {args.map_iters} iterations")},
            "clocks": clk.summary(), "iterations": len(frac), "indexed_fraction": frac,
            "voxels_with_true_orientation": float(good / max(1, got.sum())) if got.any() else 0.0,
            "seeds": n_seeds, "seeds_indexed": tried,
            "voxels_per_s": float(got.sum()) / dt}
    if rank == 0 and not args.no_cpu_baseline:
        # the same seeds on the oracle: scan + 400 x 730 refine trials + ~100 Nelder-Mead evaluations each
        cb = seed_cpu_baseline(s, host, s.vol.pos_of_index(s.voxel_indices()[:1]).astype(np.float32), q_grid,
                               400, 100.0)
        line["cpu_baseline"] = {"value": tried * cb["seconds_per_seed"], "unit": "s", "cores": cb["cores"],
                                "kind": "port",
                                "sample": cb["sample"] + f"; times the {tried} indexed seeds (growth not counted)"}
    if rank == 0:
        print(json.dumps(line, default=float), flush=True)
    return 0


def verify_fitted_completeness(ctx, fitted_geo10, seed, n_vox=64, n_or=1024):
    """Score the al400 sample's masks with the true and with the fitted geometry.

    Trials: ``n_vox`` sample voxels x (their grain's true orientation + ``n_or - 1`` random
    ones).  Returns the mean and max |C_fitted - C_true| and the share of trials whose
    (Nr_simu, Nr_intersect) did not change."""
    from grainrecon_b200 import fit as F
    from grainrecon_b200 import geometry as G
    from grainrecon_b200 import synth
    s = synth.make_sample("al400", seed=seed)
    synth.device_maps(s, ctx)
    idx = s.voxel_indices()
    rng = np.random.default_rng(seed + 17)
    pick = idx[rng.choice(len(idx), n_vox, replace=False)]
    gid = s.grain_id[pick[:, 0] - 1, pick[:, 1] - 1, pick[:, 2] - 1]
    pos = s.vol.pos_of_index(pick).astype(np.float32)
    rand_q = G.cubic_fz_orientations(n_or - 1, seed + 23).astype(np.float32)
    S9, B9, hkl, rot, R9, p = s.mex_arrays()
    gf = F.geometry_with(s.geom, fitted_geo10)
    R9f, pf = G.flat_rowmajor(gf.rot_det), gf.param20(s.nhkl)
    dc, same, hit_true = [], 0, 0
    for v in range(n_vox):
        q = np.concatenate([s.grain_q[gid[v] - 1][None].astype(np.float32), rand_q]).reshape(-1)
        a = ctx.forward_comp(pos[v], q, S9, B9, hkl, None, rot, R9, p).reshape(-1, 4)
        b = ctx.forward_comp(pos[v], q, S9, B9, hkl, None, rot, R9f, pf).reshape(-1, 4)
        ca, cb = np.nan_to_num(a[:, 2]), np.nan_to_num(b[:, 2])
        dc.append(np.abs(ca - cb))
        same += int(np.all(a[:, 0:2] == b[:, 0:2], axis=1).sum())
        hit_true += int(ca[0] > 0.9)
    dc = np.concatenate(dc)
    return {"trials": n_vox * n_or, "mean_abs_dC": float(dc.mean()), "max_abs_dC": float(dc.max()),
            "unchanged_trials": same / (n_vox * n_or), "true_orientation_C>0.9_voxels": hit_true}


def run_pair(args):
    """Spot pairing (forward_comp_pair_spots.m:73-80, grc_pair_spots) on the fe6 sample: each grain's
    orientation at 256 voxels of that grain, against the measured centroid list of all six grains
    (each grain's landings at its mean position, 0.5 px Gaussian noise, area 10 px) plus 20 spurious
    spots per projection.  Each call is synchronous (it returns the pair count); the device time
    of the K calls comes from CUDA events on the library's stream."""
    import ctypes as C

    import torch
    from grainrecon_b200 import fit as F
    from grainrecon_b200 import synth
    from grainrecon_b200._lib import PAIR_DTYPE, Context, _ptr

    rank, world, local = env_rank()
    torch.cuda.set_device(local)
    s = synth.make_sample("fe6", seed=args.seed)
    ctx = Context(local)
    synth.device_maps(s, ctx)
    g = s.geom
    S9, B9, hkl, rot, R9, p = s.mex_arrays()
    ctx.set_geometry(S9, B9, hkl, rot, R9, p)
    idx = s.voxel_indices()
    gid = s.grain_id[tuple((idx - 1).T)]
    ng = len(s.grain_q)
    q = np.asarray(s.grain_q, np.float64)
    centre = np.stack([s.vol.pos_of_index(idx[gid == k + 1]).mean(0) for k in range(ng)])
    d_grains = torch.from_numpy(np.concatenate([F.quat_to_rod(q), centre], 1).reshape(-1).copy()).cuda()
    spots = F.simulate_spots(ctx, F.geo10_of(g), d_grains, 0.5, args.seed + 1)
    rng = np.random.default_rng(args.seed + 2)
    n_fake = 20 * g.nrot
    sp_iw = torch.cat([spots.iw.long(), torch.arange(g.nrot, device="cuda").repeat_interleave(20)])
    fake = np.stack([rng.uniform(1, g.detysize, n_fake), rng.uniform(1, g.detzsize, n_fake)], 1)
    sp_uv = torch.cat([spots.uv.view(-1, 2), torch.from_numpy(fake).cuda()])
    sp = torch.cat([sp_uv, torch.full((len(sp_iw), 1), 10.0, dtype=torch.float64, device="cuda")], 1)
    order = torch.argsort(sp_iw, stable=True)
    d_sp = sp[order].contiguous().view(-1)
    n_sp = len(sp_iw)
    d_off = torch.zeros(g.nrot + 1, dtype=torch.int64, device="cuda")
    d_off[1:] = torch.cumsum(torch.bincount(sp_iw, minlength=g.nrot), 0)
    per = 256
    pos, quat = [], []
    for k in range(ng):
        mine = idx[gid == k + 1]
        pick = mine[rng.choice(len(mine), per, replace=len(mine) < per)]
        pos.append(s.vol.pos_of_index(pick))
        quat.append(np.repeat(q[k][None], per, 0))
    d_pos = torch.from_numpy(np.concatenate(pos).reshape(-1).copy()).cuda()
    d_q = torch.from_numpy(np.concatenate(quat).reshape(-1).copy()).cuda()
    n = ng * per
    pairs = ctx.pair_spots(d_pos, d_q, n, d_sp, n_sp, d_off)
    cap = max(len(pairs), 1)
    buf = torch.empty(cap * PAIR_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
    npairs = C.c_int64()
    torch.cuda.synchronize()

    def call():
        ctx._check(ctx.L.grc_pair_spots(ctx.h, _ptr(d_pos), _ptr(d_q), n, _ptr(d_sp), n_sp, _ptr(d_off),
                                        _ptr(buf), cap, C.byref(npairs)))

    for _ in range(args.warmup):
        call()
    stream = torch.cuda.ExternalStream(ctx.stream)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0 = time.perf_counter()
    ev0.record(stream)
    for _ in range(args.steps):
        call()
    ev1.record(stream)
    torch.cuda.synchronize()
    wall = (time.perf_counter() - t0) / args.steps
    dev_ms = ev0.elapsed_time(ev1) / args.steps
    assert npairs.value == len(pairs)
    line = {"metric": "spot pairing trials/s", "value": n / (dev_ms / 1e3), "unit": "trials/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": dev_ms, "higher_is_better": True,
            "dtype": "f64", "data": "synthetic",
            "config": {"workload": (f"fe6-pair: BCC Fe {ng} grains, {g.detysize}x{g.detzsize} detector, "
                                    f"{g.nrot} projections, {s.nhkl} reflections; {n} trials (each grain's "
                                    f"orientation at {per} of its voxels) against {n_sp} measured spots"),
                       "spots": n_sp, "trials": n},
            "pairs_per_step": int(npairs.value), "pairs_per_s": npairs.value / (dev_ms / 1e3),
            "wall_ms_per_step": wall * 1e3}
    print(json.dumps(line), flush=True)
    ctx.close()
    return 0


def run_fit(args):
    """Fit benchmarks: 5,000-grain orientation+centre fit (BCC Fe, 1024^2, 181 projections) or the
    10-parameter geometry fit (FCC Al, 2048^2, 361 projections, 2,000 grains, 64 starts)."""
    import torch
    from grainrecon_b200 import fit as F
    from grainrecon_b200 import synth
    from grainrecon_b200._lib import Context

    rank, world, local = env_rank()
    torch.cuda.set_device(local)
    kind = "fe6" if args.config == "fe-fit" else "al400"
    # the named set-up's geometry and lattice; a fit needs no volume or masks
    geom, cell, _, hkl, *_ = synth.named_setup(kind, seed=args.seed)
    from grainrecon_b200 import geometry as G
    ctx = Context(local)
    ctx.set_geometry(G.flat_rowmajor(np.eye(3)), G.flat_rowmajor(G.form_b(cell)), G.flat_hkl(hkl),
                     np.asarray(geom.rot_angles, np.float32), G.flat_rowmajor(geom.rot_det), geom.param20(len(hkl)))
    if args.config == "fe-fit":
        res = F.bench_grain_fit(ctx, geom, n_grains=args.fit_grains or 5000, seed=args.seed)
        lm = res["lm"]["reached"]
        metric = f"fit time to 0.1 px RMS (orientation + centre, {res['grains']} grains)"
    else:
        res = F.bench_geometry_fit(ctx, geom, n_grains=args.fit_grains or 2000, seed=args.seed,
                                   nm_iters=args.nm_iters)
        lm = res["lm"]["first_start_below"]
        res.pop("grains_array")
        fitted = res.pop("fitted_geo")
        res["fitted_geo"] = fitted.tolist()
        if not args.no_verify:
            res["completeness_with_fitted_geometry"] = verify_fitted_completeness(ctx, fitted, args.seed)
        metric = f"fit time to 0.1 px RMS (10-parameter geometry, {res['starts']} starts)"
    line = {"metric": metric, "value": lm["seconds"] if lm else None, "unit": "s", "n_gpus": 1,
            "higher_is_better": False, "dtype": "f64", "data": "synthetic",
            "config": {"workload": args.config, "geometry": kind}, "result": res}
    print(json.dumps(line, default=float), flush=True)
    ctx.close()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="al400", choices=["al400", "fe6", "al400-grow", "fe-fit", "al-geofit",
                                                                "al400-seed", "fe6-map", "al400-walk", "fe6-pair"])
    ap.add_argument("--map-iters", type=int, default=4, help="fe6-map: mapping iterations at most")
    ap.add_argument("--nr-seed", type=int, default=400, help="al400-seed: candidates refined per seed")
    ap.add_argument("--seed-batch", type=int, default=16, help="al400-seed: seeds per step")
    ap.add_argument("--fit-grains", type=int, default=0, help="0: 5,000 (fe-fit) or 2,000 (al-geofit)")
    ap.add_argument("--no-verify", action="store_true", help="al-geofit: skip the completeness re-check")
    ap.add_argument("--nm-iters", type=int, default=400)
    ap.add_argument("--grow-voxels", type=int, default=262144, help="voxels per batched-grow iteration")
    ap.add_argument("--plain-voxels", type=int, default=2000, help="voxels timed one call each")
    ap.add_argument("--seeds", type=int, default=64, help="seed voxels per step per GPU")
    ap.add_argument("--output", default="completeness", choices=["completeness", "full"],
                    help="seeding-scan output: completeness only (bit-packed mask) or the four MEX columns")
    ap.add_argument("--path", type=int, default=0, choices=[0, 1, 2, 3],
                    help="scoring kernel (grc_set_path): 0 by size, 1 per-trial, 2 CTA sweep, 3 warp scan")
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--cpu-trials", type=int, default=8192)
    ap.add_argument("--ref-trials", type=int, default=2048, help="orientations per reference step")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profile", action="store_true", help="stop after the timed device steps (for ncu)")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.config == "al400-grow":
        return run_grow(args)
    if args.config in ("fe-fit", "al-geofit"):
        return run_fit(args)
    if args.config == "al400-seed":
        return run_seed(args)
    if args.config == "fe6-map":
        return run_map(args)
    if args.config == "al400-walk":
        return run_walk(args)
    if args.config == "fe6-pair":
        return run_pair(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
