#!/usr/bin/env python
"""AO any-hit ray-query throughput on B200.

Default workload (the batched configuration): 64 procedural scenes
(heightfield + boxes family) with triangle counts log-uniform in [10k, 2M] and
AO ray counts log-uniform in [256K, 8M] (cosine-weighted from uniform surface
samples, tmin = 1e-4 diag, tmax = 0.1 diag), all traced any-hit in one
persistent batch launch (Morton sort + CUDA graph, parameters from the
autotuner), beside 64 plain per-scene launches of the same kernel family and
the reference's own CWBVH kernel rebuilt for sm_100a.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl rq|reference]
                    [--workload batched|small] [--quick]

One JSON line on rank 0.  Under torchrun each rank traces its own copy of
the workload (weak scaling, no data-path collective); time is the max over
ranks.  Rays and hits exceed L2 (inputs larger than L2 between steps).
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import json
import math
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "AO any-hit Mrays/s on 1 B200, batched/served vs plain launch; p50/p99 latency"
BATCHED_WORKLOAD = "batched: 64 heightfield+box scenes, tris log-U[10k,2M], AO any-hit rays log-U[256K,8M]"
PEAKS = ROOT / "MEASURED_PEAKS.json"


def log(*a):
    print(*a, file=sys.stderr, flush=True)


# --------------------------------------------------------------- workload --

def workload_spec(name: str, quick: bool, rank: int):
    """Scenes are the same on every rank (scene seed = item index) and every
    rank traces its own rays (ray seed per rank), so the replicas do equal
    host work and take the same code paths."""
    from cwbvh_b200.replicas import rank_seed
    from cwbvh_b200.workloads import batched_sizes
    if name == "small":
        return [dict(seed=0, ray_seed=rank_seed(0, rank) + 1000, tris=10592, rays=1 << 20, small=True)]
    tris, rays = batched_sizes(64 if not quick else 8)
    if quick:
        tris = np.minimum(tris, 200_000)
        rays = np.minimum(rays, 1 << 20)
    return [dict(seed=i, ray_seed=rank_seed(i, rank) + 1000, tris=int(t), rays=int(r), small=False)
            for i, (t, r) in enumerate(zip(tris, rays))]


def build_scenes(spec, threads_per_build: int = 1):
    import cwbvh_b200 as rq
    from cwbvh_b200 import workloads as W

    def one(s):
        V, I = W.heightfield_boxes(s["seed"]) if s["small"] else W.scene_of_size(s["seed"], s["tris"])
        hb = rq.HostBVH(V, I, rq.CWBVH, threads=threads_per_build)
        return V, I, hb

    # ranks on one node share its cores
    ranks_here = max(1, int(os.environ.get("LOCAL_WORLD_SIZE", "1")))
    workers = max(1, min(len(spec), (os.cpu_count() or 1) // ranks_here))
    with cf.ThreadPoolExecutor(max_workers=workers) as ex:
        return list(ex.map(one, spec))


# ------------------------------------------------------------------ timing --

class Clocks:
    """nvidia-smi samples (200 ms) during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.p = None
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={index}", f"--query-gpu={self.Q}", "--format=csv,noheader",
                                       "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (OSError, FileNotFoundError):
            self.p = None

    def stop(self) -> dict:
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            out, _ = self.p.communicate(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
            out, _ = self.p.communicate()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1].split()[0]))
                smax.append(float(f[2].split()[0]))
            except ValueError:
                continue
            for k, nm in enumerate(names):
                if f[5 + k].lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        loaded = [s for s in sm if s > 0.5 * max(sm)] or sm
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm)}


def time_steps(fn, steps: int, warmup: int, stream, dist=None, flush=None) -> float:
    """ms per step: CUDA events on `stream`, synchronize + barrier on both sides, max over ranks."""
    import torch
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    if flush is None:
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
    else:
        # inputs smaller than L2: write `flush` (larger than L2) before each
        # step, outside the events, so every step starts from a cold L2
        evs = []
        for _ in range(steps):
            with torch.cuda.stream(stream):
                flush.add_(1)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            fn()
            b.record(stream)
            evs.append((a, b))
        torch.cuda.synchronize()
        ms = sum(a.elapsed_time(b) for a, b in evs) / steps
    if dist is not None:
        from cwbvh_b200.replicas import max_over_ranks
        ms = max_over_ranks(ms, dist, device="cuda")
        dist.barrier()
    return ms


def measured_peak_hbm():
    try:
        p = json.loads(PEAKS.read_text())
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def measure_l2_read(stream) -> dict:
    """L2 read bandwidth (GB/s) from the library's probe kernel
    (rq_probe_l2_read_shape): coalesced L1-bypassing 16-byte loads over an
    L2-resident buffer, swept over buffer size (8/16/32/48 MB), grid
    (SMs x 8/16/32 blocks of 256 threads) and loads in flight per thread
    (4/8); the best shape is the peak."""
    import torch
    import cwbvh_b200 as rq
    with torch.cuda.stream(stream):
        buf = torch.ones((48 << 20) // 4, dtype=torch.int32, device="cuda")
        sink = torch.zeros(1, dtype=torch.int32, device="cuda")
    sweep = []
    for mb in (8, 16, 32, 48):
        n = mb << 20
        reps = max(1, (4 << 30) // n)  # ~4 GiB read per call
        for bps in (8, 16, 32):
            for loads in (4, 8):
                def run():
                    rq.check(rq.lib.rq_probe_l2_read_shape(buf.data_ptr(), n, reps, bps, loads, sink.data_ptr(),
                                                           stream.cuda_stream), "rq_probe_l2_read_shape")
                ms = time_steps(run, 5, 2, stream)
                sweep.append({"mbytes": mb, "blocks_per_sm": bps, "loads": loads,
                              "gbs": round(n * reps / (ms * 1e-3) / 1e9, 1)})
    best = max(sweep, key=lambda r: r["gbs"])
    return {"peak": best["gbs"], "best": best, "sweep": sweep}


def probe_l2_shape(args, warmup: int) -> None:
    """One shape of the L2 read probe (``--probe-l2 MB,BLOCKS_PER_SM,LOADS``),
    W + K launches of 16 passes over the buffer each, for an ncu capture of
    the probe kernel alone; prints its GB/s (CUDA events)."""
    import torch
    import cwbvh_b200 as rq
    mb, bps, loads = (int(x) for x in args.probe_l2.split(","))
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        buf = torch.ones((mb << 20) // 4, dtype=torch.int32, device="cuda")
        sink = torch.zeros(1, dtype=torch.int32, device="cuda")
    reps = 16

    def run():
        rq.check(rq.lib.rq_probe_l2_read_shape(buf.data_ptr(), mb << 20, reps, bps, loads, sink.data_ptr(),
                                               stream.cuda_stream), "rq_probe_l2_read_shape")
    ms = time_steps(run, args.steps, warmup, stream)
    print(json.dumps({"probe": "l2_read", "mbytes": mb, "blocks_per_sm": bps, "loads": loads, "reps": reps,
                      "ms": round(ms, 4), "gbs": round((mb << 20) * reps / (ms * 1e-3) / 1e9, 1)}), flush=True)


def measure_link(mbytes: int = 1024) -> dict:
    """Host link bandwidth with pinned buffers: H2D alone, D2H alone and both
    directions at once on two streams (GB/s), 1 GiB copies."""
    import torch
    n = mbytes << 20
    h = torch.empty(n, dtype=torch.uint8, pin_memory=True)
    h2 = torch.empty(n, dtype=torch.uint8, pin_memory=True)
    d = torch.empty(n, dtype=torch.uint8, device="cuda")
    d2 = torch.empty(n, dtype=torch.uint8, device="cuda")
    s1, s2 = torch.cuda.Stream(), torch.cuda.Stream()

    def timed(fn, reps=3):
        fn()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(reps):
            fn()
        torch.cuda.synchronize()
        return (time.perf_counter() - t0) / reps

    def both():
        with torch.cuda.stream(s1):
            d.copy_(h, non_blocking=True)
        with torch.cuda.stream(s2):
            h2.copy_(d2, non_blocking=True)
    h2d = n / timed(lambda: d.copy_(h, non_blocking=True)) / 1e9
    d2h = n / timed(lambda: h2.copy_(d2, non_blocking=True)) / 1e9
    duplex = 2 * n / timed(both) / 1e9
    return {"h2d_gbs": round(h2d, 1), "d2h_gbs": round(d2h, 1), "duplex_gbs": round(duplex, 1)}


def link_bound_ms(h2d_bytes: float, d2h_bytes: float, link: dict) -> float:
    """Least time to move the bytes: the two directions overlap at the duplex
    rate (half each) until the smaller is done, then the rest one way."""
    each = link["duplex_gbs"] / 2 * 1e9
    small, big = sorted((h2d_bytes, d2h_bytes))
    rest_rate = (link["h2d_gbs"] if h2d_bytes >= d2h_bytes else link["d2h_gbs"]) * 1e9
    return (small / each + (big - small) / rest_rate) * 1e3


def issue_roofline(workload: str, rays_per_s: float, sm_mhz) -> dict:
    """The bound the trace kernel actually meets: instruction issue.  Warp
    instructions per ray come from the committed ncu capture of the same
    kernel on a reduced case (profiles/issue_<workload>.json); the peak is one
    warp instruction per scheduler per cycle: SMs x 4 x the median SM clock
    sampled during the timed region."""
    f = ROOT / "profiles" / f"issue_{workload}.json"
    try:
        prof = json.loads(f.read_text())
    except Exception:
        return None
    try:
        import torch
        sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
    except Exception:
        sms = 148
    clock_note = "median SM clock in the timed region"
    if not sm_mhz:
        try:
            sm_mhz = float(json.loads(PEAKS.read_text())["sm_max_mhz"])
            clock_note = "sm_max_mhz of MEASURED_PEAKS.json (clocks not sampled in this run)"
        except Exception:
            return None
    ipr = float(prof["warp_inst_per_ray"])
    achieved = rays_per_s * ipr / 1e9
    peak = sms * 4 * float(sm_mhz) * 1e6 / 1e9
    return {"achieved": round(achieved, 1), "peak": round(peak, 1), "unit": "G warp-inst/s",
            "frac": round(achieved / peak, 4), "warp_inst_per_ray": ipr,
            "thread_inst_per_warp_inst": prof.get("thread_inst_per_warp_inst"),
            "peak_source": f"{sms} SMs x 4 schedulers x {sm_mhz:.0f} MHz ({clock_note})",
            "source": prof.get("source")}


def profile_traffic(workload: str):
    """DRAM bytes per launch of the trace kernel from the committed ncu summary, if any."""
    f = ROOT / "profiles" / f"traffic_{workload}.json"
    try:
        return json.loads(f.read_text())
    except Exception:
        return None


# ------------------------------------------------------------- CPU legs --

def cpu_sample(spec, built, target_rays: int, seed: int = 7):
    """A bounded sample of the workload on the host: rays from every scene,
    proportionally to its ray count, generated with the host's numpy RNG."""
    rng = np.random.default_rng(seed)
    total = sum(s["rays"] for s in spec)
    out = []
    for s, (V, I, hb) in zip(spec, built):
        k = max(64, int(round(target_rays * s["rays"] / total)))
        tri = rng.integers(0, I.shape[0], k)
        a = np.sqrt(rng.random(k)).astype(np.float32)
        b = rng.random(k).astype(np.float32)
        p0, p1, p2 = V[I[tri, 0]], V[I[tri, 1]], V[I[tri, 2]]
        P = p0 * (1 - a)[:, None] + p1 * (b * a)[:, None] + p2 * (1 - (1 - a) - b * a)[:, None]
        nrm = np.cross(p1 - p0, p2 - p0)
        nrm /= np.maximum(np.linalg.norm(nrm, axis=1, keepdims=True), 1e-30)
        u1, u2 = rng.random(k), rng.random(k)
        r, ph = np.sqrt(u1), 2 * np.pi * u2
        t1 = np.cross(nrm, [0.0, 0.0, 1.0])
        short = np.linalg.norm(t1, axis=1) < 0.1
        t1[short] = np.cross(nrm[short], [0.0, 1.0, 0.0])
        t1 /= np.linalg.norm(t1, axis=1, keepdims=True)
        t2 = np.cross(t1, nrm)
        d = t1 * (r * np.cos(ph))[:, None] + t2 * (r * np.sin(ph))[:, None] + nrm * np.sqrt(1 - u1)[:, None]
        dg = float(np.linalg.norm(V.max(0) - V.min(0)))
        rays = np.zeros((k, 8), np.float32)
        rays[:, 0:3], rays[:, 3] = P, 1e-4 * dg
        rays[:, 4:7], rays[:, 7] = d, 0.1 * dg
        out.append((hb, rays))
    return out


def time_cpu(sample, threads: int = 0) -> tuple[float, int]:
    from oracle import pyoracle as po
    n = sum(r.shape[0] for _, r in sample)
    t0 = time.perf_counter()
    for hb, rays in sample:
        po.trace(0, hb.nodes, hb.woop, rays, True, threads=threads)
    return time.perf_counter() - t0, n


# ------------------------------------------------------------------ main --

def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="rq", choices=["rq", "reference"])
    ap.add_argument("--workload", default="batched", choices=["batched", "small", "city", "large", "instanced"])
    ap.add_argument("--rays", type=int, default=0, help="large: total AO rays (default 64M; 16M with --quick)")
    ap.add_argument("--quick", action="store_true", help="8 smaller scenes (smoke runs)")
    ap.add_argument("--no-ref-gpu", action="store_true")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline (profiler runs)")
    ap.add_argument("--no-serving", action="store_true", help="skip the serving configuration")
    ap.add_argument("--dump-reference-inputs", default="", help=argparse.SUPPRESS)
    ap.add_argument("--subset", type=int, default=0,
                    help="batched: only the first N scenes (reduced cases for profiler captures)")
    ap.add_argument("--ray-cap", type=int, default=0, help="batched: at most this many rays per scene")
    ap.add_argument("--no-configs", action="store_true",
                    help="batched: skip the small, city and large configurations (run in their own processes)")
    ap.add_argument("--probe-l2", default="",
                    help="MB,BLOCKS_PER_SM,LOADS: run only the L2 read probe at that shape W+K times (profiler captures)")
    ap.add_argument("--profile", action="store_true",
                    help="batched/small/large: build the workload and only run the trace W+K times (profiler captures)")
    args = ap.parse_args()
    warmup = max(3, args.warmup)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.dump_reference_inputs:
        return dump_reference_inputs(args, args.dump_reference_inputs)
    if args.impl == "reference":
        return run_reference(args, world, rank, warmup)

    # ---- the other single-GPU configurations, each in its own process and
    # before this one opens the device (so no buffer, stream or context of
    # this process shares the GPU with them): the plain small scene, the city
    # and the 30M-triangle scene, with their own rooflines
    configs = None
    if (args.workload == "batched" and not args.quick and world == 1 and not args.no_configs and not args.probe_l2
            and not args.profile and args.subset == 0 and args.ray_cap == 0):
        t0 = time.time()
        configs = {"config0_plain_small": run_config_process("small", args, warmup),
                   "config1_city": run_config_process("city", args, warmup),
                   "config2_large": run_config_process("large", args, warmup)}
        log(f"[bench] configs 0-2 {time.time()-t0:.1f}s")

    import torch
    import torch.distributed as tdist
    import datetime
    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                 device_id=torch.device("cuda", local_rank))
        dist = tdist

    import cwbvh_b200 as rq
    from cwbvh_b200 import workloads as W

    if args.probe_l2:
        return probe_l2_shape(args, warmup)
    if args.workload in ("city", "large", "instanced"):
        {"city": run_city, "large": run_large, "instanced": run_instanced}[args.workload](args, world, rank, dist)
        if dist is not None:
            dist.barrier()
            dist.destroy_process_group()
        return

    spec = workload_spec(args.workload, args.quick, rank)
    if args.subset > 0:
        spec = spec[:args.subset]
    if args.ray_cap > 0:
        for sp in spec:
            sp["rays"] = min(sp["rays"], args.ray_cap)
    t0 = time.time()
    built = build_scenes(spec)
    log(f"[bench] built {len(spec)} scenes, {sum(s['tris'] for s in spec)/1e6:.1f}M tris in {time.time()-t0:.1f}s")

    stream = torch.cuda.Stream()
    ctx = rq.Context()
    scenes, rays, hits = [], [], []
    with torch.cuda.stream(stream):
        for s, (V, I, hb) in zip(spec, built):
            sc = rq.Scene.from_host(hb)
            ds = W.DeviceScene(rq.CWBVH, hb, sc, torch.from_numpy(V).cuda(), torch.from_numpy(I).cuda(),
                               W.diag(V), I.shape[0])
            r = W.ao_rays(ds, s["rays"], seed=s["ray_seed"], stream=stream)
            scenes.append(ds)
            rays.append(r)
            hits.append(torch.empty((s["rays"], 4), device="cuda"))
    torch.cuda.synchronize()
    total_rays = sum(s["rays"] for s in spec)
    items = [(ds.scene, r, h) for ds, r, h in zip(scenes, rays, hits)]
    log(f"[bench] {total_rays/1e6:.1f}M rays on device")

    if args.profile:
        # For profiler captures: only the batch (default launch shape, no
        # sort, no graph), W + K runs, so the trace kernel launches come
        # right after the set-up and nothing else is timed.
        batch = rq.Batch(ctx, items, rq.ANY, sort_threshold=-1, use_graph=False)
        for _ in range(warmup + args.steps):
            batch.run(stream)
        torch.cuda.synchronize()
        ctx.check(stream)
        log(f"[bench] profile mode: {warmup + args.steps} batch runs of {total_rays} rays")
        return

    # ---- plain per-scene launches (the denominator of the batching target)
    def plain():
        for ds, r, h in zip(scenes, rays, hits):
            rq.trace(ctx, ds.scene, r, h, rq.ANY, stream=stream)

    flush = None
    if args.workload == "small":  # 1M rays + hits (48 MB) fit in L2
        with torch.cuda.stream(stream):
            flush = torch.zeros(64 << 20, dtype=torch.int32, device="cuda")  # 256 MB > 126 MB L2
    ms_plain = time_steps(plain, args.steps, warmup, stream, dist, flush)
    ctx.check(stream)
    plain_occ = [h[:, 1].view(torch.int32).ne(-1).sum().item() for h in hits]

    # ---- batched: autotuned sort threshold / block size / stack depth, CUDA graph
    cache = os.environ.get("RQ_TUNE_CACHE") or None  # a file path chosen by the caller, e.g. under /tmp
    t0 = time.time()
    bp = rq.autotune_batch(ctx, items, rq.ANY, cache_path=cache, stream=stream)
    log(f"[bench] autotune {time.time()-t0:.1f}s -> block {bp.launch.block_size} smem {bp.launch.smem_stack} "
        f"postpone {bp.launch.postpone_ratio:.2f} fetch {bp.launch.fetch_nd}/{bp.launch.fetch_nw} "
        f"sort_threshold {bp.sort_threshold} graph {bp.use_graph}")
    batch = rq.Batch(ctx, items, rq.ANY, params=bp)
    ms_batch = time_steps(lambda: batch.run(stream), args.steps, warmup, stream, dist, flush)
    ctx.check(stream)
    batch_occ = [h[:, 1].view(torch.int32).ne(-1).sum().item() for h in hits]
    occlusion_identical = plain_occ == batch_occ

    # trace kernel alone (the dominant kernel) for the roofline
    batch.run(stream)
    ms_kernel = time_steps(lambda: rq.lib.rq_batch_run_stage(batch._h, 2, stream.cuda_stream), args.steps, warmup,
                           stream, dist, flush)
    ms_sort = time_steps(lambda: rq.lib.rq_batch_run_stage(batch._h, 1, stream.cuda_stream), 3, 1, stream, dist)
    launches_per_step = int(rq.lib.rq_batch_kernel_count(batch._h))

    # ---- clocks during a timed batched region (long enough for >= 10 samples)
    reps = max(args.steps, int(math.ceil(2000.0 / max(ms_batch, 1e-3))))
    clk = Clocks(torch.cuda.current_device())
    time.sleep(0.3)
    ms_batch2 = time_steps(lambda: batch.run(stream), reps, 1, stream, dist)
    clocks = clk.stop()
    clocks["timed_steps"] = reps

    # ---- end to end through the public API with host buffers
    host_rays = [torch.empty(r.shape, dtype=r.dtype, pin_memory=True) for r in rays]
    host_hits = [torch.empty(h.shape, dtype=h.dtype, pin_memory=True) for h in hits]
    for hr, r in zip(host_rays, rays):
        hr.copy_(r)

    def e2e():
        for hr, r in zip(host_rays, rays):
            r.copy_(hr, non_blocking=True)
        batch.run(stream)
        for hh, h in zip(host_hits, hits):
            hh.copy_(h, non_blocking=True)

    with torch.cuda.stream(stream):
        ms_e2e = time_steps(e2e, args.steps, warmup, stream, dist)

    # The same host buffers through the server (public API): each scene's rays
    # are one request; three streams overlap copies with tracing (3 x 8M rays
    # per launch measured best: 0.95 of the link bound, 16M 0.93, 4 streams 0.80).
    srv = rq.Server(hbm_budget_bytes=40 * 10 ** 9, query=rq.ANY, streams=3, max_batch_rays=8 * 1024 * 1024)
    sids = [srv.add_scene(ds.scene) for ds in scenes]
    hr_np = [h.numpy() for h in host_rays]
    hh_np = [h.numpy() for h in host_hits]

    def served_step():
        ts = [srv.submit(sid, a, b) for sid, a, b in zip(sids, hr_np, hh_np)]
        for t in ts:
            srv.wait(t)

    for _ in range(warmup):
        served_step()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        served_step()
    torch.cuda.synchronize()
    ms_e2e_served = (time.perf_counter() - t0) * 1e3 / args.steps
    if dist is not None:
        from cwbvh_b200.replicas import max_over_ranks
        ms_e2e_served = max_over_ranks(ms_e2e_served, dist, device="cuda")
    srv.close()

    # ---- algorithmic bytes per ray: 32 (ray) + 16 (hit) + 80 per node + 48 per triangle
    nodes_total, tris_total = 0, 0
    with torch.cuda.stream(stream):  # counters are allocated, written and summed on one stream
        for ds, r in zip(scenes, rays):
            hh = torch.empty((r.shape[0], 4), device="cuda")
            nv, nt = rq.trace_counted(ctx, ds.scene, r, hh, rq.ANY, stream=stream)
            nodes_total += int(nv.sum(dtype=torch.int64).item())
            tris_total += int(nt.sum(dtype=torch.int64).item())
            del hh, nv, nt
    ctx.check(stream)
    alg_bytes = 48 * total_rays + 80 * nodes_total + 48 * tris_total
    peak, peak_kind = measured_peak_hbm()
    achieved = alg_bytes / (ms_kernel * 1e-3) / 1e9
    traffic = profile_traffic(args.workload + ("_quick" if args.quick else ""))
    l2 = measure_l2_read(stream)
    l2_gbs = l2["peak"]
    link = measure_link()
    link_ms = link_bound_ms(total_rays * 32, total_rays * 16, link)

    # ---- the reference's CWBVH kernel rebuilt for sm_100a, same rays (closest-hit: its only mode)
    # (at N = 1 only, like the serving and CPU baselines below: reference figures, not the scaled value)
    ref_gpu = None
    if not args.no_ref_gpu and world == 1:
        ref_gpu, ref_hits = run_ref_gpu(scenes, rays, warmup=1, steps=2)
        if ref_hits and ref_gpu.get("value"):
            # This library's closest-hit batch on the same rays: the like-for-like figure, and the
            # closest triangles compared with the reference kernel's.
            chits = [torch.empty_like(h) for h in hits]
            citems = [(ds.scene, r, h) for ds, r, h in zip(scenes, rays, chits)]
            # closest-hit gets its own autotuned launch (refill and postponing
            # settings that suit any-hit need not suit closest-hit)
            cbp = rq.autotune_batch(ctx, citems, rq.CLOSEST, cache_path=cache, stream=stream)
            cbatch = rq.Batch(ctx, citems, rq.CLOSEST, params=cbp)
            ms_closest = time_steps(lambda: cbatch.run(stream), args.steps, warmup, stream, dist, flush)
            ctx.check(stream)
            same = total_n = bad_mine = bad_ref = 0
            for ds, mine, theirs in zip(scenes, chits, ref_hits):
                pm = torch.from_numpy(ds.host.prim_index).cuda()
                n_pm = pm.numel()
                a, b = mine[:, 1].view(torch.int32), theirs[:, 1].view(torch.int32)
                # indices are clamped into the map; addresses outside it are counted, not looked up
                bad_mine += int((a >= n_pm).sum().item())
                bad_ref += int((b >= n_pm).sum().item())
                pa = torch.where((a >= 0) & (a < n_pm), pm[a.clamp(0, n_pm - 1).long()], torch.full_like(a, -1))
                pb = torch.where((b >= 0) & (b < n_pm), pm[b.clamp(0, n_pm - 1).long()], torch.full_like(b, -1))
                same += int((pa == pb).sum().item())
                total_n += int(a.numel())
            ref_gpu["this_library_closest_hit"] = {
                "value": round(total_rays / (ms_closest * 1e-3) / 1e6, 2), "unit": "Mrays/s",
                "ms_per_step": round(ms_closest, 4),
                "launch": {"block": cbp.launch.block_size, "smem_stack": cbp.launch.smem_stack,
                           "postpone_ratio": round(cbp.launch.postpone_ratio, 3),
                           "fetch_nd_nw": [cbp.launch.fetch_nd, cbp.launch.fetch_nw],
                           "what": "one persistent batch, autotuned for closest-hit"},
                "closest_prim_ids_equal_frac": round(same / max(total_n, 1), 6),
                "hit_addresses_outside_the_primitive_map": {"this_library": bad_mine, "reference": bad_ref}}
            ref_gpu["closest_vs_reference_kernel"] = round(total_rays / (ms_closest * 1e-3) / 1e6 / ref_gpu["value"],
                                                          3)
            cbatch.close()
            del chits

    # ---- the plain config's per-kernel table: CWBVH and BVH2, any-hit and closest-hit, + the reference's BVH2
    kernels = None
    if args.workload == "small":
        kernels = run_small_kernels(args, built, scenes, rays, stream, ctx, dist, warmup, flush)

    # ---- serving configuration (continuous batching vs one request per launch)
    serving = None
    if not args.no_serving and args.workload == "batched" and not args.quick and world == 1:
        del host_rays, host_hits
        torch.cuda.empty_cache()
        t0 = time.time()
        serving = run_serving()
        log(f"[bench] serving {time.time()-t0:.1f}s")

    # ---- where batching gains over plain launches: per-scene plain launch
    # times against the batch's rate, and a regime of many small items
    batching = None
    if args.workload == "batched" and not args.quick and world == 1:
        t0 = time.time()
        batching = batching_breakdown(ctx, scenes, rays, hits, ms_batch, stream, warmup)
        batching["small_items"] = batching_small_items(ctx, stream, warmup, args.steps)
        log(f"[bench] batching breakdown {time.time()-t0:.1f}s")

    # ---- CPU baseline (oracle restatement, all host threads, bounded sample)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baseline(spec, built)

    world_rays = total_rays * world
    value = world_rays / (ms_batch * 1e-3) / 1e6
    line = {
        "metric": METRIC,
        "value": round(value, 2),
        "unit": "Mrays/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": warmup,
        "ms_per_step": round(ms_batch, 4),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded procedural scenes and AO rays; the reference's mesh.dat/samplecache.dat are not shipped)",
        "config": {
            "workload": (BATCHED_WORKLOAD + ", one persistent launch, " +
                         ("Morton sort (threshold %d rays), " % bp.sort_threshold if bp.sort_threshold >= 0
                          else "Morton sort off (autotuner), ") +
                         ("CUDA graph, " if bp.use_graph else "") + "autotuned")
            if args.workload == "batched" and not args.quick else f"{args.workload}{' (quick)' if args.quick else ''}",
            "scenes": len(spec),
            "triangles": int(sum(s["tris"] for s in spec)),
            "rays_per_gpu": int(total_rays),
            "query": "any-hit",
            "layout": "CWBVH 80 B nodes, Woop 48 B triangles, Ray 32 B, Hit 16 B",
            "launch": {"block": bp.launch.block_size, "smem_stack": bp.launch.smem_stack,
                       "postpone_ratio": round(bp.launch.postpone_ratio, 3),
                       "fetch_nd_nw": [bp.launch.fetch_nd, bp.launch.fetch_nw],
                       "sort_threshold": int(bp.sort_threshold), "cuda_graph": bool(bp.use_graph)},
            "l2": ("inputs larger than L2 (rays+hits %.1f GB per step)" % (total_rays * 48 / 1e9)) if flush is None
            else "L2 flushed before every timed step (256 MB write outside the events; rays+hits are 48 MB)",
            "parallelism": f"replicas x{world} (rays independent, no data-path collective)",
        },
        "plain_per_scene": {"value": round(world_rays / (ms_plain * 1e-3) / 1e6, 2), "unit": "Mrays/s",
                            "ms_per_step": round(ms_plain, 4), "launches_per_step": 2 * len(spec)},
        "batched_vs_plain": round(ms_plain / ms_batch, 3),
        "occlusion_identical_batched_vs_plain": occlusion_identical,
        "stages_ms": {"sort": round(ms_sort, 4), "trace_kernel": round(ms_kernel, 4)},
        "e2e": {"value": round(world_rays / (max(ms_e2e_served, 1e-9) * 1e-3) / 1e6, 2), "unit": "Mrays/s",
                "h2d_bytes_per_step": int(total_rays * 32), "d2h_bytes_per_step": int(total_rays * 16),
                "ms_per_step": round(ms_e2e_served, 4),
                "path": "rq.Server (C ABI rq_server_*): 64 requests of host pinned rays/hits per step, 3 streams; "
                        "host wall clock with the device idle on both sides",
                "single_stream": {"value": round(world_rays / (ms_e2e * 1e-3) / 1e6, 2),
                                  "ms_per_step": round(ms_e2e, 4),
                                  "path": "H2D rays + rq_batch_run + D2H hits on one stream, CUDA events"},
                "link": dict(link, bound_ms_per_step=round(link_ms, 3),
                             bound_mrays_per_s=round(total_rays / (link_ms * 1e-3) / 1e6, 1),
                             frac=round(link_ms / max(ms_e2e_served, 1e-9), 4),
                             what="host link measured in this run (pinned 1 GiB copies); bound = least time to move "
                                  "this step's H2D and D2H bytes")},
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "peak_source": f"hbm_gbs of {peak_kind}",
                     "traffic": (traffic or {}).get("dram_bytes_per_launch"),
                     "algorithmic_bytes_per_launch": int(alg_bytes),
                     "bytes_per_ray": round(alg_bytes / total_rays, 1),
                     "nodes_per_ray": round(nodes_total / total_rays, 3),
                     "tris_per_ray": round(tris_total / total_rays, 3),
                     "l2": {"peak": round(l2_gbs, 1), "frac": round(achieved / l2_gbs, 4),
                            "peak_source": "rq_probe_l2_read_shape: best of 24 shapes (8-48 MB L2-resident buffers, "
                                           "coalesced 16 B L1-bypassing loads, SMs x 8/16/32 blocks, 4/8 loads in "
                                           "flight), measured in this run",
                            "best_shape": l2["best"]},
                     "issue": issue_roofline(args.workload + ("_quick" if args.quick else ""),
                                             total_rays / (ms_kernel * 1e-3), clocks.get("sm_mhz"))},
        "gpu_launches": int(launches_per_step * args.steps),
        "clocks": clocks,
        "clocks_ms_per_step": round(ms_batch2, 4),
    }
    if serving is not None:
        line["serving"] = serving
    if configs is not None:
        line["configs"] = configs
    if batching is not None:
        line["batching"] = batching
    if kernels is not None:
        line["kernels"] = kernels
    if ref_gpu is not None:
        line["reference_cwbvh_kernel_sm100a"] = ref_gpu
        if ref_gpu.get("value"):
            line["batched_vs_reference_kernel"] = round(value / world / ref_gpu["value"], 3)
    if cpu is not None:
        line["cpu_baseline"] = cpu
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def run_serving(n_requests: int = 160, seed: int = 4242, rates=(0.25, 0.5, 0.75)):
    """Serving configuration: 16 resident scenes (~20M triangles), AO bake
    requests with ray counts log-U[4K, 4M] on a uniformly chosen scene, an HBM
    budget of 40 GB for ray/hit buffers.  Reports (1) saturated throughput of
    the continuous-batching server against one request per launch (each
    request: H2D rays, one plain launch, D2H hits, in arrival order), both with
    host pinned buffers, and (2) p50/p99 request latency for Poisson arrivals
    at fractions of the saturated request rate."""
    import threading
    import torch
    import cwbvh_b200 as rq
    from cwbvh_b200 import workloads as W

    rng = np.random.default_rng(seed)
    tris = np.exp(rng.uniform(math.log(300_000), math.log(3_000_000), 16))
    tris = (tris * 20_000_000 / tris.sum()).astype(np.int64)
    spec = [dict(seed=300 + i, tris=int(t), rays=0, small=False) for i, t in enumerate(tris)]
    built = build_scenes(spec)
    pool = 4 * 1024 * 1024
    scenes, host_rays = [], []
    for s, (V, I, hb) in zip(spec, built):
        ds = W.DeviceScene(rq.CWBVH, hb, rq.Scene.from_host(hb), torch.from_numpy(V).cuda(),
                           torch.from_numpy(I).cuda(), W.diag(V), I.shape[0])
        r = W.ao_rays(ds, pool, seed=s["seed"] + 1000)
        hr = torch.empty(r.shape, dtype=torch.float32, pin_memory=True)
        hr.copy_(r)
        scenes.append(ds)
        host_rays.append(hr.numpy())
        del r
    counts = np.exp(rng.uniform(math.log(4096), math.log(4 * 1024 * 1024), n_requests)).astype(np.int64)
    which = rng.integers(0, 16, n_requests)
    total = int(counts.sum())
    hits = torch.empty((total, 4), dtype=torch.float32, pin_memory=True).numpy()
    offs = np.concatenate([[0], np.cumsum(counts)])
    reqs = [(int(which[k]), host_rays[which[k]][:counts[k]], hits[offs[k]:offs[k + 1]]) for k in range(n_requests)]
    torch.cuda.synchronize()

    # (a) one request per launch, in arrival order
    ctx = rq.Context()
    stream = torch.cuda.Stream()
    dev_rays = torch.empty((int(counts.max()), 8), device="cuda")
    dev_hits = torch.empty((int(counts.max()), 4), device="cuda")

    def one_per_launch():
        for sid, hr, hh in reqs:
            n = hr.shape[0]
            with torch.cuda.stream(stream):
                dev_rays[:n].copy_(torch.from_numpy(hr), non_blocking=True)
                rq.trace(ctx, scenes[sid].scene, dev_rays[:n], dev_hits[:n], rq.ANY, stream=stream)
                torch.from_numpy(hh).copy_(dev_hits[:n], non_blocking=True)
        stream.synchronize()

    one_per_launch()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    one_per_launch()
    t_single = time.perf_counter() - t0
    ctx.check(stream)

    # (b) the continuous-batching server, all requests queued at once (saturation)
    srv = rq.Server(hbm_budget_bytes=40 * 10 ** 9, query=rq.ANY, streams=3, max_batch_rays=8 * 1024 * 1024)
    ids = [srv.add_scene(ds.scene) for ds in scenes]

    def burst():
        tickets = [srv.submit(ids[sid], hr, hh) for sid, hr, hh in reqs]
        return [srv.wait(t) for t in tickets]

    burst()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    stats = burst()
    t_served = time.perf_counter() - t0
    sat_rays_per_s = total / t_served
    batches = len({s["batch_id"] for s in stats})

    # (c) Poisson arrivals at fractions of the saturated request rate
    sat_req_rate = n_requests / t_served
    sweep = []
    for frac in rates:
        lam = frac * sat_req_rate
        gaps = np.random.default_rng(seed + int(frac * 1000)).exponential(1.0 / lam, n_requests)
        tickets = [None] * n_requests

        def submitter():
            nxt = time.perf_counter()
            for k, (sid, hr, hh) in enumerate(reqs):
                nxt += gaps[k]
                d = nxt - time.perf_counter()
                if d > 0:
                    time.sleep(d)
                tickets[k] = srv.submit(ids[sid], hr, hh)

        th = threading.Thread(target=submitter)
        t0 = time.perf_counter()
        th.start()
        th.join()
        st = [srv.wait(t) for t in tickets]
        wall = time.perf_counter() - t0
        lat = np.array([s["done_ms"] - s["submit_ms"] for s in st])
        sweep.append({"offered_fraction_of_saturation": frac, "req_per_s": round(lam, 1),
                      "p50_ms": round(float(np.percentile(lat, 50)), 3),
                      "p99_ms": round(float(np.percentile(lat, 99)), 3),
                      "mrays_per_s": round(total / wall / 1e6, 1),
                      "launches": len({s["batch_id"] for s in st})})
    srv.close()
    lat_sat = np.array([s["done_ms"] - s["submit_ms"] for s in stats])

    # (d) the same requests as AO bake requests at the reference's 32 rays per
    # texel: surfels in, AO out, rays generated and counted on the device
    spp = 32
    surf = []
    for ds, s in zip(scenes, spec):
        pos, nrm, rad = rq.sample_surfels(ds.vertices, ds.indices, pool // spp, s["seed"] + 2000)
        hp = [torch.empty(x.shape, dtype=torch.float32, pin_memory=True) for x in (pos, nrm, rad)]
        for h_, d_ in zip(hp, (pos, nrm, rad)):
            h_.copy_(d_)
        surf.append((hp[0].numpy(), hp[1].numpy(), hp[2].numpy(), ds.diag))
    n_surf = np.maximum(counts // spp, 1)
    ao_out = torch.empty(int(n_surf.sum()), dtype=torch.float32, pin_memory=True).numpy()
    aoffs = np.concatenate([[0], np.cumsum(n_surf)])
    bsrv = rq.Server(hbm_budget_bytes=40 * 10 ** 9, query=rq.ANY, streams=3, max_batch_rays=8 * 1024 * 1024)
    bids = [bsrv.add_scene(ds.scene) for ds in scenes]

    def bake_burst():
        tickets = []
        for k in range(n_requests):
            sid, n = int(which[k]), int(n_surf[k])
            p_, n_, r_, dg = surf[sid]
            tickets.append(bsrv.submit_bake(bids[sid], p_[:n], n_[:n], r_[:n], spp, 77 + k, 1e-4 * dg, 0.1 * dg, 0.0,
                                            ao_out[aoffs[k]:aoffs[k + 1]]))
        return [bsrv.wait(t) for t in tickets]

    bake_burst()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    bstats = bake_burst()
    t_bake = time.perf_counter() - t0
    bsrv.close()
    bake_rays = int(n_surf.sum()) * spp
    lat_b = np.array([s["done_ms"] - s["submit_ms"] for s in bstats])
    bake = {"what": "the same 160 requests as AO bake requests: n/32 surfels each, 32 rays per surfel generated on "
                    "the device, occlusion counted per surfel in the trace epilogue; 36 B per surfel in, 4 B out",
            "mrays_per_s": round(bake_rays / t_bake / 1e6, 1), "rays": bake_rays,
            "h2d_bytes": int(n_surf.sum()) * 36, "d2h_bytes": int(n_surf.sum()) * 4,
            "p50_ms": round(float(np.percentile(lat_b, 50)), 3), "p99_ms": round(float(np.percentile(lat_b, 99)), 3),
            "launches": len({s["batch_id"] for s in bstats})}
    return {
        "workload": "16 resident scenes (%.1fM tris), %d AO any-hit bake requests, rays log-U[4K,4M] (%.0fM total), "
                    "HBM budget 40 GB, 3 streams, <= 8M rays per launch, host pinned buffers"
                    % (tris.sum() / 1e6, n_requests, total / 1e6),
        "served_mrays_per_s": round(sat_rays_per_s / 1e6, 1),
        "one_request_per_launch_mrays_per_s": round(total / t_single / 1e6, 1),
        "served_vs_one_per_launch": round(t_single / t_served, 3),
        "saturated": {"p50_ms": round(float(np.percentile(lat_sat, 50)), 3),
                      "p99_ms": round(float(np.percentile(lat_sat, 99)), 3), "launches": batches},
        "poisson": sweep,
        "bake_requests_saturated": bake,
        "timing": "host wall clock with the device idle on both sides (the server spans three streams)",
    }


def run_ref_gpu(scenes, rays, warmup: int, steps: int, kind: int = 0):
    """The reference's rtTraceCWBVH (kind 0) or rtTraceBVH2 (kind 1)
    (oracle/_ref, compiled from its sources for sm_100a, shipped grids) on the
    same scenes and rays."""
    import torch
    try:
        from oracle import pyoracle as po
        if not po.ref_available():
            return {"unavailable": "oracle/_ref/libref.so not built"}, None
        lib = po.ref()
    except Exception as e:  # pragma: no cover
        return {"unavailable": str(e)}, None
    # The reference kernel has a 40-entry stack without an overflow check; a
    # tree of depth d needs at most 2d entries.
    # The BVH2 kernel's stack holds 32 entries (a tree of depth d needs d).
    deepest = max(ds.host.info["depth"] for ds in scenes)
    if kind == 0 and 2 * deepest > 40:
        return {"unavailable": f"tree depth {deepest} could overflow the reference's 40-entry stack"}, None
    if kind == 1 and deepest > 31:
        return {"unavailable": f"tree depth {deepest} could overflow the reference's 32-entry stack"}, None
    bind, trace = (lib.ref_bind_cwbvh, lib.ref_trace_cwbvh) if kind == 0 else (lib.ref_bind_bvh2, lib.ref_trace_bvh2)
    tag = "rtTraceCWBVH" if kind == 0 else "rtTraceBVH2"
    import re
    import tempfile
    out_hits = [torch.empty((r.shape[0], 4), device="cuda") for r in rays]
    total = sum(r.shape[0] for r in rays)
    sys.stdout.flush()
    tmp = tempfile.TemporaryFile(mode="w+b")
    saved = os.dup(1)
    try:
        os.dup2(tmp.fileno(), 1)  # rtTraceCWBVH logs its own event-timed duration per call

        def step():
            for ds, r, h in zip(scenes, rays, out_hits):
                dn, dw, dp = C_buffers(ds.scene)
                bind(dn, dw, dp)
                trace(r.data_ptr(), h.data_ptr(), r.shape[0])
        for _ in range(warmup):
            step()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(steps):
            step()
        torch.cuda.synchronize()
        wall_ms = (time.perf_counter() - t0) * 1e3 / steps
    finally:
        os.dup2(saved, 1)
        os.close(saved)
    tmp.seek(0)
    txt = tmp.read().decode(errors="replace")
    tmp.close()
    per_call = [float(m) for m in re.findall(r"([0-9.]+)MS, [0-9.]+MRays/s \(" + tag, txt)]
    timed = per_call[len(per_call) - steps * len(rays):] if len(per_call) >= steps * len(rays) else []
    ms = sum(timed) / steps if timed else wall_ms
    out = {"value": round(total / (ms * 1e-3) / 1e6, 2), "unit": "Mrays/s", "ms_per_step": round(ms, 3),
           "wall_ms_per_step": round(wall_ms, 3),
           "query": "closest-hit (the reference has no any-hit kernel)",
           "timing": f"sum of the reference's own CUDA-event kernel times (its log line per {tag} call)"
           if timed else f"host wall clock around synchronous {tag} calls",
           "grid": "as shipped (CWBVH: 32x32 blocks of 32x2 threads; BVH2: one 128-thread block per 128 rays)"}
    if kind == 0:
        out["occupancy_filling_grid"] = ref_cwbvh_full_grid(lib, scenes, rays, warmup, steps, total)
    return out, [h for h in out_hits]


def ref_cwbvh_full_grid(lib, scenes, rays, warmup: int, steps: int, total: int) -> dict:
    """The reference's own CWBVH kernel, unmodified, launched with as many
    32x2-thread blocks as are resident at once on the device instead of its
    shipped 32x32 grid (oracle/ref_harness.cu, ref_trace_cwbvh_grid), timed
    with CUDA events on the legacy default stream it runs on: what the
    reference's kernel does on a grid that fills a B200."""
    import ctypes as C
    import torch
    counter = torch.zeros(1, dtype=torch.int32, device="cuda")
    hits = [torch.empty((r.shape[0], 4), device="cuda") for r in rays]
    used = C.c_int(0)

    def step():
        for ds, r, h in zip(scenes, rays, hits):
            dn, dw, dp = C_buffers(ds.scene)
            lib.ref_bind_cwbvh(dn, dw, dp)
            err = lib.ref_trace_cwbvh_grid(r.data_ptr(), h.data_ptr(), r.shape[0], 0, counter.data_ptr(),
                                           C.byref(used))
            if err:
                raise RuntimeError(f"ref_trace_cwbvh_grid: CUDA error {err}")
    stream = torch.cuda.default_stream()
    for _ in range(warmup):
        step()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    return {"value": round(total / (ms * 1e-3) / 1e6, 2), "unit": "Mrays/s", "ms_per_step": round(ms, 3),
            "blocks": int(used.value), "grid": f"{used.value} blocks of 32x2 threads ({used.value / sms:.0f} per SM, "
                                              "all resident at once); shipped: 1024 blocks",
            "timing": "CUDA events around the launches (scene binds included)"}


def C_buffers(scene):
    import ctypes as C
    import cwbvh_b200 as rq
    n, w, p = C.c_void_p(), C.c_void_p(), C.c_void_p()
    rq.check(rq.lib.rq_scene_device_buffers(scene._h, C.byref(n), C.byref(w), C.byref(p)), "rq_scene_device_buffers")
    return n, w, p


def cpu_baseline(spec, built):
    try:
        from oracle import pyoracle as po
        threads = po.oracle().oracle_max_threads()
    except Exception as e:
        return {"unavailable": str(e)}
    sample = cpu_sample(spec, built, target_rays=1 << 21)
    time_cpu(sample[:2], threads)  # warm
    dt, n = time_cpu(sample, threads)
    if dt < 10.0:  # aim for >= 10 s of CPU work
        reps = int(math.ceil(10.0 / max(dt, 1e-3)))
        dt = 0.0
        for _ in range(reps):
            d, _ = time_cpu(sample, threads)
            dt += d
        n *= reps
    return {"value": round(n / dt / 1e6, 3), "unit": "Mrays/s", "cores": threads, "kind": "port",
            "sample": f"{n} AO any-hit rays drawn from all scenes in proportion to their ray counts, CWBVH, "
                      f"oracle/oracle.c with OpenMP over {threads} threads, {dt:.1f}s"}


def run_small_kernels(args, built, scenes, rays, stream, ctx, dist, warmup, flush):
    """Plain launches of both kernel families on the plain config's scene and
    rays (CWBVH and BVH2, any-hit and closest-hit), and the reference's BVH2
    kernel (closest-hit) on the same rays."""
    import torch
    import cwbvh_b200 as rq
    from cwbvh_b200 import workloads as W
    V, I, _ = built[0]
    r = rays[0]
    hb2 = rq.HostBVH(V, I, rq.BVH2)
    with torch.cuda.stream(stream):
        sc2 = rq.Scene.from_host(hb2)
        h = torch.empty((r.shape[0], 4), device="cuda")
    out = {}
    for sc, nm in ((scenes[0].scene, "cwbvh"), (sc2, "bvh2")):
        for q, qn in ((rq.ANY, "any"), (rq.CLOSEST, "closest")):
            ms = time_steps(lambda: rq.trace(ctx, sc, r, h, q, stream=stream), args.steps, warmup, stream, dist,
                            flush)
            out[f"{nm}_{qn}"] = {"mrays_per_s": round(r.shape[0] / (ms * 1e-3) / 1e6, 2), "ms": round(ms, 4)}
    ctx.check(stream)
    if not args.no_ref_gpu:
        ds2 = W.DeviceScene(rq.BVH2, hb2, sc2, None, None, W.diag(V), I.shape[0])
        out["reference_bvh2_kernel_sm100a"], _ = run_ref_gpu([ds2], [r], 1, 3, kind=1)
    return out


def _counted_bytes(ctx, scene, rays, query, stream):
    """Algorithmic bytes of one CWBVH pass: 32 + 16 per ray, 80 per node
    fetched, 48 per triangle tested (counts from rq_trace_counted)."""
    import torch
    import cwbvh_b200 as rq
    with torch.cuda.stream(stream):
        hh = torch.empty((rays.shape[0], 4), device="cuda")
        nv, nt = rq.trace_counted(ctx, scene, rays, hh, query, stream=stream)
        nodes = int(nv.sum(dtype=torch.int64).item())
        tris = int(nt.sum(dtype=torch.int64).item())
        del hh, nv, nt
    return 48 * int(rays.shape[0]) + 80 * nodes + 48 * tris, nodes, tris


def batching_breakdown(ctx, scenes, rays, hits, ms_batch: float, stream, warmup: int) -> dict:
    """Each scene's plain launch timed alone (CUDA events) against the time
    its rays take at the batch's overall rate; the difference is that
    launch's tail (its last waves running with the GPU partly idle) plus its
    launch overhead -- all that one persistent launch over every item can
    remove.  Summed per quartile of the scenes' ray counts."""
    import cwbvh_b200 as rq
    total = sum(int(r.shape[0]) for r in rays)
    rate = total / ms_batch  # rays per ms in the batch
    rows = []
    for ds, r, h in zip(scenes, rays, hits):
        ms = time_steps(lambda: rq.trace(ctx, ds.scene, r, h, rq.ANY, stream=stream), 3, 1, stream)
        rows.append((int(r.shape[0]), ds.n_tris, ms, ms - r.shape[0] / rate))
    ctx.check(stream)
    rows.sort()
    q = []
    for k in range(4):
        part = rows[k * len(rows) // 4:(k + 1) * len(rows) // 4]
        q.append({"scenes": len(part), "rays": [part[0][0], part[-1][0]],
                  "triangles_mean": int(np.mean([p[1] for p in part])),
                  "plain_ms": round(sum(p[2] for p in part), 3),
                  "at_batch_rate_ms": round(sum(p[0] for p in part) / rate, 3),
                  "tail_ms_per_launch": round(float(np.mean([p[3] for p in part])), 4)})
    return {"per_quartile_of_rays": q, "plain_sum_ms": round(sum(p[2] for p in rows), 3),
            "batched_ms": round(ms_batch, 3),
            "tail_ms_per_launch_mean": round(float(np.mean([p[3] for p in rows])), 4),
            "what": "each scene's plain launch timed alone vs its rays at the batch's rate; the difference is the "
                    "launch's tail and overhead, which one persistent launch removes"}


def batching_small_items(ctx, stream, warmup: int, steps: int, n_items: int = 64, n_rays: int = 256 * 1024) -> dict:
    """Batching where it has most to remove: 64 small scenes (10k-20k
    triangles, the low end of the batched configuration) with 256K AO rays
    each, as 64 plain launches and as one batch launch (CUDA graph)."""
    import torch
    import cwbvh_b200 as rq
    from cwbvh_b200 import workloads as W
    rng = np.random.default_rng(99)
    tris = np.exp(rng.uniform(math.log(10_000), math.log(20_000), n_items)).astype(np.int64)
    items, keep = [], []
    for k, t in enumerate(tris):
        V, I = W.scene_of_size(500 + k, int(t))
        ds = W.upload(V, I, rq.CWBVH)
        r = W.ao_rays(ds, n_rays, seed=600 + k, stream=stream)
        h = torch.empty((n_rays, 4), device="cuda")
        items.append((ds.scene, r, h))
        keep.append(ds)
    torch.cuda.synchronize()

    def plain():
        for sc, r, h in items:
            rq.trace(ctx, sc, r, h, rq.ANY, stream=stream)
    ms_plain = time_steps(plain, steps, warmup, stream)
    occ_plain = [int(h[:, 1].view(torch.int32).ne(-1).sum().item()) for _, _, h in items]
    b = rq.Batch(ctx, items, rq.ANY, sort_threshold=-1, use_graph=True)
    ms_batch = time_steps(lambda: b.run(stream), steps, warmup, stream)
    ctx.check(stream)
    occ_batch = [int(h[:, 1].view(torch.int32).ne(-1).sum().item()) for _, _, h in items]
    b.close()
    total = n_items * n_rays
    return {"scenes": n_items, "triangles": [int(tris.min()), int(tris.max())], "rays_per_scene": n_rays,
            "plain_mrays_per_s": round(total / ms_plain / 1e3, 1), "batched_mrays_per_s": round(total / ms_batch / 1e3, 1),
            "batched_vs_plain": round(ms_plain / ms_batch, 3), "occlusion_identical": occ_plain == occ_batch}


def run_config_process(workload: str, args, warmup: int, timeout_s: int = 900) -> dict:
    """One configuration's bench line from `bench.py --workload <workload>`
    in a child process on the same GPU (no CPU baseline there: the CPU figure
    is the default line's), minus the keys the parent line already carries."""
    cmd = [sys.executable, str(ROOT / "bench.py"), "--workload", workload, "--steps", str(args.steps),
           "--warmup", str(warmup), "--no-cpu"]
    if args.no_ref_gpu:
        cmd.append("--no-ref-gpu")
    env = dict(os.environ)
    for k in ("RANK", "LOCAL_RANK", "WORLD_SIZE", "LOCAL_WORLD_SIZE"):
        env.pop(k, None)
    try:
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout_s, env=env, cwd=str(ROOT))
    except subprocess.TimeoutExpired:
        return {"unavailable": f"bench.py --workload {workload} exceeded {timeout_s}s"}
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    if r.returncode != 0 or not lines:
        tail = (r.stderr or "").strip().splitlines()[-1:] or ["no output"]
        return {"unavailable": f"bench.py --workload {workload} exited {r.returncode}: {tail[0][:300]}"}
    d = json.loads(lines[-1])
    for k in ("metric", "n_gpus", "higher_is_better", "scaling", "vs_baseline", "data", "dtype", "steps", "warmup"):
        d.pop(k, None)
    d["command"] = " ".join(["python", "bench.py"] + cmd[2:])
    return d


def _pass(name, n_rays, ms, alg=None, peak=None, l2=None):
    d = {"rays": int(n_rays), "ms": round(ms, 4), "mrays_per_s": round(n_rays / (ms * 1e-3) / 1e6, 2)}
    if alg is not None:
        b, nodes, tris = alg
        gbs = b / (ms * 1e-3) / 1e9
        d.update({"bytes_per_ray": round(b / n_rays, 1), "nodes_per_ray": round(nodes / n_rays, 3),
                  "tris_per_ray": round(tris / n_rays, 3), "achieved_gbs": round(gbs, 1)})
        if peak:
            d["hbm_frac"] = round(gbs / peak, 4)
        if l2:
            d["l2_frac"] = round(gbs / l2, 4)
    return d


def _single_line(args, world, warmup, workload: str, value: float, ms: float, extra: dict):
    line = {"metric": METRIC, "value": round(value, 2), "unit": "Mrays/s", "n_gpus": world, "steps": args.steps,
            "warmup": warmup, "ms_per_step": round(ms, 4), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded procedural scene; the reference's mesh.dat/samplecache.dat are not shipped)",
            "config": {"workload": workload, "l2": "inputs larger than L2",
                       "parallelism": f"replicas x{world} (rays independent, no data-path collective)"}}
    line.update(extra)
    return line


def run_city(args, world, rank, dist):
    """Single mid-size scene: a 1M-triangle city (10k box/prism buildings,
    log-normal heights, ground grid), 4096x4096 pinhole primary rays
    closest-hit, then one AO any-hit ray per primary hit (tmax = 0.05 diag).
    The passes are reported separately and combined."""
    import torch
    import cwbvh_b200 as rq
    from cwbvh_b200 import workloads as W
    warmup = max(3, args.warmup)
    t0 = time.time()
    V, I = rq.gen_city(rank, 10000)
    hb = rq.HostBVH(V, I, rq.CWBVH)
    log(f"[bench] city {I.shape[0]/1e6:.2f}M tris built in {time.time()-t0:.1f}s")
    stream = torch.cuda.Stream()
    ctx = rq.Context()
    with torch.cuda.stream(stream):
        sc = rq.Scene.from_host(hb)
    dg = W.diag(V)
    lo, hi = V.min(0), V.max(0)
    ext = hi - lo
    eye = (float(lo[0] - 0.05 * ext[0]), float(lo[1] - 0.05 * ext[1]), float(0.25 * max(ext[0], ext[1])))
    look = (float(0.5 * (lo[0] + hi[0])), float(0.5 * (lo[1] + hi[1])), 0.0)
    w = h = 2048 if args.quick else 4096
    n = w * h
    prim = rq.camera_rays(eye, look, (0.0, 0.0, 1.0), 60.0, w, h, 0.0, 10.0 * dg, stream=stream, tile=(4, 8))
    with torch.cuda.stream(stream):
        ph = torch.empty((n, 4), device="cuda")
    ms_prim = time_steps(lambda: rq.trace(ctx, sc, prim, ph, rq.CLOSEST, stream=stream), args.steps, warmup,
                         stream, dist)
    out = {}

    def gen():
        pos, nrm, rad = rq.surfels_from_hits(prim, ph, sc, stream=stream)
        out["ao"] = rq.aorays(pos, nrm, rad, 1, seed=rank + 77, tmin=1e-4 * dg, tmax=0.05 * dg, offset_scale=0.0,
                              stream=stream)
    ms_gen = time_steps(gen, args.steps, warmup, stream, dist)
    ao = out["ao"]
    with torch.cuda.stream(stream):
        ah = torch.empty((n, 4), device="cuda")
    ms_ao = time_steps(lambda: rq.trace(ctx, sc, ao, ah, rq.ANY, stream=stream), args.steps, warmup, stream, dist)
    # the same AO rays Morton-sorted inside a one-item batch (sort + trace + scatter of hits)
    sah = torch.empty((n, 4), device="cuda")
    sb = rq.Batch(ctx, [(sc, ao, sah)], rq.ANY, sort_threshold=0, use_graph=True)
    ms_ao_sorted = time_steps(lambda: sb.run(stream), args.steps, warmup, stream, dist)
    ctx.check(stream)
    torch.cuda.synchronize()
    hit_frac = float((ph[:, 1].view(torch.int32) >= 0).float().mean().item())
    occ = float((ah[:, 1].view(torch.int32) != -1).float().mean().item())
    same = bool(torch.equal(ah[:, 1].view(torch.int32) != -1, sah[:, 1].view(torch.int32) != -1))
    peak, peak_kind = measured_peak_hbm()
    l2 = measure_l2_read(stream)["peak"]
    a_prim = _counted_bytes(ctx, sc, prim, rq.CLOSEST, stream)
    a_ao = _counted_bytes(ctx, sc, ao, rq.ANY, stream)
    ref = {}
    if not args.no_ref_gpu:
        ref, ref_hits = run_ref_gpu([W.DeviceScene(rq.CWBVH, hb, sc, None, None, dg, I.shape[0])], [prim], 1, 2)
        if ref_hits:
            mine = ph[:, 1].view(torch.int32)
            theirs = ref_hits[0][:, 1].view(torch.int32)
            pm = torch.from_numpy(hb.prim_index).cuda()
            n_pm = pm.numel()
            pid = lambda a: torch.where((a >= 0) & (a < n_pm), pm[a.clamp(0, n_pm - 1).long()],  # noqa: E731
                                        torch.full_like(a, -1))
            ref["closest_prim_ids_equal_frac"] = round(float((pid(mine) == pid(theirs)).float().mean().item()), 6)
    total = 2 * n
    ms_total = ms_prim + ms_gen + ms_ao
    extra = {
        "passes": {"primary_closest": _pass("primary", n, ms_prim, a_prim, peak, l2),
                   "ao_raygen": {"ms": round(ms_gen, 4), "what": "surfels_from_hits + aorays (1 spp)"},
                   "ao_any": _pass("ao", n, ms_ao, a_ao, peak, l2),
                   "ao_any_morton_sorted": _pass("ao_sorted", n, ms_ao_sorted)},
        "primary_hit_fraction": round(hit_frac, 4), "ao_occluded_fraction": round(occ, 4),
        "ao_sorted_occlusion_identical": same,
        "triangles": int(I.shape[0]), "image": f"{w}x{h}",
        "roofline": {"bound": "hbm", "achieved": _pass("", n, ms_ao, a_ao)["achieved_gbs"], "peak": peak,
                     "unit": "GB/s", "frac": _pass("", n, ms_ao, a_ao, peak)["hbm_frac"],
                     "peak_source": f"hbm_gbs of {peak_kind}", "traffic": None,
                     "l2": {"peak": round(l2, 1), "frac": _pass("", n, ms_ao, a_ao, None, l2)["l2_frac"]},
                     "kernel": "AO any-hit pass"},
    }
    if ref:
        extra["reference_cwbvh_kernel_sm100a_primary"] = ref
    line = _single_line(args, world, warmup, f"city: {I.shape[0]/1e6:.2f}M tris, {w}x{h} primary closest-hit "
                        "(camera rays in 4x8-pixel tiles) + 1 AO any-hit ray per primary hit (tmax 0.05 diag); "
                        "value = both passes + raygen",
                        world * total / (ms_total * 1e-3) / 1e6, ms_total, extra)
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_instanced(args, world, rank, dist):
    """Two-level city: 64 block templates (16 buildings each, from the city
    generator) placed 625 times on a 25 x 25 grid with quarter-turn rotations
    (10,000 buildings) under a top-level CWBVH, against the same city
    flattened into one mesh: 4096x4096 primary closest-hit and one AO any-hit
    ray per primary hit through both."""
    import torch
    import cwbvh_b200 as rq
    from cwbvh_b200 import workloads as W
    warmup = max(3, args.warmup)
    rng = np.random.default_rng(77 + rank)
    templates = [rq.gen_city(1000 + i, 16) for i in range(64)]
    blas = [rq.HostBVH(V, I, rq.CWBVH) for V, I in templates]
    side, block = 25, 80.0
    n_inst = side * side
    bi = rng.integers(0, len(templates), n_inst).astype(np.int32)
    M = np.zeros((n_inst, 3, 4), np.float32)
    Vs, Is, nv = [], [], 0
    for k in range(n_inst):
        r = int(rng.integers(0, 4))
        c, s_ = [(1, 0), (0, 1), (-1, 0), (0, -1)][r]
        R = np.array([[c, -s_, 0], [s_, c, 0], [0, 0, 1]], np.float64)
        ctr = np.array([block / 2, block / 2, 0.0])
        off = np.array([(k % side) * block, (k // side) * block, 0.0])
        M[k, :, :3] = R
        M[k, :, 3] = off + ctr - R @ ctr
        V, I = templates[bi[k]]
        Vs.append((V.astype(np.float64) @ R.T + M[k, :, 3].astype(np.float64)).astype(np.float32))
        Is.append(I + nv)
        nv += V.shape[0]
    FV, FI = np.concatenate(Vs), np.concatenate(Is).astype(np.int32)
    t0 = time.time()
    fhb = rq.HostBVH(FV, FI, rq.CWBVH)
    log(f"[bench] instanced city: {n_inst} instances of {len(templates)} blocks; flat {FI.shape[0]/1e6:.2f}M tris "
        f"built in {time.time()-t0:.1f}s")
    stream = torch.cuda.Stream()
    ctx = rq.Context()
    with torch.cuda.stream(stream):
        scenes = [rq.Scene.from_host(h) for h in blas]
        flat = rq.Scene.from_host(fhb)
    tlas = rq.Tlas(scenes, M, bi)
    top = tlas.buffers()
    inst_bytes = sum(h.nodes.nbytes + h.woop.nbytes for h in blas) + top["nodes"].nbytes + top["rows"].nbytes
    flat_bytes = fhb.nodes.nbytes + fhb.woop.nbytes
    dg = W.diag(FV)
    lo, hi = FV.min(0), FV.max(0)
    ext = hi - lo
    eye = (float(lo[0] - 0.05 * ext[0]), float(lo[1] - 0.05 * ext[1]), float(0.25 * max(ext[0], ext[1])))
    look = (float(0.5 * (lo[0] + hi[0])), float(0.5 * (lo[1] + hi[1])), 0.0)
    w = h = 2048 if args.quick else 4096
    n = w * h
    prim = rq.camera_rays(eye, look, (0.0, 0.0, 1.0), 60.0, w, h, 0.0, 10.0 * dg, stream=stream, tile=(4, 8))
    with torch.cuda.stream(stream):
        fh = torch.empty((n, 4), device="cuda")
        ih = torch.empty((n, 4), device="cuda")
        ii = torch.empty(n, dtype=torch.int32, device="cuda")
    ms_flat_p = time_steps(lambda: rq.trace(ctx, flat, prim, fh, rq.CLOSEST, stream=stream), args.steps, warmup,
                           stream, dist)
    ms_inst_p = time_steps(lambda: rq.trace_instanced(ctx, tlas, prim, ih, rq.CLOSEST, ii, stream=stream),
                           args.steps, warmup, stream, dist)
    pos, nrm, rad = rq.surfels_from_hits(prim, fh, flat, stream=stream)
    ao = rq.aorays(pos, nrm, rad, 1, seed=rank + 78, tmin=1e-4 * dg, tmax=0.05 * dg, offset_scale=0.0, stream=stream)
    with torch.cuda.stream(stream):
        fa = torch.empty((n, 4), device="cuda")
        ia = torch.empty((n, 4), device="cuda")
    ms_flat_a = time_steps(lambda: rq.trace(ctx, flat, ao, fa, rq.ANY, stream=stream), args.steps, warmup, stream,
                           dist)
    ms_inst_a = time_steps(lambda: rq.trace_instanced(ctx, tlas, ao, ia, rq.ANY, None, stream=stream), args.steps,
                           warmup, stream, dist)
    ctx.check(stream)
    torch.cuda.synchronize()
    fhit = fh[:, 1].view(torch.int32) >= 0
    ihit = ih[:, 1].view(torch.int32) >= 0
    tdiff = (fh[:, 0] - ih[:, 0]).abs() / fh[:, 0].abs().clamp(min=1e-30)
    both = fhit & ihit
    occ_same = float(((fa[:, 1].view(torch.int32) != -1) == (ia[:, 1].view(torch.int32) != -1)).float().mean())
    total_ms = ms_inst_p + ms_inst_a
    extra = {
        "passes": {"primary_closest": {"instanced": _pass("", n, ms_inst_p), "flattened": _pass("", n, ms_flat_p)},
                   "ao_any": {"instanced": _pass("", n, ms_inst_a), "flattened": _pass("", n, ms_flat_a)}},
        "agreement": {"primary_hit_same_frac": round(float((fhit == ihit).float().mean()), 6),
                      "primary_t_rel_p999": round(float(tdiff[both].float().kthvalue(
                          max(1, int(0.999 * int(both.sum())))).values), 8),
                      "ao_occlusion_same_frac": round(occ_same, 6)},
        "scene_bytes": {"instanced": int(inst_bytes), "flattened": int(flat_bytes)},
        "instances": n_inst, "templates": len(templates), "flat_triangles": int(FI.shape[0]), "image": f"{w}x{h}",
    }
    line = _single_line(args, world, warmup, f"instanced city: {n_inst} instances of {len(templates)} 16-building "
                        f"blocks ({FI.shape[0]/1e6:.2f}M tris flattened), {w}x{h} primary closest-hit (4x8-pixel tiles) "
                        "+ 1 AO any-hit ray per pixel; value = both instanced passes", world * 2 * n / (total_ms * 1e-3) / 1e6,
                        total_ms, extra)
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_large(args, world, rank, dist):
    """Single large scene: displaced subdivided spheres + terrain tiles
    (30M triangles; 3M with --quick), 16M surfels x 4 spp = 64M incoherent
    AO any-hit rays (tmin 1e-4 diag, tmax 0.1 diag), unsorted vs
    Morton-sorted; the scene is far larger than L2, so node fetches go to HBM."""
    import torch
    import cwbvh_b200 as rq
    from cwbvh_b200 import workloads as W
    warmup = max(3, args.warmup)
    n_tris = 3_000_000 if args.quick else 30_000_000
    n_surf = (1 << 22) if args.quick else (1 << 24)
    if args.rays:
        n_surf = max(1, args.rays // 4)
    spp = 4
    V, I = rq.gen_spheres_terrain(rank, n_tris)
    t0 = time.time()
    hb = rq.HostBVH(V, I, rq.CWBVH)
    t_host_build = time.time() - t0
    log(f"[bench] large {I.shape[0]/1e6:.1f}M tris built in {time.time()-t0:.1f}s "
        f"(nodes {hb.nodes.nbytes/1e9:.2f} GB, woop {hb.woop.nbytes/1e9:.2f} GB)")
    stream = torch.cuda.Stream()
    ctx = rq.Context()
    with torch.cuda.stream(stream):
        sc = rq.Scene.from_host(hb)
        v = torch.from_numpy(V).cuda()
        i = torch.from_numpy(I).cuda()
        pos, nrm, rad = rq.sample_surfels(v, i, n_surf, seed=rank + 1000, stream=stream)
        dg = W.diag(V)
        rays = rq.aorays(pos, nrm, rad, spp, seed=rank + 2000, tmin=1e-4 * dg, tmax=0.1 * dg, offset_scale=0.0,
                         stream=stream)
        del pos, nrm, rad
        n = rays.shape[0]
        hits = torch.empty((n, 4), device="cuda")
        shits = torch.empty((n, 4), device="cuda")
    if args.profile:  # profiler captures: only the unsorted trace, W + K launches
        for _ in range(warmup + args.steps):
            rq.trace(ctx, sc, rays, hits, rq.ANY, stream=stream)
        torch.cuda.synchronize()
        ctx.check(stream)
        log(f"[bench] profile mode: {warmup + args.steps} traces of {n} rays")
        return
    ms_plain = time_steps(lambda: rq.trace(ctx, sc, rays, hits, rq.ANY, stream=stream), args.steps, warmup, stream,
                          dist)
    # the same mesh built on the GPU (linear BVH, then 0 or 2 treelet passes, collapsed to CWBVH)
    gpu_trees = {}
    with torch.cuda.stream(stream):
        ghits = torch.empty((n, 4), device="cuda")
    for method, passes in ((rq.GPU_BUILD_LBVH, 0), (rq.GPU_BUILD_LBVH, 2), (rq.GPU_BUILD_PLOC, 0),
                           (rq.GPU_BUILD_PLOC, 2)):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        gsc = rq.Scene.build_gpu(v, i, optimize_passes=passes, method=method, stream=stream)
        torch.cuda.synchronize()
        t_gpu_build = time.perf_counter() - t0
        ms_gpu_tree = time_steps(lambda: rq.trace(ctx, gsc, rays, ghits, rq.ANY, stream=stream), args.steps, warmup,
                                 stream, dist)
        ctx.check(stream)
        torch.cuda.synchronize()
        same = float(((ghits[:, 1].view(torch.int32) != -1) == (hits[:, 1].view(torch.int32) != -1)).float().mean())
        tag = "lbvh" if method == rq.GPU_BUILD_LBVH else "ploc"
        gpu_trees[f"{tag}_treelet_passes_{passes}"] = {"build_s": round(t_gpu_build, 3),
                                                 "mrays_per_s": round(n / (ms_gpu_tree * 1e-3) / 1e6, 2),
                                                 "occlusion_same_frac": round(same, 6)}
        del gsc
    del v, i, ghits
    with torch.cuda.stream(stream):
        occl = torch.zeros(n // spp, dtype=torch.int32, device="cuda")

    def fused():
        occl.zero_()
        rq.trace_ao(ctx, sc, rays, spp, occluded=occl, stream=stream)
    with torch.cuda.stream(stream):
        ms_fused = time_steps(fused, args.steps, warmup, stream, dist)
    sb = rq.Batch(ctx, [(sc, rays, shits)], rq.ANY, sort_threshold=0, use_graph=True)
    ms_sorted = time_steps(lambda: sb.run(stream), args.steps, warmup, stream, dist)
    ms_sort = time_steps(lambda: rq.lib.rq_batch_run_stage(sb._h, 1, stream.cuda_stream), 3, 1, stream, dist)
    ms_sorted_kernel = time_steps(lambda: rq.lib.rq_batch_run_stage(sb._h, 2, stream.cuda_stream), args.steps,
                                  warmup, stream, dist)
    ctx.check(stream)
    torch.cuda.synchronize()
    same = bool(torch.equal(hits[:, 1].view(torch.int32) != -1, shits[:, 1].view(torch.int32) != -1))
    occ = float((hits[:, 1].view(torch.int32) != -1).float().mean().item())
    fused_same = bool(torch.equal(occl, (hits[:, 1].view(torch.int32) != -1).view(-1, spp).sum(1, dtype=torch.int32)))
    peak, peak_kind = measured_peak_hbm()
    l2 = measure_l2_read(stream)["peak"]
    alg = _counted_bytes(ctx, sc, rays, rq.ANY, stream)
    unsorted = _pass("unsorted", n, ms_plain, alg, peak, l2)
    best = min(ms_plain, ms_sorted, ms_fused)
    extra = {
        "passes": {"unsorted": unsorted,
                   "morton_sorted": dict(_pass("sorted", n, ms_sorted), sort_ms=round(ms_sort, 4),
                                         trace_kernel_ms=round(ms_sorted_kernel, 4)),
                   "fused_ao_counts": dict(_pass("fused", n, ms_fused),
                                           what="rq_trace_ao: per-surfel occluded counts in the trace epilogue, "
                                                "no hit buffer (memset of the counts included)")},
        "gpu_built_tree": dict(gpu_trees, host_build_s=round(t_host_build, 2),
                               what="rq_build_scene_gpu: Morton-ordered radix tree (lbvh) or locally-ordered "
                                    "clustering (ploc), treelet restructuring passes, collapsed to CWBVH on the "
                                    "device"),
        "sorted_occlusion_identical": same, "fused_counts_identical": fused_same,
        "ao_occluded_fraction": round(occ, 4),
        "triangles": int(I.shape[0]), "scene_bytes": int(hb.nodes.nbytes + hb.woop.nbytes),
        "roofline": {"bound": "hbm", "achieved": unsorted["achieved_gbs"], "peak": peak, "unit": "GB/s",
                     "frac": unsorted["hbm_frac"], "peak_source": f"hbm_gbs of {peak_kind}",
                     "traffic": (profile_traffic("large" + ("_quick" if args.quick else "")) or {}).get(
                         "dram_bytes_per_launch"),
                     "l2": {"peak": round(l2, 1), "frac": unsorted["l2_frac"]},
                     "issue": issue_roofline("large" + ("_quick" if args.quick else ""), n / (ms_plain * 1e-3), None),
                     "kernel": "unsorted AO any-hit trace"},
    }
    line = _single_line(args, world, warmup, f"large: {I.shape[0]/1e6:.1f}M tris, {n_surf} surfels x {spp} spp "
                        "AO any-hit, unsorted vs Morton-sorted vs fused AO counts; value = the fastest", world * n / (best * 1e-3) / 1e6,
                        best, extra)
    if rank == 0:
        print(json.dumps(line), flush=True)


def dump_reference_inputs(args, path: str) -> None:
    """Writes the reference arm's inputs -- each scene's CWBVH node and Woop
    buffers and the bounded ray sample -- to an .npz, so that the arm's own
    process times the CPU traversal without loading librq."""
    spec = workload_spec(args.workload, args.quick, 0)
    built = build_scenes(spec)
    sample = cpu_sample(spec, built, target_rays=1 << 20)
    arrays = {}
    for k, (hb, rays) in enumerate(sample):
        arrays[f"nodes{k}"] = np.ascontiguousarray(hb.nodes)
        arrays[f"woop{k}"] = np.ascontiguousarray(hb.woop)
        arrays[f"rays{k}"] = rays
    np.savez(path, n=len(sample), triangles=sum(s["tris"] for s in spec),
             rays_total=sum(s["rays"] for s in spec), **arrays)


def run_reference(args, world, rank, warmup):
    """Reference arm: the reference has no CPU traversal, so its path is timed
    through the C restatement (oracle/oracle.c, kind "port") on the host cores,
    each step a bounded sample of the same workload.  The scenes are built and
    the sample drawn by a child process (which loads librq); this process only
    loads the restatement."""
    if rank != 0:
        return
    import tempfile
    import types
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "ref_inputs.npz")
        cmd = [sys.executable, str(ROOT / "bench.py"), "--workload", args.workload, "--dump-reference-inputs", path]
        if args.quick:
            cmd.append("--quick")
        env = dict(os.environ)
        for k in ("RANK", "LOCAL_RANK", "WORLD_SIZE", "LOCAL_WORLD_SIZE"):
            env.pop(k, None)
        subprocess.run(cmd, check=True, env=env, cwd=str(ROOT))
        z = np.load(path)
        sample = [(types.SimpleNamespace(nodes=z[f"nodes{k}"], woop=z[f"woop{k}"]), z[f"rays{k}"])
                  for k in range(int(z["n"]))]
        tris, rays_total = int(z["triangles"]), int(z["rays_total"])
    from oracle import pyoracle as po
    threads = po.oracle().oracle_max_threads()
    for _ in range(min(warmup, 1)):
        time_cpu(sample, threads)
    dt, n = 0.0, 0
    for _ in range(args.steps):
        d, k = time_cpu(sample, threads)
        dt += d
        n += k
    value = n / dt / 1e6
    workload = BATCHED_WORKLOAD if args.workload == "batched" and not args.quick else \
        f"{args.workload}{' (quick)' if args.quick else ''}"
    line = {
        "metric": METRIC, "value": round(value, 3), "unit": "Mrays/s", "n_gpus": 1, "steps": args.steps,
        "warmup": warmup, "ms_per_step": round(dt / args.steps * 1e3, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": workload, "triangles": tris, "rays_per_gpu": rays_total, "query": "any-hit",
                   "sample_per_step": f"{n // args.steps} rays drawn from all scenes in proportion to their ray "
                                      "counts (a bounded sample of the workload)"},
        "impl": "reference",
        "cpu_baseline": {"value": round(value, 3), "unit": "Mrays/s", "cores": threads, "kind": "port",
                         "sample": f"{n // args.steps} rays per step from all scenes; the reference has no CPU "
                                   f"traversal, its CWBVH algorithm restated in C (oracle/oracle.c)"},
        "e2e": {"value": round(value, 3), "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
