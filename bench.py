#!/usr/bin/env python3
"""Benchmark of the path-tracing hot path on B200.

Default workload (the one the headline is quoted on): the closest-hit query
set -- 1,000,000 fp32 triangles (uniform centroids in [0,1]^3, N(0, 0.005^2)
vertex jitter) in the reference's SAH BVH, 4,194,304 rays from a radius-2
sphere towards uniform points of the cube. One step = one closest-hit pass
over all rays (BVHAccel::Intersect semantics, bit-exact hit IDs).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints ONE JSON line. Under torchrun (N > 1) every rank traces its own copy of
the query set on its own GPU with no collective on the data path (weak
scaling); the step time is the max over ranks.

--impl reference times the reference's own CPU implementation of the same
query (its sources compiled in place with its shipped -O3 -ffast-math flags
and OpenMP, oracle/_ref/libprr_ref_fast.so; the C restatement if that library
is absent) on all host cores.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

N_TRIS = 1_000_000
N_RAYS = 4_194_304
WORKLOAD = "closest-hit query set: 1,000,000 fp32 triangles, 4,194,304 rays"
METRIC = "Mrays/s"
FALLBACK_HBM_GBS = 6650.0


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def init_dist(world, local):
    import torch
    import torch.distributed as dist
    if world > 1 and not dist.is_initialized():
        from datetime import timedelta
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=timedelta(seconds=120))
    return world > 1


def barrier(on):
    if on:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x, on):
    if not on:
        return x
    import torch
    import torch.distributed as dist
    dev = torch.device("cuda", torch.cuda.current_device()) if torch.cuda.is_available() else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# GPU busy-wait queued before each timed step's start event (about 30 ms at
# 1.97 GHz): a host stall shorter than this (a driver call held up by the
# clock sampler) then falls before the step instead of inside it.
SLEEP_CYCLES = 60_000_000


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            # nvidia-smi's start-up holds the driver for a while and stalls
            # CUDA calls: let it deliver its first sample before any timing
            deadline = time.time() + 10.0
            while not self.lines and time.time() < deadline and self.proc.poll() is None:
                time.sleep(0.05)
            time.sleep(0.3)
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.15)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for name, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return FALLBACK_HBM_GBS, "fallback"


def profiled_traffic(kernel: str):
    """dram bytes per launch recorded by the ncu capture summarised under
    profiles/ (a `traffic_bytes_per_launch: N` line), or None."""
    for f in sorted((ROOT / "profiles").glob(f"{kernel}*.md")):
        for line in f.read_text().splitlines():
            if line.strip().startswith("traffic_bytes_per_launch:"):
                try:
                    return float(line.split(":", 1)[1].strip().split()[0])
                except ValueError:
                    return None
    return None


def workload_arrays():
    from photorealisticrender4610_b200 import scenes
    return scenes.query_set(N_TRIS, N_RAYS, seed=1)


def parse_launch(text):
    """'block=128,persistent=1' (or 'paths=1048576,block=128,stack=12,ordered=1'
    for the wavefront) -> launch config dict."""
    out = {}
    for kv in filter(None, (text or "").split(",")):
        k, v = kv.split("=")
        out[{"block": "block_size"}.get(k, k)] = int(v)
    return out


def traversal_work(verts, o, d, threads):
    """Mean interior visits I and triangle tests T per ray, counted by the
    oracle's traversal on the same rays (sample of 2^20 rays)."""
    from oracle.loader import PortOracle
    port = PortOracle()
    m = port.mesh(verts)
    k = min(len(o), 1 << 20)
    _, _, _, vis, tst = m.intersect(o[:k], d[:k], threads=threads, stats=True)
    return float(vis.mean()), float(tst.mean())


_CPU_MESH = {}


def cpu_reference_rate(verts, o, d, n_sample, threads):
    """Reference CPU closest-hit throughput (Mrays/s) on n_sample rays with
    `threads` OpenMP threads (the BVH is built once, untimed: a traversal
    rate, like the GPU number)."""
    from oracle import loader
    if "mesh" not in _CPU_MESH:
        t0 = time.perf_counter()
        if loader.reference_available(fast=True):
            mesh, kind = loader.ReferenceOracle(fast=True).mesh(verts), "reference"
        else:
            mesh, kind = loader.PortOracle().mesh(verts), "port"
        build_s = time.perf_counter() - t0
        mesh.intersect(o[:4096], d[:4096], threads=threads)
        _CPU_MESH.update(kind=kind, mesh=mesh, build_s=build_s)
    mesh, kind = _CPU_MESH["mesh"], _CPU_MESH["kind"]
    t0 = time.perf_counter()
    mesh.intersect(o[:n_sample], d[:n_sample], threads=threads)
    return n_sample / (time.perf_counter() - t0) / 1e6, kind


def query_config(world):
    """The query-set workload as both arms name it."""
    return {"workload": WORKLOAD, "rays_per_step": N_RAYS, "triangles": N_TRIS, "seed": 1,
            "l2": "GPU arm: L2 flushed (512 MB write) before every timed step",
            "parallelism": f"replica x{world}" if world > 1 else "1 GPU"}


def run_reference(args, rank, world):
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    verts, o, d = workload_arrays()
    sample = N_RAYS
    for _ in range(args.warmup):
        cpu_reference_rate(verts, o, d, 1 << 16, threads)
    rates = []
    kind = None
    t_all = time.perf_counter()
    for k in range(args.steps):
        r, kind = cpu_reference_rate(verts, o, d, sample, threads)
        rates.append(r)
    total = time.perf_counter() - t_all
    value = float(np.mean(rates))
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "Mrays/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": total / max(1, args.steps) * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": query_config(world),
        "threads": threads,
        "cpu_baseline": {"value": value, "unit": "Mrays/s", "cores": threads, "kind": kind,
                         "sample": f"all {N_RAYS} query rays per step (the BVH built once, "
                                   "untimed)"},
        "e2e": {"value": value, "unit": "Mrays/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args, rank, world, on):
    import torch
    import photorealisticrender4610_b200 as prr

    dev = torch.device("cuda", torch.cuda.current_device())
    verts, o, d = workload_arrays()
    scene = prr.Scene.single_mesh(verts)
    # the scene build (SAH tree on the host cores, then the upload), timed on a
    # second build so the first one's context set-up is not counted
    t0 = time.perf_counter()
    second = prr.Scene.single_mesh(verts)
    build_s = time.perf_counter() - t0
    # release it now (a collection during the timed steps would free device
    # memory between them)
    del second
    import gc
    gc.collect()
    torch.cuda.synchronize()
    O = torch.from_numpy(o).to(dev)
    D = torch.from_numpy(d).to(dev)
    flush = torch.empty(512 << 20, dtype=torch.uint8, device=dev)  # > 126 MB L2

    # autotune the launch shape on this scene (untimed)
    configs = [{"block_size": 128, "persistent": 1}]
    for block in (128, 256):
        for refill in (4, 8, 12):
            configs.append({"block_size": block, "persistent": 2, "batch": refill})
        for leaf in (8, 16, 24):
            configs.append({"block_size": block, "persistent": 3, "batch": 8, "leaf_batch": leaf})
    # the same launch shapes after a coherence reordering of the rays (inside
    # the timed call)
    for sort in (1, 3, 4, 5):
        for refill in (8, 12, 16):
            configs.append({"block_size": 128, "persistent": 2, "batch": refill, "sort_rays": sort})
        configs.append({"block_size": 128, "persistent": 1, "sort_rays": sort})
    if args.launch:
        configs = [parse_launch(args.launch)]
    best, best_ms = None, math.inf
    tuned = []
    for cfg in configs if len(configs) > 1 else []:
        times = []
        for _ in range(2):
            flush.zero_()
            torch.cuda._sleep(SLEEP_CYCLES)
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record()
            scene.mesh_intersect(0, O, D, config=cfg)
            e.record()
            torch.cuda.synchronize()
            times.append(s.elapsed_time(e))
        tuned.append((min(times), cfg))
        if min(times) < best_ms:
            best, best_ms = cfg, min(times)
    if best is None:
        best = configs[0]

    for _ in range(args.warmup):
        flush.zero_()
        scene.mesh_intersect(0, O, D, config=best)
    torch.cuda.synchronize()

    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    with ClockSampler(dev.index if world == 1 else int(os.environ.get("LOCAL_RANK", 0))) as clk:
        barrier(on)
        torch.cuda.synchronize()
        # keep the GPU busy (about 0.3 s) while the host enqueues all K steps,
        # so no host-side latency falls between a step's two events: a driver
        # call can wait tens of ms on the nvidia-smi clock sampler, which a
        # per-step cushion did not always cover
        torch.cuda._sleep(SLEEP_CYCLES * 10)
        for k in range(args.steps):
            flush.zero_()
            starts[k].record()
            hid, t = scene.mesh_intersect(0, O, D, config=best)
            ends[k].record()
        torch.cuda.synchronize()
        barrier(on)
    kernel_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    ms_step = max_over_ranks(float(np.mean(kernel_ms)), on)
    ms_median = max_over_ranks(float(np.median(kernel_ms)), on)
    value = N_RAYS * world / (ms_step * 1e-3) / 1e6

    assert int((hid >= 0).sum().item()) > 0.99 * N_RAYS
    if args.kernel_only:
        if rank == 0:
            print(json.dumps({"kernel_ms": kernel_ms, "launch": best, "mrays_s": value}))
        return 0

    # end to end through the host-buffer C ABI call (pinned host arrays)
    ho = torch.from_numpy(o).pin_memory().numpy()
    hd = torch.from_numpy(d).pin_memory().numpy()
    hid_h = torch.empty(N_RAYS, dtype=torch.int32).pin_memory().numpy()
    t_h = torch.empty(N_RAYS, dtype=torch.float32).pin_memory().numpy()
    # the host call traces chunks of at most 1M rays, where reordering the
    # rays costs relatively more: its launch shape is chosen among the fastest
    # kernel shape with and without reordering, by timing the call itself
    e2e_cfg = best
    unsorted = [c for _, c in sorted(tuned, key=lambda x: x[0]) if not c.get("sort_rays")]
    if unsorted and unsorted[0] != best:
        host_ms = {}
        for cand in (best, unsorted[0]):
            scene.mesh_intersect_host(0, ho, hd, hid_h, t_h, config=cand)
            ts = []
            for _ in range(3):
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                scene.mesh_intersect_host(0, ho, hd, hid_h, t_h, config=cand)
                ts.append(time.perf_counter() - t0)
            host_ms[json.dumps(cand)] = min(ts)
        e2e_cfg = json.loads(min(host_ms, key=host_ms.get))
    scene.mesh_intersect_host(0, ho, hd, hid_h, t_h, config=e2e_cfg)
    e2e_ms = []
    for _ in range(max(3, args.steps)):
        barrier(on)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        scene.mesh_intersect_host(0, ho, hd, hid_h, t_h, config=e2e_cfg)
        e2e_ms.append((time.perf_counter() - t0) * 1e3)
    e2e_step = max_over_ranks(float(np.median(e2e_ms)), on)
    e2e_value = N_RAYS * world / (e2e_step * 1e-3) / 1e6
    assert np.array_equal(hid_h, hid.cpu().numpy())

    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    I, T = traversal_work(verts, o, d, threads)
    bytes_per_ray = 24 + 8 + 64 * I + 36 * T
    peak, peak_kind = measured_peaks()
    achieved = bytes_per_ray * N_RAYS / (float(np.mean(kernel_ms)) * 1e-3) / 1e9
    traffic = profiled_traffic("k_mesh_closest")
    cpu_rate, cpu_kind = cpu_reference_rate(verts, o, d, N_RAYS, threads)
    cpu_rate_1, _ = cpu_reference_rate(verts, o, d, 131072, 1)
    clocks = clk.summary()
    line = {
        "metric": METRIC, "value": value, "unit": "Mrays/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": query_config(world),
        "run": {"launch": best, "e2e_launch": e2e_cfg,
                "tuned_fastest": [[round(ms, 3), c] for ms, c in sorted(tuned, key=lambda x: x[0])[:6]],
                "step_ms": [round(x, 3) for x in kernel_ms],
                "median_ms": ms_median, "e2e_ms": [round(x, 3) for x in e2e_ms]},
        "e2e": {"value": e2e_value, "unit": "Mrays/s", "h2d_bytes_per_step": N_RAYS * 24,
                "d2h_bytes_per_step": N_RAYS * 8},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic,
                     "limiter": "L1/L2 latency and SIMT issue, not HBM: the BVH and triangles "
                                "stay in L2 (DRAM a few % busy), about 12 of 32 lanes active "
                                "per warp instruction",
                     "peak_source": f"{peak_kind} hbm_gbs",
                     "bytes_per_ray": bytes_per_ray, "interior_visits": I, "tri_tests": T},
        "cpu_baseline": {"value": cpu_rate, "unit": "Mrays/s", "cores": threads,
                         "kind": cpu_kind, "sample": f"all {N_RAYS} query rays, one pass",
                         "one_core": {"value": cpu_rate_1, "sample": "first 131072 query rays"}},
        "bvh_build_s": {"ours": build_s, "ours_threads": threads,
                        "reference": _CPU_MESH.get("build_s"), "reference_threads": 1},
        "clocks": clocks,
        "gpu_launches": args.steps * (6 if best.get("sort_rays") else 1),
    }
    if world == 1 and args.extras != "none":
        # the other north-star targets on the same box, as keys of this line
        for name in args.extras.split(","):
            t0 = time.perf_counter()
            if name == "museum":
                sub = render_result(args, rank, world, on, "museum", min(args.steps, 5), 3,
                                    crop_check=True)
            elif name == "caustics":
                sub = caustics_result(args, rank, world, on, min(args.steps, 5), 3)
            elif name == "serving":
                sub = serving_result(args, rank, world, n_requests=60, arms_text="none")
            else:
                raise ValueError(f"unknown extra workload {name}")
            sub = {k: v for k, v in sub.items() if k not in EXTRA_DROP}
            sub["bench_s"] = time.perf_counter() - t0
            line[name] = sub
    print(json.dumps(line), flush=True)
    return 0


# keys of a workload's own line that its entry under the headline line leaves out
EXTRA_DROP = ("n_gpus", "higher_is_better", "scaling", "vs_baseline", "dtype", "data")


def _scenes():
    return __import__("photorealisticrender4610_b200.scenes", fromlist=["x"])


RENDER_WORKLOADS = {
    # name: (scene factory, max spp, depth, description, adaptive (min spp, threshold) or None)
    "museum": (lambda: _scenes().museum_like(),
               64, 8, "museum-like: 6 displaced level-7 icospheres (1,966,082 triangles), "
               "2048x1024 HDR sky, 1920x1080, 64 spp, depth 8", None),
    "cornell": (lambda: _scenes().cornell_box(),
                16, 5, "Cornell box 256x256, 16 spp, depth 5", None),
    # the reference's own render settings (main.cpp:11-20) on the museum-like scene
    "museum-adaptive": (lambda: _scenes().museum_like(960, 540),
                        256, 12, "museum-like scene with the reference renderer's main.cpp "
                        "settings: 960x540, adaptive 1..256 spp, Welford threshold 0.01, "
                        "depth 12", (1, 0.01)),
}


# Algorithmic bytes of a wavefront frame, per unit of work counted by
# prr_render_counts: a closest-hit ray reads its origin and direction (24 B)
# and writes its hit record (16 B); a shadow ray reads origin, direction and
# tmax (28 B) and writes its visibility byte; each interior node visited reads
# the two child boxes of one 64 B node, each triangle test the 36 B of v0, e1,
# e2, each object leaf 16 B (sphere centre and radius, or a mesh's root). The
# shading stages read and write per path-bounce the path state they need: a
# surface hit 132 B (hit record, ray, throughput, radiance, RNG state, flags
# in; next ray, throughput, radiance, RNG state out), a mirror/glass hit 104 B,
# a miss 60 B; the film adds 12 B per pixel.
FRAME_BYTES = {"closest_ray": 40, "shadow_ray": 29, "node": 64, "tri": 36, "object": 16,
               "surface": 132, "delta": 104, "miss": 60, "pixel": 12}


def frame_bytes(c, npix):
    B = FRAME_BYTES
    return (c["closest_rays"] * B["closest_ray"] + c["shadow_rays"] * B["shadow_ray"] +
            (c["closest_nodes"] + c["shadow_nodes"]) * B["node"] +
            (c["closest_tris"] + c["shadow_tris"]) * B["tri"] +
            (c["closest_objects"] + c["shadow_objects"]) * B["object"] +
            c["surface_hits"] * B["surface"] + c["delta_hits"] * B["delta"] +
            c["misses"] * B["miss"] + npix * B["pixel"])


def run_render(args, rank, world, on):
    line = render_result(args, rank, world, on, args.workload, args.steps, args.warmup)
    if line is not None:
        print(json.dumps(line), flush=True)
    return 0


def render_result(args, rank, world, on, workload, steps, warmup, crop_check=False):
    """Samples/s of the plain megakernel and of the wavefront integrator on a
    full frame (value = wavefront, the faster one; both reported). Returns the
    JSON line's dict on rank 0 (None elsewhere). crop_check adds the rMSE of a
    32x32 crop at 4096 spp against the reference renderer."""
    import torch
    import photorealisticrender4610_b200 as prr

    factory, spp, depth, desc_text, adaptive = RENDER_WORKLOADS[workload]
    min_spp, thr = adaptive if adaptive else (None, 0.05)
    dev = torch.device("cuda", torch.cuda.current_device())
    desc = factory()
    if args.size:
        desc.width, desc.height = (int(v) for v in args.size.split("x"))
        desc_text += f" (resized to {desc.width}x{desc.height})"
    if args.spp:
        spp = args.spp
        desc_text += f" (spp {spp})"
    scene = prr.Scene.from_desc(desc)
    npix = desc.width * desc.height
    if args.launch:
        cfg = parse_launch(args.launch)
        scene.set_wavefront(cfg.get("paths", 0), cfg.get("block_size", 0), True,
                            cfg.get("stack", 0), cfg.get("ordered", 1), cfg.get("refill", 0))
        tuned = cfg
    else:
        # tune on enough samples per pixel (a power of two, so the candidate
        # pass sizes divide it) that the largest candidate pass (64M paths)
        # fits in the tuning render, or on the whole frame
        tune_spp = 4
        while tune_spp < spp and npix * tune_spp < (1 << 26):
            tune_spp *= 2
        tuned = scene.autotune(min(tune_spp, spp), depth)

    flush = torch.empty(512 << 20, dtype=torch.uint8, device=dev)  # > 126 MB L2

    def timed(mode, steps):
        ms = []
        rays = None
        for _ in range(steps):
            flush.zero_()
            torch.cuda._sleep(SLEEP_CYCLES)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            img, cnt, rays = scene.render(spp, depth, seed=1, mode=mode, slices=0,
                                          count_rays=True, min_spp=min_spp, threshold=thr)
            b.record()
            torch.cuda.synchronize()
            ms.append(a.elapsed_time(b))
        timed.samples = int(cnt.sum().item())  # samples actually taken (adaptive: the spp map)
        return ms, img, rays

    if not args.kernel_only:
        timed("plain", 1)
    timed("wavefront", warmup)
    with ClockSampler(dev.index) as clk:
        barrier(on)
        wf_ms, wf_img, wf_rays = timed("wavefront", steps)
        barrier(on)
    wf_launches = scene.stats()["last_render_launches"] * steps
    if args.kernel_only:
        if rank == 0:
            print(json.dumps({"frame_ms": wf_ms,
                              "msamples_s": timed.samples / np.mean(wf_ms) / 1e3,
                              "launch": tuned}))
        return None
    samples = timed.samples
    timed("plain", 1)
    pl_ms, pl_img, pl_rays = timed("plain", max(1, min(steps, 3)))
    wf_step = max_over_ranks(float(np.mean(wf_ms)), on)
    # the plain renderer is the comparison, not the headline: its median frame,
    # so one host stall longer than the queued busy-wait does not set the ratio
    pl_step = max_over_ranks(float(np.median(pl_ms)), on)
    value = samples * world / (wf_step * 1e-3) / 1e6
    plain_value = samples * world / (pl_step * 1e-3) / 1e6
    rays = wf_rays.cpu().numpy()
    rel = float(((wf_img - pl_img) ** 2).sum() / (pl_img ** 2).sum())

    # end to end: the C ABI call plus the copy of the image to pinned host memory
    host = torch.empty((desc.height, desc.width, 3), dtype=torch.float32).pin_memory()
    e2e = []
    for _ in range(max(3, steps)):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        img, _ = scene.render(spp, depth, seed=1, mode="wavefront", min_spp=min_spp,
                              threshold=thr)
        host.copy_(img)
        torch.cuda.synchronize()
        e2e.append((time.perf_counter() - t0) * 1e3)
    e2e_value = samples * world / (float(np.median(e2e)) * 1e-3) / 1e6
    # the frame's work, counted by a separate (untimed) counting render
    _, counts = scene.render_counts(spp, depth, seed=1, min_spp=min_spp, threshold=thr)
    if rank != 0:
        return None
    peak, peak_kind = measured_peaks()
    alg = frame_bytes(counts, npix)
    achieved = alg / (wf_step * 1e-3) / 1e9
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": None,
                "peak_source": f"{peak_kind} hbm_gbs",
                "basis": "algorithmic bytes of the whole wavefront frame (traversal steps "
                         "and hit classes counted by prr_render_counts, bytes per unit in "
                         "bench.FRAME_BYTES) / frame time",
                "bytes_per_frame": alg, "bytes_per_unit": FRAME_BYTES,
                "counts": counts,
                "nodes_per_closest_ray": counts["closest_nodes"] / max(1, counts["closest_rays"]),
                "tris_per_closest_ray": counts["closest_tris"] / max(1, counts["closest_rays"]),
                "nodes_per_shadow_ray": counts["shadow_nodes"] / max(1, counts["shadow_rays"]),
                "tris_per_shadow_ray": counts["shadow_tris"] / max(1, counts["shadow_rays"])}
    crop = None
    if crop_check:
        from oracle import loader
        if loader.reference_available():
            win = (desc.width // 2 - 16, desc.height // 2 - 16, desc.width // 2 + 16,
                   desc.height // 2 + 16)
            gimg, _ = scene.render(4096, depth, seed=1, mode="wavefront", window=win)
            rimg, _ = loader.ReferenceOracle().scene(desc).render(depth, 4096, 1, window=win)
            g64 = gimg.cpu().numpy().astype(np.float64)
            crop = {"window": list(win), "spp": 4096,
                    "rel_mse": float(((g64 - rimg) ** 2).sum() / max((rimg.astype(np.float64) ** 2).sum(), 1e-30)),
                    "against": "the reference renderer (its sources compiled in place, IEEE "
                               "flags) on the same per-sample RNG streams"}
    threads = os.cpu_count() or 1
    cpu = None
    from oracle import loader
    if loader.reference_available(fast=True):
        ref = loader.ReferenceOracle(fast=True)
        rs = ref.scene(desc)
        win = (desc.width // 2 - 32, desc.height // 2 - 32, desc.width // 2 + 32,
               desc.height // 2 + 32)
        cspp = 16 if not adaptive else spp
        t0 = time.perf_counter()
        _, rcnt = rs.render(depth, cspp, 1, window=win, threads=threads, min_spp=min_spp,
                            threshold=thr)
        dt = time.perf_counter() - t0
        cpu = {"value": float(np.sum(rcnt)) / dt / 1e6, "unit": "Msamples/s", "cores": threads,
               "kind": "reference",
               "sample": f"64x64 centre crop at {cspp} spp" + (" (adaptive)" if adaptive else "")}
    line = {
        "metric": "Msamples/s", "value": value, "unit": "Msamples/s", "n_gpus": world,
        "steps": steps, "warmup": warmup, "ms_per_step": wf_step,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": desc_text, "mode": "wavefront", "autotuned": tuned,
                   "l2": "flushed (512 MB write) before every timed frame",
                   "frame_ms": [round(x, 3) for x in wf_ms],
                   "plain_frame_ms": [round(x, 3) for x in pl_ms]},
        "plain_msamples_s": plain_value, "wavefront_vs_plain": value / plain_value,
        "plain_vs_wavefront_rel_mse": rel,
        "mrays_s": float(rays.sum()) / (wf_step * 1e-3) / 1e6,
        "rays_per_frame": {"closest": int(rays[0]), "shadow": int(rays[1])},
        "e2e": {"value": e2e_value, "unit": "Msamples/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": npix * 12},
        "roofline": roofline,
        "crop_check": crop,
        "cpu_baseline": cpu,
        "clocks": clk.summary(),
        "gpu_launches": wf_launches,
    }
    return line


CAUSTICS = ("caustics: glass sphere (r=1, IOR 1.5) over a diffuse plane, light of intensity 100 "
            "at (0,4,0); 2,000,000 photons traced, grid radius 0.02, 64-nearest gather at every "
            "camera hit; 1024x1024, 32 spp, depth 8")


# Algorithmic bytes of the caustic render kernel (the step's dominant one), per
# unit counted by prr_render_caustics_counts: each (pixel, sample) writes its
# 16 B contribution and the film stage reads it back; each photon a gather's
# cell walk tests reads 16 B of the cell-sorted copy (position, power r), each
# one inside the radius 16 B more (power g, b); the image is 12 B per pixel.
CAUSTIC_BYTES = {"sample": 32, "photon_tested": 16, "photon_inside": 16, "pixel": 12}


def run_caustics(args, rank, world, on):
    line = caustics_result(args, rank, world, on, args.steps, args.warmup)
    if line is not None:
        print(json.dumps(line), flush=True)
    return 0


def caustics_result(args, rank, world, on, steps, warmup):
    """One step = trace 2M photons + build the photon grid + render the frame
    with the caustic gather. value = camera samples/s of the whole step.
    Returns the JSON line's dict on rank 0 (None elsewhere)."""
    import torch
    import photorealisticrender4610_b200 as prr
    from photorealisticrender4610_b200 import scenes

    dev = torch.device("cuda", torch.cuda.current_device())
    desc = scenes.caustics()
    scene = prr.Scene.from_desc(desc)
    pm = prr.PhotonMap()
    n_ph, radius, spp, k, depth = 2_000_000, 0.02, 32, 64, 8
    npix = desc.width * desc.height
    flush = torch.empty(512 << 20, dtype=torch.uint8, device=dev)

    def step():
        flush.zero_()
        torch.cuda._sleep(SLEEP_CYCLES)
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
        ev[0].record()
        pm.emit(scene, n_ph, seed=1, max_depth=depth)
        ev[1].record()
        pm.build(radius)
        ev[2].record()
        img = pm.render_caustics(scene, spp, max_depth=depth, seed=1, k_nearest=k)
        ev[3].record()
        torch.cuda.synchronize()
        return [ev[i].elapsed_time(ev[i + 1]) for i in range(3)], img

    def api_step():
        """The same step as a user makes it: emit, build, render."""
        pm.emit(scene, n_ph, seed=1, max_depth=depth)
        pm.build(radius)
        return pm.render_caustics(scene, spp, max_depth=depth, seed=1, k_nearest=k)

    for _ in range(warmup):
        step()
    with ClockSampler(dev.index) as clk:
        barrier(on)
        launches0 = pm.launches()
        phases = [step()[0] for _ in range(steps)]
        launches = pm.launches() - launches0
        barrier(on)
    ph = np.array(phases)
    step_ms = max_over_ranks(float(ph.sum(1).mean()), on)
    value = npix * spp * world / (step_ms * 1e-3) / 1e6
    stored, grid_res = pm.info()
    # end to end: the same step through the API plus the image copied to pinned host memory
    host = torch.empty((desc.height, desc.width, 3), dtype=torch.float32).pin_memory()
    e2e = []
    for _ in range(max(3, steps)):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        img = api_step()
        host.copy_(img)
        torch.cuda.synchronize()
        e2e.append((time.perf_counter() - t0) * 1e3)
    e2e_value = npix * spp * world / (float(np.median(e2e)) * 1e-3) / 1e6
    # the render's gather work, counted by a separate (untimed) counting render
    _, counts = pm.render_caustics_counts(scene, spp, max_depth=depth, seed=1, k_nearest=k)
    if rank != 0:
        return None
    render_ms = float(ph[:, 2].mean())
    B = CAUSTIC_BYTES
    alg = (npix * spp * B["sample"] + counts["photons_tested"] * B["photon_tested"] +
           counts["photons_inside"] * B["photon_inside"] + npix * B["pixel"])
    peak, peak_kind = measured_peaks()
    achieved = alg / (render_ms * 1e-3) / 1e9
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": profiled_traffic("k_caustic_samples"),
                "peak_source": f"{peak_kind} hbm_gbs",
                "kernel": "k_caustic_samples + k_caustic_dense + k_caustic_film (one render call)",
                "traffic_kernel": "k_caustic_samples",
                "limiter": "latency and issue, not HBM: the photon grid and the scene stay in L2 "
                           "(DRAM under 3% busy); the sample kernel issues on about 72% of "
                           "cycles with 49% of warps resident (64 registers)",
                "basis": "algorithmic bytes of the render + gather (gather work counted by "
                         "prr_render_caustics_counts, bytes per unit in bench.CAUSTIC_BYTES) / "
                         "its CUDA-event time",
                "bytes_per_render": alg, "bytes_per_unit": CAUSTIC_BYTES, "counts": counts,
                "photons_tested_per_gather": counts["photons_tested"] / max(1, counts["gathers"])}
    cpu = None
    from oracle import loader
    if loader.reference_available(fast=True):
        threads = os.cpu_count() or 1
        rs = loader.ReferenceOracle(fast=True).scene(desc)
        n_cpu = 200_000
        t0 = time.perf_counter()
        rs.photon_emit(n_cpu, 1, max_depth=depth, threads=threads)
        dt = time.perf_counter() - t0
        cpu = {"value": n_cpu / dt / 1e6, "unit": "Mphotons/s", "cores": threads,
               "kind": "reference", "sample": f"{n_cpu} photons traced by Photon.cpp's trace"}
    line = {
        "metric": "Msamples/s", "value": value, "unit": "Msamples/s", "n_gpus": world,
        "steps": steps, "warmup": warmup, "ms_per_step": step_ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": CAUSTICS, "photons_stored": stored, "grid_res": grid_res,
                   "l2": "flushed (512 MB write) before every timed step",
                   "phase_ms": {"emit": float(ph[:, 0].mean()), "grid": float(ph[:, 1].mean()),
                                "render_gather": float(ph[:, 2].mean())}},
        "mphotons_s": n_ph / (float(ph[:, 0].mean()) * 1e-3) / 1e6,
        "e2e": {"value": e2e_value, "unit": "Msamples/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": npix * 12},
        "roofline": roofline,
        "cpu_baseline": cpu,
        "clocks": clk.summary(),
        "gpu_launches": launches,
    }
    return line


def serving_pool():
    """Eight procedural scenes of about 10k, 30k, 100k, 300k, 600k, 1M, 1.5M
    and 2M triangles, built like the museum-like scene (displaced icospheres
    under the HDR sky: 2 / 6 level-4, 5 level-5, 4 level-6, 2 / 6 level-7
    spheres) and the query set (1M / 1.5M triangle soups under the same sky)."""
    from photorealisticrender4610_b200 import scenes as sc
    pool = []
    for level, spheres in ((4, 2), (4, 6), (5, 5), (6, 4), (7, 2)):
        pool.append(sc.museum_like(512, 512, level=level, env_size=(1024, 512), spheres=spheres))
    for n in (1_000_000, 1_500_000):
        d = sc.SceneDesc(width=512, height=512, name=f"soup{n}")
        m = d.add_material(sc.Material(sc.DIFFUSE, (0.7, 0.6, 0.5), 0.6, 0.0))
        v, _, _ = sc.query_set(n, 1, seed=n)
        d.objects.append(sc.MeshObject(v, m))
        d.env = pool[0].env
        d.camera = sc.Camera(eye=(2.2, 1.6, 2.4), target=(0.5, 0.5, 0.5), fovv=40, fovh=45)
        pool.append(d)
    pool.append(sc.museum_like(512, 512, level=7, env_size=(1024, 512)))
    return pool


def run_serving(args, rank, world, on):
    line = serving_result(args, rank, world)
    if line is not None:
        print(json.dumps(line), flush=True)
    return 0


def serving_result(args, rank, world, n_requests=None, arms_text=None):
    """Continuous-batching server (wavefront steps) under Poisson arrivals,
    beside the same server on megakernel steps and the plain renderer run one
    request at a time in arrival order. Returns the JSON line's dict on rank 0
    (None elsewhere)."""
    import math
    import threading
    import torch
    import photorealisticrender4610_b200 as prr

    if rank != 0:
        return None
    rng = np.random.Generator(np.random.PCG64(7))
    pool = serving_pool()
    scenes_ = [prr.Scene.from_desc(d) for d in pool]
    tris = [d.n_triangles() for d in pool]
    sizes = [(256, 256), (512, 512), (1024, 1024), (1920, 1080)]
    n = n_requests or args.requests
    gaps = rng.exponential(1.0 / args.rate, n)
    arrive = np.cumsum(gaps) - gaps[0]
    reqs = []
    for k in range(n):
        spp = int(round(math.exp(rng.uniform(math.log(4), math.log(args.max_spp)))))
        reqs.append((int(rng.integers(0, len(pool))), sizes[int(rng.integers(0, 4))], spp))
    depth = 8
    total_samples = sum(w * h * spp for _, (w, h), spp in reqs)

    # outputs in pinned host memory; past 256 requests, a ring of 256 buffers
    # of the largest size (a buffer is reused by every 256th request)
    ring = min(n, 256)
    big = max(w * h for _, (w, h), _ in reqs)
    bufs = [torch.empty(big * 3, dtype=torch.float32).pin_memory().numpy() for _ in range(ring)]
    host = [bufs[k % ring][:w * h * 3].reshape(h, w, 3) for k, (_, (w, h), _) in enumerate(reqs)]

    def serve(max_active, samples_per_step, arrive=arrive, integrator="wavefront"):
        """Replays the arrival schedule against a server; returns latencies,
        the wall span and the server stats."""
        srv = prr.Server(max_active=max_active, samples_per_step=samples_per_step,
                         integrator=integrator)
        for s_ in scenes_:
            srv.add_scene(s_)
        srv.wait(srv.submit(0, 2, depth, size=(64, 64)))  # warm-up
        launches0 = srv.stats()["launches"]
        ids = [None] * n
        t_start = time.perf_counter()

        def submitter():
            for k, (sc_, size, spp) in enumerate(reqs):
                delay = arrive[k] - (time.perf_counter() - t_start)
                if delay > 0:
                    time.sleep(delay)
                ids[k] = srv.submit(sc_, spp, depth, seed=k + 1, size=size, out=host[k])

        th = threading.Thread(target=submitter)
        th.start()
        th.join()
        infos = [srv.wait(i) for i in ids]
        st = srv.stats()
        st["timed_launches"] = st["launches"] - launches0
        srv.close()
        lat = np.array([i["done_s"] - i["submit_s"] for i in infos])
        span = max(i["done_s"] for i in infos) - min(i["submit_s"] for i in infos)
        return lat, span, st

    with ClockSampler(torch.cuda.current_device()) as clk:
        lat, span, st = serve(args.max_active, 1 << 20)
    served_rate = total_samples / span / 1e6
    busy_rate = total_samples / st["busy_s"] / 1e6
    arms = set((arms_text or args.serving_arms).split(","))
    if "all" in arms:
        arms = {"megakernel", "one", "sustainable"}

    def pct(lat_, span_, st_):
        return {"p50_s": float(np.percentile(lat_, 50)), "p99_s": float(np.percentile(lat_, 99)),
                "msamples_s": total_samples / span_ / 1e6,
                "busy_msamples_s": total_samples / st_["busy_s"] / 1e6}
    extra = {}
    if "megakernel" in arms:  # the same schedule on megakernel steps (request tiles)
        extra["megakernel_steps"] = pct(*serve(args.max_active, 1 << 20, integrator="megakernel"))
    if "one" in arms:  # one request at a time in arrival order, plain megakernel
        extra["one_at_a_time"] = pct(*serve(1, 1 << 24, integrator="megakernel"))
    if "sustainable" in arms:
        # the same requests arriving at 70% of the measured busy throughput
        # (mean work per request / capacity)
        sus_rate = 0.7 * busy_rate * 1e6 / (total_samples / n)
        sus, sus_span, sus_st = serve(args.max_active, 1 << 20, arrive * (args.rate / sus_rate))
        extra["sustainable"] = dict(pct(sus, sus_span, sus_st), rate_per_s=sus_rate, load=0.7)
    line = {
        "metric": "served p50/p99 latency (s) and Msamples/s", "value": float(np.percentile(lat, 99)),
        "unit": "s (p99 latency)", "n_gpus": world, "steps": n, "warmup": 1,
        "ms_per_step": float(np.mean(lat)) * 1e3, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "serving: Poisson arrivals over a pool of 8 procedural scenes "
                               f"({min(tris)}-{max(tris)} triangles), resolution from "
                               "{256^2, 512^2, 1024^2, 1920x1080}, spp log-uniform "
                               f"[4, {args.max_spp}], depth {depth}",
                   "requests": n, "rate_per_s": args.rate, "max_active": args.max_active,
                   "offered_msamples_s": total_samples / (arrive[-1] + 1e-9) / 1e6,
                   "total_samples": total_samples},
        "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
        "served_msamples_s": served_rate, "served_busy_msamples_s": busy_rate,
        "worker_s": {"span": span, "steps": int(st["steps"]), "busy": st["busy_s"],
                     "admit": st["admit_s"], "complete": st["complete_s"]},
        "server_steps": "wavefront (all running requests in one set of ordered ray queues)",
        **extra,
        "failed": int(st["failed"]),
        "gpu_launches": int(st["timed_launches"]),
        "e2e": {"value": served_rate, "unit": "Msamples/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": int(np.mean([w * h * 12 for _, (w, h), _ in reqs]))},
        "clocks": clk.summary(),
    }
    return line


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--launch", default="", help="fixed launch shape, e.g. block=128,persistent=0")
    ap.add_argument("--workload", choices=["query", "museum", "cornell", "museum-adaptive",
                                           "serving", "caustics"],
                    default="query")
    ap.add_argument("--requests", type=int, default=120, help="serving: number of requests")
    ap.add_argument("--rate", type=float, default=50.0, help="serving: Poisson arrivals per s")
    ap.add_argument("--max-spp", type=int, default=256, help="serving: spp upper bound")
    ap.add_argument("--max-active", type=int, default=64, help="serving: concurrent requests")
    ap.add_argument("--serving-arms", default="all",
                    help="serving: comparison runs beside the wavefront server, 'all' or a comma "
                         "list of megakernel, one, sustainable (or 'none')")
    ap.add_argument("--size", default="", help="render workloads: WxH override")
    ap.add_argument("--spp", type=int, default=0, help="render workloads: spp override")
    ap.add_argument("--kernel-only", action="store_true",
                    help="time the kernel only (no e2e, no CPU baseline): profiling runs")
    ap.add_argument("--extras", default="museum,caustics,serving",
                    help="query workload at 1 GPU: other workloads measured after the headline "
                         "and added as keys of its line (comma list, or 'none')")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    rank, world, local = dist_env()
    if args.impl == "reference":
        if world > 1 and rank != 0:
            return 0
        return run_reference(args, rank, world)
    on = init_dist(world, local)
    try:
        if args.workload == "serving":
            return run_serving(args, rank, world, on)
        if args.workload == "caustics":
            return run_caustics(args, rank, world, on)
        if args.workload != "query":
            return run_render(args, rank, world, on)
        return run_ours(args, rank, world, on)
    finally:
        if on:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
