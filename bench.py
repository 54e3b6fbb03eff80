#!/usr/bin/env python3
"""Benchmark: paths/s of PATH_TRACING on the 2.1M-triangle heightfield scene.

Workload (one step): a 1920x1080 film at 64 samples per pixel, maximum
bounce 8, Russian roulette from bounce 5, over a seeded 1024x1024-cell fractal
heightfield (2,097,152 triangles) with 2,000 spheres of log-uniform radius
0.1-2 (matte/plastic/metal/glass, roughness U(0.05, 0.6)) under a Perez sky
(turbidity 2.5, sun elevation 35 degrees).  Synthetic, generated from a fixed
seed; no dataset is read.

`value` is device-timed throughput with the scene resident in HBM; `e2e` runs
the whole job through the public API from host arrays each step (scene upload
and acceleration-structure build, render, RGBA8 read-back).  The scene and
the wavefront buffers (several hundred MB) exceed the 126 MB L2 between steps.

Multi-GPU: the passes are independent, so N ranks render N independent
replicas of the job (weak scaling, no collective on the data path).

At N=1 the line also carries the job-mix measurements (``batched``: 256 jobs
through the batch engine against the per-job renderer; ``served``: Poisson
arrival sweeps with p50/p99 latency), see :func:`batched_and_served`.

``--impl reference`` times the CPU restatement of the reference CPURenderer
(the oracle) on all host threads on a bounded row sample of the same job.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "paths/s"
CONFIG = {"workload": "terrain_2.1M_tris+2000_spheres_perez_1920x1080_pt64spp_bounce8", "resolution": [1920, 1080],
          "spp": 64, "max_bounce": 8, "min_rr": 5, "triangles": 2097152, "spheres": 2000,
          "l2": "inputs larger than L2 (scene + wavefront > 126 MB)"}


# Algorithmic bytes of one traced ray in k_trace: ray-list entry (4 B), origin
# and direction records (2 x 16 B), hit record (16 B).  BVH node and triangle
# fetches are data-dependent and not counted.
TRACE_RECORD_BYTES = 52
# Traversal is bound by instruction issue, not by HBM: its roofline is the
# fraction of the SMs' issue slots (4 warp instructions per SM per cycle) it
# uses.  Warp instructions per traced ray and DRAM bytes per traced ray come
# from an ncu capture of one whole 1-spp pass of this workload (the small case
# of the same scene, camera and rays); the bench scales them by the rays each
# launch traced and divides by the launch times it measures with CUDA events.
TRACE_WARP_INST_PER_RAY = 600.4
TRACE_DRAM_BYTES_PER_RAY = 135.1
TRACE_PROFILE = "profiles/k_trace_terrain_spheres_1080p_1spp.md"
ISSUE_SLOTS_PER_SM_CYCLE = 4
# Algorithmic bytes per item of the queue stages (fixed record sizes):
#   k_raygen            per path: state 48 (beta, radiance, meta) + ray 32 + list entries 8
#   k_sort_count        per work item: list entry 4 + meta 16 + hit 16 + key 1
#   k_sort_scatter      per work item: key 1 + list entry 4 + sorted entry 4
#   k_ray_list_ordered  per path scanned: mask 1; per ray listed: entry 4
QUEUE_BYTES = {"raygen": 88, "sort_count": 37, "sort_scatter": 9}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cells", type=int, default=1024)
    ap.add_argument("--spp", type=int, default=64)
    ap.add_argument("--bvh-builder", default="device", choices=["device", "host"],
                    help="mesh hierarchy builder of the scene commits (device: built on the GPU; host: binned SAH)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched and served job-mix measurements")
    ap.add_argument("--jobs", type=int, default=256, help="jobs of the batched mix")
    ap.add_argument("--batch-only", action="store_true",
                    help="run only the batched job mix (per-job arm and engine arm) and print its JSON object")
    ap.add_argument("--engine-only", action="store_true", help="with --batch-only: skip the per-job arm and the served sweep")
    ap.add_argument("--no-autotune", action="store_true", help="engine arm with the default wavefront shape")
    ap.add_argument("--no-large", action="store_true",
                    help="skip the large scene (10M-triangle terrain, 50k blob instances, 4096x2048 image light, 3840x2160)")
    ap.add_argument("--large-only", action="store_true", help="render only the large scene and print its JSON object")
    ap.add_argument("--large-spp", type=int, default=16,
                    help="samples per pixel of the large scene (its stated workload is 256; the default run takes 16 to stay within minutes)")
    return ap.parse_args()


def reduce_over_ranks(x, world, device, op="max"):
    """Max (or sum) of a per-rank scalar over all ranks; the identity at N=1.
    Every rank calls it at the same point with the same op."""
    if world == 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return float(t.item())


def replica_throughput(units_per_rank, seconds_per_rank, world, device):
    """Whole-job throughput of N independent replicas: the units all ranks
    processed over the slowest rank's time."""
    total_units = reduce_over_ranks(units_per_rank, world, device, "sum")
    slowest = reduce_over_ranks(seconds_per_rank, world, device, "max")
    return total_units / slowest, slowest


def build_scene(cells):
    from dayflower_b200.scene import generators as G
    from dayflower_b200.scene.compiler import compile_scene
    return compile_scene(G.terrain_spheres(cells=cells, n_spheres=2000, resolution=(1920, 1080), seed=2), layout_version=2)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    def __init__(self, index=0):
        self.index = index
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def start(self):
        def run():
            q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
                 "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
            while not self._stop.is_set():
                try:
                    out = subprocess.run(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + q, "--format=csv,noheader,nounits"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True, timeout=5).stdout.strip()
                    if out:
                        self.samples.append([x.strip() for x in out.split(",")])
                except Exception:
                    pass
                self._stop.wait(0.2)
        self._t = threading.Thread(target=run, daemon=True)
        self._t.start()

    def stop(self):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for s in self.samples for k in range(4) if len(s) > 4 + k and "Active" in s[4 + k] and "Not" not in s[4 + k]})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.samples)}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# The CPU sample: rows spread evenly over the whole image (every ROW_STRIDE-th
# row from row ROW_OFFSET), 1 sample per pixel of the same job, so that its
# mix of sky, terrain and sphere pixels is the image's own.  The 1-thread
# figure uses every third row of that sample.
ROW_STRIDE, ROW_OFFSET = 36, 18


def cpu_baseline(compiled, threads=None, stride=ROW_STRIDE, offset=ROW_OFFSET):
    """Times the oracle (the CPU restatement of CPURenderer) on a strided row sample of the job."""
    from oracle import dfo
    threads = threads or os.cpu_count() or 1
    o = dfo.OracleScene(compiled)
    rows = len(range(offset, o.height, stride))
    t0 = time.perf_counter()
    res = o.render(2, spp=1, max_bounce=CONFIG["max_bounce"], min_rr=CONFIG["min_rr"], rows=(offset, o.height), row_step=stride,
                   threads=threads)
    dt = time.perf_counter() - t0
    paths = o.width * rows
    return {"value": paths / dt, "unit": METRIC, "cores": threads, "kind": "port", "rays_per_s": res["rays"] / dt,
            "seconds": dt, "paths": paths, "rays": res["rays"],
            "sample": "%d rows (every %dth from row %d) x %d px x 1 spp of the same job: %d paths, %d rays, %.1f s on %d threads"
                      % (rows, stride, offset, o.width, paths, res["rays"], dt, threads)}


def cpu_baselines(compiled):
    """All host threads on the strided sample, and one thread on every third row of it
    (the reference CPURenderer renders on one thread, AbstractCPURenderer.java:215-246)."""
    b = cpu_baseline(compiled)
    one = cpu_baseline(compiled, threads=1, stride=3 * ROW_STRIDE)
    b["one_thread"] = {k: one[k] for k in ("value", "rays_per_s", "seconds", "paths", "rays", "sample")}
    return b


def batched_and_served(args, device=0):
    """The job-mix workloads on one GPU.

    Batched: 256 path-tracing jobs (square resolutions log-uniform 64^2 ..
    1024^2, spp in {1, 4, 16, 64}, maximum bounce in {4, 8, 20}) over eight
    seeded scenes (10 .. 10k spheres, 10k .. 2M-triangle heightfields, point,
    spot and area lights), rendered (a) one job at a time through the per-job
    GPURenderer, each scene resident on its own handle, and (b) all submitted
    at once to the RenderEngine (FIFO segments) after its autotuner picked the
    wavefront shape on 32 of the jobs.  Both arms end with every job's RGBA8
    image read back to the host.

    Served: Poisson arrival streams of the same jobs at rates 10 .. 500 jobs/s
    into the running engine, with round-robin and with shortest-first segment
    order; latency is submit to done at the job's own spp, reported for all
    jobs and for the 64-spp ones.  The per-job comparison serves the same
    arrivals live with one renderer, one job at a time in arrival order.
    """
    import numpy as np
    from dayflower_b200 import GPURenderer, RenderEngine
    from dayflower_b200 import serve as SV
    from dayflower_b200.scene import generators as G
    from dayflower_b200.scene.compiler import compile_scene

    scenes = [compile_scene(G.job_mix_scene(i), layout_version=2) for i in range(8)]
    jobs = G.job_mix(args.jobs)
    paths = float(sum(j["width"] * j["height"] * j["samples"] for j in jobs))

    # (a) per-job renderer
    handles = []
    for cs in scenes:
        h = GPURenderer(device=device)
        h.setScene(cs)
        handles.append(h)
    cams = [np.array(cs.arrays["cameraArray"], dtype=np.float32) for cs in scenes]

    def plain(js):
        times = []
        for j in js:
            t0 = time.perf_counter()
            h = handles[j["scene"]]
            c = cams[j["scene"]].copy()
            c[17], c[18] = j["width"], j["height"]
            h.updateCamera(c)
            h.setImage(j["width"], j["height"])
            h.setMaximumBounce(j["maximum_bounce"])
            h.setSeed(j["seed"])
            h.setup()
            h.render(j["samples"])
            h.getImage()
            times.append(time.perf_counter() - t0)
        return times

    service, t_plain, plain_launches = None, None, None
    if not args.engine_only:
        plain(jobs[:4])
        t0 = time.perf_counter()
        service = plain(jobs)
        t_plain = time.perf_counter() - t0
        plain_launches = sum(h.getCounters()["launches"] for h in handles)
    for h in handles:
        h.dispose()

    # (b) engine
    eng = RenderEngine(device=device)
    try:
        ids = [eng.add_scene(cs) for cs in scenes]
        del ids
        tuned = eng.config() if args.no_autotune else eng.autotune(jobs[:32])
        eng.configure(**dict(tuned, policy=1))
        warm = [eng.submit(**j) for j in jobs[:4]]
        eng.run()
        for k in warm:
            eng.release(k)
        s0 = eng.stats()
        t0 = time.perf_counter()
        ks = [eng.submit(**j) for j in jobs]
        eng.run()
        imgs = [eng.image(k) for k in ks]
        t_eng = time.perf_counter() - t0
        s1 = eng.stats()
        for k in ks:
            eng.release(k)
        batched = {
            "workload": "job mix: %d PT jobs over 8 seeded scenes, 64^2..1024^2, spp {1,4,16,64}, bounce {4,8,20}" % len(jobs),
            "jobs": len(jobs), "paths": paths, "engine_paths_per_s": paths / t_eng, "engine_s": t_eng,
            "engine_rays_per_s": (s1["rays"] - s0["rays"]) / t_eng,
            "plain_per_job_paths_per_s": paths / t_plain if t_plain else None, "plain_per_job_s": t_plain,
            "speedup_vs_plain_per_job": t_plain / t_eng if t_plain else None,
            "engine_config": eng.config(), "engine_gpu_launches": s1["kernel_launches"] - s0["kernel_launches"],
            "plain_gpu_launches": plain_launches, "image_bytes_read": int(sum(x.nbytes for x in imgs)),
            "timing": "wall clock over submit -> all RGBA8 images on the host, both arms",
        }
        if args.engine_only or args.batch_only:
            return batched, None
        # served: Poisson arrivals into the running engine, round-robin and shortest-first segment
        # orders, against one per-job renderer serving the same arrivals live
        served = []
        lams = (10, 25, 50, 100, 250, 500)
        arrivals = {lam: SV.poisson_arrivals(lam, min(len(jobs), max(16, int(4 * lam))), seed=lam) for lam in lams}
        subsets = {lam: [jobs[i % len(jobs)] for i in range(len(arrivals[lam]))] for lam in lams}

        def pct(lat, sub, which):
            """Latency percentiles of all jobs, the 64-spp jobs (all <= 1024^2) or the small ones (<= 256^2)."""
            if which == "all":
                x = lat
            elif which == "spp64":
                x = lat[np.array([j["samples"] == 64 and j["width"] * j["height"] <= 1024 * 1024 for j in sub])]
            else:
                x = lat[np.array([j["width"] * j["height"] <= 256 * 256 for j in sub])]
            return SV.percentiles(x) if len(x) else {"p50_s": None, "p99_s": None}

        def row(lat, sub):
            out = {}
            for which in ("all", "spp64", "small"):
                p = pct(lat, sub, which)
                pre = "" if which == "all" else which + "_"
                out[pre + "p50_s"], out[pre + "p99_s"] = p["p50_s"], p["p99_s"]
            return out

        for policy in (0, 2):
            eng.configure(**dict(tuned, policy=policy))
            eng.start()
            for lam in lams:
                sub, arr = subsets[lam], arrivals[lam]
                r = SV.run_served(eng, sub, arr)
                served.append(dict({"policy": "round_robin" if policy == 0 else "shortest_first", "lambda_per_s": lam, "jobs": len(sub),
                                    "spp64_jobs": int(sum(j["samples"] == 64 for j in sub)),
                                    "small_jobs": int(sum(j["width"] * j["height"] <= 256 * 256 for j in sub)),
                                    "paths_per_s": r["paths_per_s"], "states": r["states"]}, **row(r["latency_s"], sub)))
            eng.stop()
    finally:
        eng.close()
    # the per-job comparison, live: one GPURenderer per scene, one job at a time in arrival order
    live = []
    if not args.engine_only:
        handles = []
        for cs in scenes:
            h = GPURenderer(device=device)
            h.setScene(cs)
            handles.append(h)

        def render_one(j):
            h = handles[j["scene"]]
            c = cams[j["scene"]].copy()
            c[17], c[18] = j["width"], j["height"]
            h.updateCamera(c)
            h.setImage(j["width"], j["height"])
            h.setMaximumBounce(j["maximum_bounce"])
            h.setSeed(j["seed"])
            h.setup()
            h.render(j["samples"])
            h.getImage()

        render_one(jobs[0])
        for lam in lams:
            sub, arr = subsets[lam], arrivals[lam]
            lat = SV.run_per_job_served(render_one, sub, arr)
            live.append(dict({"lambda_per_s": lam, "jobs": len(sub)}, **row(lat, sub)))
        for h in handles:
            h.dispose()
    return batched, {"latency": "submit -> done at the job's spp (engine clock); spp64: the 64-spp jobs (all <= 1024^2); "
                                "small: jobs of <= 256^2 pixels",
                     "round_robin": "every admitted job one 64K-path segment in turn",
                     "shortest_first": "the next segment to the admitted job with the fewest paths left",
                     "sweep": served,
                     "plain_per_job_live": {"how": "one GPURenderer serving the same arrivals one job at a time in arrival order, "
                                                   "latency arrival -> RGBA8 image on the host", "sweep": live}}


def large_scene_run(args, device=0):
    """The large single scene, one job through the per-job renderer: a
    9,999,392-triangle fractal terrain plus 50,000 instances of a 5,120-triangle
    seeded blob (Disney materials), an ImageLight of a seeded 4096x2048 HDR
    environment with a 0.5 degree sun of radiance 5e4; 3840x2160 film,
    PATH_TRACING, maximum bounce 20, Russian roulette from bounce 5.  Timed
    region: render(spp) with the scene resident (device events); the scene
    upload and acceleration build are reported separately."""
    from dayflower_b200 import GPURenderer, RenderingAlgorithm
    from dayflower_b200.scene import generators as G
    from dayflower_b200.scene.compiler import compile_scene

    t0 = time.perf_counter()
    cs = compile_scene(G.large_scene(), layout_version=2)
    t_compile = time.perf_counter() - t0
    r = GPURenderer(device=device)
    try:
        t0 = time.perf_counter()
        r.setScene(cs)
        t_scene = time.perf_counter() - t0
        r.setRenderingAlgorithm(RenderingAlgorithm.PATH_TRACING)
        r.setMaximumBounce(20)
        r.setMinimumBounceRussianRoulette(5)
        r.setup()
        r.render(1)  # warm-up pass
        r.clear()
        spp = args.large_spp
        assert r.render(spp)
        ms = r.lastRenderMillis()
        c = r.getCounters()
        W, H = r.resolution
        img = r.getImage()
        paths = W * H * spp
        return {"workload": "large: 9,999,392-tri terrain + 50,000 x 5,120-tri blob instances, Disney, 4096x2048 image light, "
                            "3840x2160, PT %d spp, bounce 20, RR 5" % spp,
                "paths_per_s": paths / (ms / 1000.0), "rays_per_s": c["rays"] / (ms / 1000.0), "render_s": ms / 1000.0,
                "paths": paths, "rays_per_path": c["rays"] / paths, "gpu_launches": c["launches"],
                "triangles_total": cs.stats["triangles"], "instances": cs.stats["primitives"] - 1,
                "host_compile_s": t_compile, "set_scene_s": t_scene, "scene_bytes": int(cs.nbytes()),
                "image_mean": float(img[..., :3].mean()), "timing": "device events around render(spp), scene resident"}
    finally:
        r.dispose()


def run_reference(args, rank):
    """The reference arm: the CPU restatement of CPURenderer on all host threads.
    One step is the strided row sample of the job (the same sample as the
    cpu_baseline of the GPU arm); value = its paths over its time."""
    if rank != 0:
        return
    compiled = build_scene(args.cells)
    res = []
    for i in range(args.warmup + args.steps):
        r = cpu_baseline(compiled)
        if i >= args.warmup:
            res.append(r)
    paths = sum(x["paths"] for x in res)
    secs = sum(x["seconds"] for x in res)
    v = paths / secs
    line = {"metric": METRIC, "value": v, "unit": METRIC, "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1000.0 * secs / len(res), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": CONFIG, "impl": "reference",
            "rays_per_s": sum(x["rays"] for x in res) / secs,
            "cpu_baseline": {"value": v, "unit": METRIC, "cores": res[0]["cores"], "kind": "port", "sample": res[0]["sample"],
                             "step": "one step = the row sample above (not the whole 64-spp job)"},
            "e2e": {"value": v, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return
    if args.batch_only:
        if rank == 0:
            print(json.dumps(batched_and_served(args, 0)[0]), flush=True)
        return
    if args.large_only:
        if rank == 0:
            print(json.dumps(large_scene_run(args, 0)), flush=True)
        return
    import torch
    import torch.distributed as dist
    if world > 1:
        dist.init_process_group("nccl", init_method="env://", timeout=__import__("datetime").timedelta(seconds=600))
    torch.cuda.set_device(local)
    from dayflower_b200 import GPURenderer, RenderingAlgorithm

    compiled = build_scene(args.cells)
    W, H = CONFIG["resolution"]
    r = GPURenderer(device=local)
    builder = GPURenderer.BVH_DEVICE if args.bvh_builder == "device" else GPURenderer.BVH_HOST
    r.setBVHBuilder(builder)
    r.setScene(compiled)
    r.setRenderingAlgorithm(RenderingAlgorithm.PATH_TRACING)
    r.setMaximumBounce(CONFIG["max_bounce"])
    r.setMinimumBounceRussianRoulette(CONFIG["min_rr"])
    r.setSeed(0x5EED0000 + rank)
    r.setup()

    def step():
        r.clear()
        assert r.render(args.spp)
        return r.lastRenderMillis()

    for _ in range(args.warmup):
        step()
    # Per-launch device events for the roofline of the traversal kernel; they
    # stay on through the timed steps so k_trace is timed live.
    r.setStageTiming(True)
    step()
    clocks = ClockSampler(local)
    clocks.start()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    ms = []
    rays = 0
    launches = 0
    kstats = {}
    for _ in range(args.steps):
        ms.append(step())
        c = r.getCounters()
        rays += c["rays"]
        launches += c["launches"]
        for k, v in r.kernelStats().items():  # per kernel kind: device ms, launches (this call), items (since clear)
            a = kstats.setdefault(k, {"ms": 0.0, "launches": 0, "items": 0})
            for f in a:
                a[f] += v[f]
    torch.cuda.synchronize()
    clk = clocks.stop()
    paths_per_step = W * H * args.spp
    value, slowest_s = replica_throughput(paths_per_step * args.steps, sum(ms) / 1000.0, world, "cuda")
    total_ms = slowest_s * 1000.0
    rays_all = reduce_over_ranks(rays, world, "cuda", "sum")
    if world > 1:
        dist.barrier()

    # end to end through the public API from host arrays: every step uploads
    # the compiled scene (setScene builds the acceleration structure), sets up
    # the film, renders and reads the RGBA8 image back.  The renderer handle is
    # created once, as a serving process would.
    e2e = None
    if not args.no_e2e:
        h2d = compiled.nbytes()
        q = GPURenderer(device=local)
        q.setBVHBuilder(builder)
        q.setRenderingAlgorithm(RenderingAlgorithm.PATH_TRACING)
        q.setMaximumBounce(CONFIG["max_bounce"])
        q.setMinimumBounceRussianRoulette(CONFIG["min_rr"])

        parts = {"set_scene_s": 0.0, "setup_s": 0.0, "render_s": 0.0, "read_image_s": 0.0}

        def e2e_step():
            t = [time.perf_counter()]
            q.setScene(compiled)
            t.append(time.perf_counter())
            q.setup()
            t.append(time.perf_counter())
            q.render(args.spp)
            t.append(time.perf_counter())
            im = q.getImage()
            t.append(time.perf_counter())
            for k, a_, b_ in zip(parts, t, t[1:]):
                parts[k] += b_ - a_
            return im

        e2e_step()  # warm-up
        for k in parts:
            parts[k] = 0.0
        if world > 1:
            dist.barrier()
        e_steps = 2
        t0 = time.perf_counter()
        for _ in range(e_steps):
            img = e2e_step()
        dt = time.perf_counter() - t0
        commit_ms = q.commitMillis()
        e2e_value, _ = replica_throughput(paths_per_step * e_steps, dt, world, "cuda")
        q.dispose()
        e2e = {"value": e2e_value, "unit": METRIC, "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(img.nbytes), "steps": e_steps,
               "per_step_s": {k: v / e_steps for k, v in parts.items()}, "last_commit_ms": commit_ms,
               "note": "per step: setScene from host arrays (upload + acceleration build) + setup + render(%d) + RGBA8 read-back" % args.spp}

    if rank == 0:
        peak, peak_kind = peaks()
        tr = kstats["trace"]
        rays_per_launch = tr["items"] / tr["launches"]
        launch_ms = tr["ms"] / tr["launches"]
        hbm_achieved = rays_per_launch * TRACE_RECORD_BYTES / (launch_ms / 1000.0) / 1e9
        # issue-slot roofline of the traversal at the SM clock measured during the timed steps
        sms = torch.cuda.get_device_properties(local).multi_processor_count
        f_hz = (clk["sm_mhz"] or 1965.0) * 1e6
        issue_peak = ISSUE_SLOTS_PER_SM_CYCLE * sms * f_hz / 1e9
        issue_achieved = rays_per_launch * TRACE_WARP_INST_PER_RAY / (launch_ms / 1000.0) / 1e9

        def queue(name, nbytes):
            k = kstats[name]
            if not k["launches"] or k["ms"] <= 0.0:
                return None
            gbs = nbytes / (k["ms"] / 1000.0) / 1e9
            return {"achieved": gbs, "unit": "GB/s", "frac": gbs / peak, "launches": k["launches"], "ms": k["ms"],
                    "items": k["items"], "bytes": nbytes, "share": k["ms"] / total_ms}

        rl = kstats["ray_list"]
        stages = {n: queue(n, kstats[n]["items"] * QUEUE_BYTES[n]) for n in ("raygen", "sort_count", "sort_scatter")}
        stages["ray_list"] = queue("ray_list", rl["launches"] * W * H + 4 * rl["items"])
        stages["shade"] = {"ms": kstats["shade"]["ms"], "launches": kstats["shade"]["launches"], "items": kstats["shade"]["items"],
                           "share": kstats["shade"]["ms"] / total_ms}
        line = {
            "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic (seeded heightfield + spheres, no dataset)", "config": dict(CONFIG, spp=args.spp), "bvh_builder": args.bvh_builder,
            "rays_per_s": rays_all / (total_ms / 1000.0), "rays_per_path": rays / (paths_per_step * args.steps),
            "gpu_launches": launches,
            "roofline": {"bound": "issue", "kernel": "k_trace", "achieved": issue_achieved, "peak": issue_peak, "unit": "G warp-instructions/s",
                         "frac": issue_achieved / issue_peak,
                         "peak_kind": "%d issue slots x %d SMs x %.0f MHz (median SM clock of the timed steps)" % (ISSUE_SLOTS_PER_SM_CYCLE, sms, f_hz / 1e6),
                         "warp_inst_per_ray": TRACE_WARP_INST_PER_RAY,
                         "traffic": rays_per_launch * TRACE_DRAM_BYTES_PER_RAY,
                         "traffic_source": "DRAM bytes per traced ray (%.0f) and warp instructions per ray from the ncu capture of one 1-spp pass "
                                           "in %s, scaled by the rays of a launch; not measured in this run" % (TRACE_DRAM_BYTES_PER_RAY, TRACE_PROFILE),
                         "hbm": {"achieved": hbm_achieved, "peak": peak, "unit": "GB/s", "frac": hbm_achieved / peak, "peak_kind": peak_kind,
                                 "algorithmic_bytes_per_ray": TRACE_RECORD_BYTES},
                         "launches": tr["launches"], "launch_ms": launch_ms, "rays_per_launch": rays_per_launch,
                         "trace_share": tr["ms"] / total_ms},
            "queue_stages": stages,
            "clocks": clk,
            "e2e": e2e,
        }
        if not args.no_cpu:
            line["cpu_baseline"] = cpu_baselines(compiled)
    r.dispose()
    if rank == 0:
        if world == 1 and not args.no_batch:
            line["batched"], line["served"] = batched_and_served(args, local)
        if world == 1 and not args.no_large:
            line["large"] = large_scene_run(args, local)
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
