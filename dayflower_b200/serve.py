"""Served rendering: a request loop over :class:`RenderEngine` that submits
jobs as they arrive while earlier ones are on the GPU, and the latency
statistics of such a run.

The engine admits each arrival into the running wavefront at the next bounce
iteration (round-robin or shortest-first over admitted jobs), so a job's
latency to its target spp is its queueing plus its share of the device.  For
comparison, :func:`run_per_job_served` serves the same arrivals live with one
per-job renderer (one job on the GPU at a time, in arrival order), and
:func:`fifo_latencies` computes that from measured per-job render times.
"""
from __future__ import annotations

import threading
import time
from typing import Dict, List, Sequence

import numpy as np


def poisson_arrivals(rate_per_s: float, n: int, seed: int = 0) -> np.ndarray:
    """Arrival times (seconds from 0) of n jobs of a Poisson process."""
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1.0 / rate_per_s, size=n))


def run_served(engine, jobs: Sequence[dict], arrivals: Sequence[float], timeout_s: float = 600.0,
               release: bool = True) -> Dict[str, object]:
    """Submits jobs[i] at arrivals[i] (seconds after the call) to a started
    engine from a client thread, waits for all of them and returns per-job
    latencies (engine clock, submit to done) and the run's throughput."""
    ids: List[int] = [0] * len(jobs)
    err: List[BaseException] = []

    def client():
        t0 = time.perf_counter()
        try:
            for i, (job, at) in enumerate(zip(jobs, arrivals)):
                d = at - (time.perf_counter() - t0)
                if d > 0:
                    time.sleep(d)
                ids[i] = engine.submit(**job)
        except BaseException as ex:  # reported to the caller
            err.append(ex)

    t_start = time.perf_counter()
    th = threading.Thread(target=client)
    th.start()
    th.join()
    if err:
        raise err[0]
    for i in ids:
        engine.wait(i, timeout_s=timeout_s)
    wall = time.perf_counter() - t_start
    infos = [engine.info(i) for i in ids]
    if release:
        for i in ids:
            engine.release(i)
    lat = np.array([x["done_s"] - x["submit_s"] for x in infos])
    paths = float(sum(x["paths_total"] for x in infos))
    states = {x["state"] for x in infos}
    return {"latency_s": lat, "paths": paths, "wall_s": wall, "paths_per_s": paths / wall, "states": sorted(states)}


def run_per_job_served(render_one, jobs: Sequence[dict], arrivals: Sequence[float]) -> np.ndarray:
    """The per-job comparison, run live: a client thread delivers jobs[i] at
    arrivals[i] into a queue, and one server (this thread, one GPURenderer
    job at a time, as ``render_one(job)`` renders it to its RGBA8 image)
    takes them in arrival order.  Returns each job's latency (arrival to its
    image on the host), in seconds."""
    import queue
    q: "queue.Queue" = queue.Queue()
    lat = np.zeros(len(jobs))
    t0 = time.perf_counter()

    def client():
        for i, at in enumerate(arrivals):
            d = at - (time.perf_counter() - t0)
            if d > 0:
                time.sleep(d)
            q.put((i, time.perf_counter()))
        q.put(None)

    th = threading.Thread(target=client)
    th.start()
    while True:
        item = q.get()
        if item is None:
            break
        i, t_arrival = item
        render_one(jobs[i])
        lat[i] = time.perf_counter() - t_arrival
    th.join()
    return lat


def fifo_latencies(service_s: Sequence[float], arrivals: Sequence[float]) -> np.ndarray:
    """Latencies (arrival to finish) of one server that renders jobs one at a
    time in arrival order, each taking service_s[i]."""
    free_at = 0.0
    out = np.empty(len(service_s))
    for i, (s, a) in enumerate(zip(service_s, arrivals)):
        start = max(free_at, a)
        free_at = start + s
        out[i] = free_at - a
    return out


def percentiles(lat: np.ndarray) -> Dict[str, float]:
    return {"p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)), "max_s": float(np.max(lat)),
            "mean_s": float(np.mean(lat))}
