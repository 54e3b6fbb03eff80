"""Host logic of the served and batched workloads (no GPU): arrival process,
the one-job-at-a-time comparison queue, and the job-mix generator."""
import math

import numpy as np

from dayflower_b200 import serve as SV
from dayflower_b200.scene import generators as G


def test_poisson_arrivals_rate_and_order():
    a = SV.poisson_arrivals(200.0, 20000, seed=1)
    assert np.all(np.diff(a) > 0)
    assert abs(a[-1] / len(a) - 1 / 200.0) < 0.05 / 200.0 * 4


def test_fifo_latencies_queue_by_hand():
    # server busy until 3, then 3..5, then idle until 10, 10..11
    lat = SV.fifo_latencies([3.0, 2.0, 1.0], [0.0, 1.0, 10.0])
    assert np.allclose(lat, [3.0, 4.0, 1.0])


def test_percentiles():
    p = SV.percentiles(np.arange(1, 101, dtype=float))
    assert math.isclose(p["p50_s"], 50.5) and p["max_s"] == 100.0


def test_job_mix_distribution():
    jobs = G.job_mix(4096, seed=5)
    sides = np.array([j["width"] for j in jobs])
    assert sides.min() >= 64 and sides.max() <= 1024
    assert all(j["width"] == j["height"] for j in jobs)
    # log-uniform side: the median side is near sqrt(64 * 1024) = 256
    assert 220 <= np.median(sides) <= 300
    assert {j["samples"] for j in jobs} == {1, 4, 16, 64}
    assert {j["maximum_bounce"] for j in jobs} == {4, 8, 20}
    assert {j["scene"] for j in jobs} == set(range(8))
    assert G.job_mix(16, seed=3) == G.job_mix(16, seed=3)


def test_job_mix_scene_sizes():
    tris = sorted(2 * c * c for c in G.JOB_MIX_CELLS)
    assert tris[0] >= 10000 and tris[-1] == 2_000_000
    assert G.JOB_MIX_SPHERES[0] == 10 and G.JOB_MIX_SPHERES[-1] == 10000
    assert sorted(G.JOB_MIX_CELL_ORDER) == list(range(8))
    sc = G.job_mix_scene(2)
    kinds = {type(l).__name__ for l in sc.lights}
    assert kinds == {"PointLight", "SpotLight", "DiffuseAreaLight"}


def test_live_per_job_server_matches_the_fifo_queue():
    # the live comparison arm on a fake renderer: each job takes its service time, one at a time in arrival order
    import time
    service = [0.06, 0.01, 0.01, 0.05, 0.01]
    arrivals = [0.0, 0.01, 0.02, 0.2, 0.21]
    jobs = [{"service": s} for s in service]
    lat = SV.run_per_job_served(lambda j: time.sleep(j["service"]), jobs, arrivals)
    want = SV.fifo_latencies(service, arrivals)
    assert np.all(lat >= want - 1e-3)
    assert np.all(lat <= want + 0.03)
