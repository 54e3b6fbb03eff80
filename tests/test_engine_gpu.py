"""Batch and serving engine (RenderEngine) on the device.

A job's samples use the same counter-based random numbers as the per-job
renderer for the same seed, so its film must match a GPURenderer render of the
same scene, and must be the same alone and in a mix of other jobs, up to the
order of the film's float additions (rtol 1e-4).  Against the CPU oracle the
engine is held to the path-tracing criterion: >= 99% of pixels pass the
two-sample 3-sigma test at equal spp.
"""
import threading
import time

import numpy as np
import pytest

from dayflower_b200 import RenderEngine
from dayflower_b200 import RenderingAlgorithm as RA
from dayflower_b200.scene import generators as G
from dayflower_b200.scene.compiler import compile_scene

from . import parity as PT

pytestmark = pytest.mark.gpu

FILM_RTOL = 1e-4


@pytest.fixture(scope="module")
def scenes():
    return {
        "cornell": compile_scene(G.cornell_box(resolution=(96, 96))),
        "mixed": compile_scene(G.small_mixed_scene(resolution=(80, 48)), layout_version=2),
        "quadrics": compile_scene(G.quadrics_scene(resolution=(64, 48))),
        "terrain": compile_scene(G.terrain_spheres(cells=64, n_spheres=100, resolution=(72, 40), seed=5), layout_version=2),
    }


@pytest.fixture(scope="module")
def engine(scenes):
    e = RenderEngine()
    e.configure(capacity=1 << 15, iterations_per_launch=4)  # small pool: slots are refilled many times per job
    ids = {k: e.add_scene(v) for k, v in scenes.items()}
    yield e, ids
    e.close()


def res_of(cs):
    cam = cs.arrays["cameraArray"]
    return int(cam[17]), int(cam[18])


def films_close(a, b):
    (sa, qa, na), (sb, qb, nb) = a, b
    assert np.array_equal(na, nb), "sample counts differ"
    assert np.allclose(sa, sb, rtol=FILM_RTOL, atol=1e-5)
    assert np.allclose(qa, qb, rtol=FILM_RTOL, atol=1e-5)


def run_alone(e, sid, w, h, spp, bounce, seed):
    j = e.submit(sid, w, h, spp, maximum_bounce=bounce, seed=seed)
    e.run(timeout_s=120)
    assert e.info(j)["state"] == "done"
    f = e.film(j)
    e.release(j)
    return f


@pytest.mark.parametrize("name", ["cornell", "mixed", "quadrics"])
def test_engine_job_matches_per_job_renderer(engine, scenes, name):
    e, ids = engine
    cs = scenes[name]
    w, h = res_of(cs)
    g = PT.render_gpu(cs, RA.PATH_TRACING, spp=6, max_bounce=8, seed=77)
    f = run_alone(e, ids[name], w, h, 6, 8, 77)
    films_close(f, (g["sum"], g["sumsq"], g["count"]))


@pytest.mark.parametrize("name", ["cornell", "mixed", "quadrics"])
@pytest.mark.parametrize("kind,algorithm", [(1, RA.RAY_CASTING), (2, RA.DEPTH_CAMERA), (3, RA.AMBIENT_OCCLUSION), (4, RA.RAY_TRACING)])
def test_engine_one_step_jobs_match_per_job_renderer(engine, scenes, name, kind, algorithm):
    # RAY_CASTING and DEPTH_CAMERA jobs end at their camera ray; AMBIENT_OCCLUSION and RAY_TRACING trace their
    # occlusion rays or ray tree in one step; each sample is the per-job renderer's (GPURenderer.java:65-77)
    from dayflower_b200.engine import JOB_AMBIENT_OCCLUSION, JOB_DEPTH_CAMERA, JOB_RAY_CASTING, JOB_RAY_TRACING
    assert (JOB_RAY_CASTING, JOB_DEPTH_CAMERA, JOB_AMBIENT_OCCLUSION, JOB_RAY_TRACING) == (1, 2, 3, 4)
    e, ids = engine
    cs = scenes[name]
    w, h = res_of(cs)
    g = PT.render_gpu(cs, algorithm, spp=3, seed=91, max_bounce=8, ao_samples=12, ao_distance=30.0)
    others = [e.submit(ids["terrain"], 32, 24, 2, maximum_bounce=4, seed=5)]  # shares the wavefront with a path-traced job
    j = e.submit(ids[name], w, h, 3, seed=91, kind=kind, maximum_bounce=8, ambient_occlusion_samples=12, maximum_distance=30.0)
    e.run(timeout_s=120)
    assert e.info(j)["state"] == "done"
    f = e.film(j)
    e.release(j)
    for o in others:
        e.release(o)
    films_close(f, (g["sum"], g["sumsq"], g["count"]))


def test_engine_job_same_alone_and_in_mix(engine, scenes):
    e, ids = engine
    w, h = res_of(scenes["cornell"])
    alone = run_alone(e, ids["cornell"], w, h, 8, 20, 1234)
    # the same job between others of different scenes, sizes, spp and bounce limits
    others = [e.submit(ids["terrain"], 72, 40, 4, maximum_bounce=4, seed=9),
              e.submit(ids["quadrics"], 50, 30, 3, maximum_bounce=20, seed=10),
              e.submit(ids["mixed"], 33, 17, 16, maximum_bounce=8, seed=11)]
    j = e.submit(ids["cornell"], w, h, 8, maximum_bounce=20, seed=1234)
    others += [e.submit(ids["terrain"], 128, 64, 2, maximum_bounce=8, seed=12)]
    e.run(timeout_s=120)
    for k in others + [j]:
        assert e.info(k)["state"] == "done"
    films_close(e.film(j), alone)
    for k in others + [j]:
        e.release(k)


@pytest.mark.parametrize("name,spp", [("cornell", 16), ("terrain", 8)])
def test_engine_against_oracle(engine, scenes, name, spp):
    e, ids = engine
    cs = scenes[name]
    w, h = res_of(cs)
    s, q, n = run_alone(e, ids[name], w, h, spp, 8, 0x5EED1234)
    o = PT.render_oracle(cs, RA.PATH_TRACING, spp=spp, max_bounce=8)
    ok, mg, mo = PT.sigma_test({"sum": s, "sumsq": q, "count": n}, o)
    assert ok >= PT.PIXEL_PASS, "3-sigma pass rate %.4f" % ok
    assert abs(mg.mean() - mo.mean()) <= 0.02 * max(mo.mean(), 1e-3) + 1e-4


def test_served_jobs_arriving_while_others_run(scenes):
    e = RenderEngine()
    try:
        e.configure(capacity=1 << 16, iterations_per_launch=2)
        sid = e.add_scene(scenes["cornell"])
        tid = e.add_scene(scenes["terrain"])
        w, h = res_of(scenes["cornell"])
        ref = run_alone(e, sid, w, h, 12, 20, 4321)
        e.start()
        first = e.submit(tid, 256, 256, 32, maximum_bounce=8, seed=3)  # keeps the wavefront busy
        ids, errors = [], []

        def client(k):
            try:
                time.sleep(0.005 * k)
                ids.append(e.submit(sid, w, h, 12, maximum_bounce=20, seed=4321))
            except Exception as ex:  # pragma: no cover - reported below
                errors.append(ex)

        threads = [threading.Thread(target=client, args=(k,)) for k in range(4)]
        for t in threads:
            t.start()
        # a progressive image of the long job while it runs
        time.sleep(0.01)
        _, _, n_mid = e.film(first)
        for t in threads:
            t.join()
        assert not errors
        for k in ids + [first]:
            e.wait(k, timeout_s=120)
        e.stop()
        assert n_mid.max() <= 32
        for k in ids:
            info = e.info(k)
            assert info["state"] == "done" and info["done_s"] >= info["admit_s"] >= info["submit_s"] > 0
            films_close(e.film(k), ref)
        _, _, n_end = e.film(first)
        assert np.all(n_end <= 32) and n_end.sum() > 0
        st = e.stats()
        assert st["paths_retired"] >= sum(e.info(k)["paths_total"] for k in ids + [first])
        assert st["overflow"] == 0
    finally:
        e.close()


def test_cancel_and_budget_admission(scenes):
    cs = scenes["cornell"]
    probe = RenderEngine()
    probe.configure(capacity=1 << 14)
    sid = probe.add_scene(cs)
    used0 = None
    try:
        j = probe.submit(sid, 8, 8, 1)
        probe.run(timeout_s=60)
        used0 = probe.stats()["device_bytes_used"] - 8 * 8 * 32  # wavefront + scene
    finally:
        probe.close()
    film = 200 * 200 * 32
    e = RenderEngine(memory_budget_bytes=used0 + int(1.5 * film))  # room for one 200x200 film at a time
    try:
        e.configure(capacity=1 << 14)
        sid = e.add_scene(cs)
        e.start()
        a = e.submit(sid, 200, 200, 4, maximum_bounce=6, seed=1)
        b = e.submit(sid, 200, 200, 4, maximum_bounce=6, seed=2)
        e.wait(a, timeout_s=120)
        time.sleep(0.05)
        assert e.info(b)["state"] == "queued"  # a's film still holds the budget
        e.release(a)
        e.wait(b, timeout_s=120)
        assert e.info(b)["state"] == "done"
        e.release(b)
        # cancellation: a long job ends as cancelled with part of its paths done
        c = e.submit(sid, 200, 200, 4096, maximum_bounce=20, seed=3)
        time.sleep(0.05)
        e.cancel(c)
        e.wait(c, timeout_s=120)
        info = e.info(c)
        assert info["state"] == "cancelled"
        e.release(c)
        e.stop()
    finally:
        e.close()


def test_engine_rejects_bad_jobs(engine):
    e, ids = engine
    with pytest.raises(ValueError):
        e.submit(63, 8, 8, 1)
    with pytest.raises(ValueError):
        e.submit(ids["cornell"], 0, 8, 1)
    with pytest.raises(ValueError):
        e.submit(ids["cornell"], 8, 8, 0)
    with pytest.raises(ValueError):
        e.submit(ids["cornell"], 8, 8, 1, kind=5)  # no such rendering algorithm
    with pytest.raises(ValueError):
        e.submit(ids["cornell"], 8, 8, 1, kind=3, ambient_occlusion_samples=0)  # setSamples out of range
