"""GPU tests of the batched multi-scene launch (pt_batch_*), its autotuner and the serving loop
(pt_server_*): every film must equal pt_render's for the same scene and description, bit for bit,
alone or in any mix."""
import time

import numpy as np
import pytest

from conftest import assert_bit_equal
import polytope_b200 as pb
from polytope_b200 import workloads as W

pytestmark = pytest.mark.gpu


def small_jobs(n=10, seed=5):
    work = W.batched_workload(n, seed=seed, min_tris=500, max_tris=30_000, resolutions=(16, 24, 40), spps=(1, 3, 4))
    jobs = []
    for k, (meshes, env, d) in enumerate(work):
        scene = pb.Scene(meshes, env)
        flags = pb.RENDER_NEE | (pb.RENDER_JITTER if k % 2 else 0)
        rd = pb.render_desc(d["width"], d["height"], d["spp"], d["max_depth"], d["camera"], d["seed"], flags)
        jobs.append((scene, rd))
    return jobs


def solo(scene, rd):
    return pb.render(scene, rd.width, rd.height, rd.spp, rd.max_depth,
                     dict(eye=tuple(rd.camera.eye), look_at=tuple(rd.camera.look_at), up=tuple(rd.camera.up),
                          fov=rd.camera.fov_deg), rd.seed, rd.flags)


@pytest.mark.parametrize("pipeline", [0, 1, 2], ids=["fused", "wavefront", "paths"])
def test_batch_films_equal_solo_renders(cuda_device, pipeline):
    jobs = small_jobs()
    t = pb.default_tuning()
    t.pipeline = pipeline
    b = pb.Batch(jobs, t)
    b.run()
    for i, (scene, rd) in enumerate(jobs):
        rgb, prim = b.output(i)
        srgb, sprim = solo(scene, rd)
        assert_bit_equal(rgb, srgb, f"film {i}")
        assert_bit_equal(prim, sprim, f"prim {i}")
    assert b.rays_traced() > sum(rd.width * rd.height * rd.spp for _, rd in jobs)
    b.run()  # graph replay gives the same films
    assert_bit_equal(b.output(3)[0], solo(*jobs[3])[0], "replay")


def test_batch_tunings_and_autotune(cuda_device):
    jobs = small_jobs(6, seed=9)
    ref = [solo(s, rd)[0] for s, rd in jobs]
    for tpb, chunk, stack, wave, pipe in ((64, 32, 0, 0, 0), (256, 128, 64, 1000, 0), (128, 64, 48, 3000, 0),
                                          (128, 64, 0, 0, 1), (64, 32, 32, 700, 1), (256, 128, 64, 5000, 1),
                                          (128, 64, 0, 0, 2), (64, 32, 24, 900, 2)):
        t = pb.BatchTuning(wave, tpb, stack, chunk, pipe)
        b = pb.Batch(jobs, t)
        b.run()
        for i in range(len(jobs)):
            assert_bit_equal(b.output(i)[0], ref[i], f"tuning {tpb}/{chunk}/{stack}/{wave} item {i}")
    best, ms, trials = pb.autotune(jobs)
    assert ms > 0 and len(trials) >= 5
    assert best.threads_per_block in (64, 128, 256) and best.queue_chunk % 32 == 0
    b = pb.Batch(jobs, best)
    b.run()
    assert_bit_equal(b.output(0)[0], ref[0], "autotuned")


def tuning(pipeline):
    t = pb.default_tuning()
    t.pipeline = pipeline
    return t


@pytest.mark.parametrize("policy", [pb.SERVE_OLDEST_FIRST, pb.SERVE_FAIR_SHARE], ids=["oldest", "fair"])
@pytest.mark.parametrize("pipeline", [0, 1, 2], ids=["fused", "wavefront", "paths"])
def test_server_results_same_alone_and_in_the_mix(cuda_device, pipeline, policy):
    jobs = small_jobs(12, seed=13)
    srv = pb.Server(max_inflight=64, wave_pixels=2048, tuning=tuning(pipeline), policy=policy)
    alone = []
    for scene, rd in jobs:  # one request at a time
        t = srv.submit(scene, rd)
        assert srv.wait(t, 60000) == 2
        alone.append(srv.fetch(t))
    tickets = [srv.submit(scene, rd) for scene, rd in jobs]  # all at once: interleaved waves
    for t, (a_rgb, a_prim), (scene, rd) in zip(tickets, alone, jobs):
        assert srv.wait(t, 60000) == 2
        st, lat = srv.poll(t)
        assert st == 2 and lat >= 0
        tm = srv.timing(t)
        assert 0 <= tm["admitted_ms"] <= tm["first_wave_ms"] <= tm["last_wave_ms"] <= tm["done_ms"]
        assert abs(tm["done_ms"] - lat) < 1e-6
        rgb, prim = srv.fetch(t)
        assert_bit_equal(rgb, a_rgb, "mix vs alone")
        assert_bit_equal(prim, a_prim, "mix vs alone prim")
        assert_bit_equal(rgb, solo(scene, rd)[0], "server vs pt_render")
    s = srv.stats()
    assert s["completed"] == 24 and s["waves"] >= 12 and s["rays_traced"] > 0 and s["device_bytes_in_use"] == 0
    assert s["host_bytes_in_use"] == 0 and s["waves_launched"] == s["waves"] and s["busy_ms"] > 0
    assert s["plan_ms"] >= 0 and s["retire_wait_ms"] >= 0 and s["blocked_ms"] >= 0
    srv.close()


@pytest.mark.parametrize("pipeline", [0, 1, 2], ids=["fused", "wavefront", "paths"])
def test_server_admission_by_memory_budget(cuda_device, pipeline):
    jobs = small_jobs(6, seed=17)
    # budget for about one request's film at a time: admissions wait for memory to free up
    srv = pb.Server(max_inflight=8, memory_budget=40 * 40 * 28 + 4096, wave_pixels=512, tuning=tuning(pipeline))
    tickets = [srv.submit(scene, rd) for scene, rd in jobs]
    for t, (scene, rd) in zip(tickets, jobs):
        assert srv.wait(t, 60000) == 2
        assert_bit_equal(srv.fetch(t)[0], solo(scene, rd)[0], "budgeted")
    srv.close()


def test_server_host_budget_backpressure(cuda_device):
    jobs = small_jobs(6, seed=29)
    biggest = max(rd.width * rd.height for _, rd in jobs)
    # room for about two finished films: later admissions wait until earlier results are fetched
    srv = pb.Server(max_inflight=8, wave_pixels=4096, host_budget=2 * 16 * biggest + 512, tuning=tuning(pb.PIPELINE_PATHS))
    tickets = [srv.submit(scene, rd) for scene, rd in jobs]
    for t, (scene, rd) in zip(tickets, jobs):
        assert srv.wait(t, 60000) == 2
        assert_bit_equal(srv.fetch(t)[0], solo(scene, rd)[0], "host budget")
    scene, rd = jobs[0]
    small = pb.Server(max_inflight=2, host_budget=256)
    with pytest.raises(pb.PolytopeError) as e:
        small.submit(scene, rd)
    assert e.value.code == pb.PT_EINVAL and "host budget" in str(e.value)
    small.close()
    srv.close()


def test_server_poisson_arrivals_latency(cuda_device):
    jobs = small_jobs(8, seed=21)
    srv = pb.Server(max_inflight=32, wave_pixels=4096)
    rng = np.random.default_rng(19)
    tickets = []
    for i in range(40):
        time.sleep(float(rng.exponential(1.0 / 500.0)))
        scene, rd = jobs[int(rng.integers(len(jobs)))]
        tickets.append(srv.submit(scene, rd))
    lats = []
    for t in tickets:
        assert srv.wait(t, 60000) == 2
        lats.append(srv.poll(t)[1])
        srv.fetch(t)
    assert np.percentile(lats, 99) >= np.percentile(lats, 50) > 0
    srv.close()


def test_server_cancel_queued_and_in_flight_requests(cuda_device):
    """pt_server_cancel: a queued request ends at once; an admitted one stops getting work and ends
    after the waves already queued with its work; the others still finish with pt_render's films,
    and every byte of device memory and host arena goes back.  A wait that runs out returns
    PT_ETIMEOUT with the request's current state."""
    jobs = small_jobs(4, seed=31)
    meshes, env = W.instanced_scene(level=6, instances=3)
    big_scene = pb.Scene(meshes, env)
    big = pb.render_desc(1024, 1024, 16, 5, W.INSTANCED_CAMERA, 3, pb.RENDER_NEE)
    t = pb.default_tuning()
    t.pipeline = pb.PIPELINE_PATHS
    # one request at a time, small waves: the big request spans hundreds of waves
    srv = pb.Server(max_inflight=1, wave_pixels=1 << 16, tuning=t)
    ta = srv.submit(big_scene, big)
    others = [srv.submit(scene, rd) for scene, rd in jobs]
    # a wait that runs out reports the timeout and the state so far
    with pytest.raises(pb.PolytopeError) as e:
        srv.wait(ta, 1)
    assert e.value.code == pb.PT_ETIMEOUT
    # the last queued request is cancelled while the big one runs
    assert srv.poll(others[-1])[0] == pb.REQ_QUEUED
    srv.cancel(others[-1])
    assert srv.poll(others[-1])[0] == pb.REQ_CANCELLED
    assert srv.wait(others[-1], 1000) == pb.REQ_CANCELLED
    # the big request is cancelled once its first wave is queued
    deadline = time.time() + 30
    while srv.timing(ta)["first_wave_ms"] < 0 and time.time() < deadline:
        time.sleep(0.001)
    assert srv.poll(ta)[0] == pb.REQ_ADMITTED
    srv.cancel(ta)
    assert srv.wait(ta, 60000) == pb.REQ_CANCELLED
    for tk, (scene, rd) in zip(others[:-1], jobs[:-1]):
        assert srv.wait(tk, 60000) == pb.REQ_DONE
        assert_bit_equal(srv.fetch(tk)[0], solo(scene, rd)[0], "film after a cancellation")
    for tk in (ta, others[-1]):
        with pytest.raises(pb.PolytopeError) as e:
            srv.fetch(tk)
        assert e.value.code == pb.PT_ECANCELED
    s = srv.stats()
    assert s["cancelled"] == 2 and s["completed"] == len(jobs) - 1
    assert s["device_bytes_in_use"] == 0 and s["host_bytes_in_use"] == 0 and s["active"] == 0 and s["pending"] == 0
    # the big request stopped early: far fewer waves than its 16,777,216 paths would take
    assert s["waves"] < (1024 * 1024 * 16) >> 16
    # cancelling a finished or unknown request is refused
    tk = srv.submit(*jobs[0])
    assert srv.wait(tk, 60000) == pb.REQ_DONE
    with pytest.raises(pb.PolytopeError) as e:
        srv.cancel(tk)
    assert e.value.code == pb.PT_EINVAL
    srv.fetch(tk)
    with pytest.raises(pb.PolytopeError):
        srv.cancel(10 ** 9)
    srv.close()
    big_scene.close()
