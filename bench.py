"""Benchmark: the intersection microbench (plain per-frame launch of pt_trace).

Workload: a displaced icosphere subdivided 8 times (1,310,720 faces, radius 1, 3-octave value
noise amplitude 0.05, seed 7) and 16,777,216 rays (origins uniform on a radius-3 sphere,
directions toward uniform points of the unit ball, seed 11; even rays closest-hit, odd rays any-hit
with tmax = distance to the target).  One step traces every ray once.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line (rank 0).  `value` is Mrays/s with rays already in HBM (device pointers);
`e2e` is the same through the C ABI with pinned host buffers (copies inside the timed region).
`roofline.achieved` counts the reference algorithm's bytes per ray (32 B per node test, 44 B per
face test, 28 B ray in, 16 B hit out) from the per-ray test counts of one counted pass.
With N > 1 every rank traces its own full ray set against a replica of the scene (weak scaling,
no collective on the data path).
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_RAYS = 16_777_216
WORKLOAD = "intersection microbench: icosphere-8 displaced (1,310,720 tris), 16,777,216 rays (half any-hit)"


def clocks_sampler():
    """Sample SM clocks and throttle reasons with nvidia-smi while the timed region runs."""
    q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")
    idx = os.environ.get("CUDA_VISIBLE_DEVICES", "0").split(",")[0] or "0"
    try:
        p = subprocess.Popen(["nvidia-smi", f"--id={idx}", f"--query-gpu={q}", "--format=csv,noheader,nounits", "-lms", "200"],
                             stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
    except (FileNotFoundError, OSError):
        return None
    lines = []
    t = threading.Thread(target=lambda: lines.extend(iter(p.stdout.readline, "")), daemon=True)
    t.start()
    return p, lines, t


def clocks_summary(handle):
    if handle is None:
        return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
    p, lines, t = handle
    p.terminate()
    try:
        p.wait(timeout=5)
    except subprocess.TimeoutExpired:
        p.kill()
    t.join(timeout=2)
    sm, mx, reasons = [], [], set()
    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    for ln in lines:
        parts = [x.strip() for x in ln.split(",")]
        if len(parts) < 7:
            continue
        try:
            sm.append(float(parts[0]))
            mx.append(float(parts[1]))
        except ValueError:
            continue
        for nm, v in zip(names, parts[3:7]):
            if v.lower() == "active":
                reasons.add(nm)
    return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
            "reasons": sorted(reasons), "samples": len(sm)}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def profiled_traffic():
    """DRAM bytes per launch of the trace kernel from the committed ncu summary, if any."""
    try:
        with open(os.path.join(ROOT, "profiles", "trace_persistent_kernel_microbench.json")) as f:
            return json.load(f).get("dram_bytes_per_launch_full_size")
    except (OSError, ValueError):
        return None


def build_scenes(pb, specs, threads=16):
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(threads) as ex:
        return list(ex.map(lambda sp: pb.Scene(sp[0], sp[1]), specs))


def bench_batched(pb, torch, n_scenes=256):
    """256 uneven scenes: one autotuned batched launch vs one plain pt_render launch per scene, the
    plain launch both with pt_render's default pipeline (the persistent path kernel, the fastest
    single-frame launch) and with the one-thread-per-path fused kernel."""
    import ctypes as C
    from polytope_b200 import workloads as W
    work = W.batched_workload(n_scenes)
    scenes = build_scenes(pb, [(w[0], w[1]) for w in work])
    jobs = [(sc, pb.render_desc(d["width"], d["height"], d["spp"], d["max_depth"], d["camera"], d["seed"], pb.RENDER_NEE))
            for sc, (_, _, d) in zip(scenes, work)]
    fused = [(sc, pb.render_desc(d["width"], d["height"], d["spp"], d["max_depth"], d["camera"], d["seed"],
                                 pb.RENDER_NEE | pb.RENDER_FUSED)) for sc, (_, _, d) in zip(scenes, work)]
    wavefront = [(sc, pb.render_desc(d["width"], d["height"], d["spp"], d["max_depth"], d["camera"], d["seed"],
                                     pb.RENDER_NEE | pb.RENDER_WAVEFRONT)) for sc, (_, _, d) in zip(scenes, work)]
    outs = [torch.empty(rd.width * rd.height * 3, dtype=torch.float32, device="cuda") for _, rd in jobs]
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def plain(js, per_frame=None):
        # pt_render with device films only queues its work, so the events bracket the GPU time of
        # 256 back-to-back frames on the stream
        for (sc, rd), o in zip(js[:8], outs):
            pb.check(pb.lib.pt_render(sc.handle, C.byref(rd), o.data_ptr(), None, pb.MEM_DEVICE, None))
        torch.cuda.synchronize()
        marks = [torch.cuda.Event(enable_timing=True) for _ in js] if per_frame is not None else []
        e0.record()
        for k, ((sc, rd), o) in enumerate(zip(js, outs)):
            pb.check(pb.lib.pt_render(sc.handle, C.byref(rd), o.data_ptr(), None, pb.MEM_DEVICE, None))
            if marks:
                marks[k].record()
        e1.record()
        e1.synchronize()
        for sc, _ in js[:1]:
            assert sc.status() == pb.PT_OK
        if marks:
            per_frame[:] = [e0.elapsed_time(marks[0])] + [a.elapsed_time(b) for a, b in zip(marks, marks[1:])]
        return e0.elapsed_time(e1)

    frame_ms, frame_wf_ms = [], []
    plain_ms = plain(jobs, frame_ms)
    fused_ms = plain(fused)
    wavefront_ms = plain(wavefront, frame_wf_ms)
    best_pick_ms = sum(min(a, b) for a, b in zip(frame_ms, frame_wf_ms))
    best, _, trials = pb.autotune(jobs[::8])
    b = pb.Batch(jobs, best)
    b.run()
    e0.record()
    b.run()
    e1.record()
    e1.synchronize()
    batch_ms = e0.elapsed_time(e1)
    rays = b.rays_traced()
    b.close()
    # How much of the plain arm's time is the GPU left underfilled by small frames?  Each frame's
    # rays (one-item batches, untimed: the same rays as pt_render's) against its own plain time;
    # frames of at least 4,194,304 paths fill the GPU many times over and set the plain kernel's
    # full rate on these scenes.  At that rate for every frame the plain arm would take ideal_ms,
    # the most that batching alone (filling the GPU) can recover.
    frame_rays = []
    for job in jobs:
        one = pb.Batch([job])
        one.run()
        frame_rays.append(one.rays_traced())
        one.close()
    paths = [rd.width * rd.height * rd.spp for _, rd in jobs]
    big = [k for k, n in enumerate(paths) if n >= 1 << 22]
    full_rate = sum(frame_rays[k] for k in big) / sum(frame_ms[k] for k in big)  # rays per ms
    ideal_ms = sum(frame_rays) / full_rate
    small = [k for k, n in enumerate(paths) if n < 1 << 20]
    breakdown = {"frames_full_rate": len(big), "full_rate_mrays_s": round(full_rate / 1e3, 1),
                 "plain_ideal_ms": round(ideal_ms, 2), "batching_bound": round(plain_ms / ideal_ms, 3),
                 "batched_vs_ideal": round(ideal_ms / batch_ms, 3),
                 "small_frames": len(small), "small_frames_rays_share": round(sum(frame_rays[k] for k in small) / sum(frame_rays), 4),
                 "small_frames_time_share": round(sum(frame_ms[k] for k in small) / sum(frame_ms), 4),
                 "frame_rays_sum_equals_batch": sum(frame_rays) == rays}
    return {"workload": f"{n_scenes} scenes (displaced icosphere + boxes, 1k-500k tris log-uniform), 64^2-512^2, 4/16/64 spp, depth 6, NEE",
            "tris": int(sum(sum(len(m.faces) for m in w[0]) for w in work)),
            "paths": int(sum(rd.width * rd.height * rd.spp for _, rd in jobs)), "rays": int(rays),
            "plain_ms": round(plain_ms, 2), "plain_mrays_s": round(rays / plain_ms / 1e3, 1),
            "plain_fused_ms": round(fused_ms, 2), "plain_fused_mrays_s": round(rays / fused_ms / 1e3, 1),
            "plain_wavefront_ms": round(wavefront_ms, 2), "plain_wavefront_mrays_s": round(rays / wavefront_ms / 1e3, 1),
            "plain_best_pick_ms": round(best_pick_ms, 2), "plain_best_pick_mrays_s": round(rays / best_pick_ms / 1e3, 1),
            "speedup_vs_best_pick_plain": round(best_pick_ms / batch_ms, 3),
            "batched_ms": round(batch_ms, 2), "batched_mrays_s": round(rays / batch_ms / 1e3, 1),
            "speedup": round(plain_ms / batch_ms, 3), "speedup_vs_fused_plain": round(fused_ms / batch_ms, 3),
            "tuning": best.as_dict(), "autotune_trials": len(trials),
            "plain_underfill": breakdown,
            "timing": "CUDA events around 256 sequential pt_render calls (device films; default pipeline = persistent "
                      "path kernel, PT_RENDER_FUSED and PT_RENDER_WAVEFRONT) and around one batch graph replay; best pick: "
                      "per frame the faster of the default and the wavefront pipeline; plain_underfill: an event after "
                      "each plain call (default pipeline), frames of >= 4,194,304 paths set the full rate"}


def bench_render(pb, torch, cpu=True, cpu_rows=16, threads=None):
    """Full path trace of the instanced scene (6,553,602 tris, 1920x1080, 64 spp, depth 8, NEE):
    the plain pt_render launch vs the autotuned wave engine on the same frame (a one-item batch),
    and the film against the reference's CPU render of a band of rows at equal spp."""
    import ctypes as C
    from polytope_b200 import workloads as W
    meshes, env = W.instanced_scene()
    d = dict(W.INSTANCED_RENDER)
    scene = pb.Scene(meshes, env)
    rd = pb.render_desc(d["width"], d["height"], d["spp"], d["max_depth"], d["camera"], d["seed"], pb.RENDER_NEE)
    npix = rd.width * rd.height
    samples = npix * rd.spp
    out = torch.empty(npix * 3, dtype=torch.float32, device="cuda")
    prim = torch.empty(npix, dtype=torch.int32, device="cuda")
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed(fn, reps=3):
        fn()
        torch.cuda.synchronize()
        ts = []
        for _ in range(reps):
            e0.record()
            fn()
            e1.record()
            e1.synchronize()
            ts.append(e0.elapsed_time(e1))
        return statistics.median(ts)

    rd_fused = pb.render_desc(d["width"], d["height"], d["spp"], d["max_depth"], d["camera"], d["seed"],
                              pb.RENDER_NEE | pb.RENDER_FUSED)
    fused_ms = timed(lambda: pb.check(pb.lib.pt_render(scene.handle, C.byref(rd_fused), out.data_ptr(), prim.data_ptr(),
                                                       pb.MEM_DEVICE, None)))
    fused_film = out.view(rd.height, rd.width, 3).cpu().numpy()
    plain_ms = timed(lambda: pb.check(pb.lib.pt_render(scene.handle, C.byref(rd), out.data_ptr(), prim.data_ptr(),
                                                       pb.MEM_DEVICE, None)))
    film = out.view(rd.height, rd.width, 3).cpu().numpy()
    prim_ids = prim.view(rd.height, rd.width).cpu().numpy().view(np.uint32)
    assert scene.status() == pb.PT_OK
    # the same frame on the two-level (instanced) layout: one copy of the sphere instead of five
    two = pb.Scene(meshes, env, two_level=True)
    two_ms = timed(lambda: pb.check(pb.lib.pt_render(two.handle, C.byref(rd), out.data_ptr(), prim.data_ptr(),
                                                     pb.MEM_DEVICE, None)))
    two_film = out.view(rd.height, rd.width, 3).cpu().numpy().astype(np.float64)
    two_prim = prim.view(rd.height, rd.width).cpu().numpy().view(np.uint32)
    f64 = film.astype(np.float64)
    two_level = {"ms": round(two_ms, 2), "msamples_s": round(samples / two_ms / 1e3, 1), "pipeline": "fused (two-level scenes)",
                 "device_bytes": int(two.info().device_bytes), "flattened_device_bytes": int(scene.info().device_bytes),
                 "memory_ratio": round(scene.info().device_bytes / two.info().device_bytes, 2),
                 "rel_rmse_vs_flattened": float(np.sqrt(((two_film - f64) ** 2).mean()) / np.sqrt((f64 ** 2).mean())),
                 "primary_ids_equal_frac": float((two_prim == prim_ids).mean())}
    two.close()
    best, _, trials = pb.autotune([(scene, rd)])
    b = pb.Batch([(scene, rd)], best)
    tuned_ms = timed(b.run)
    rays = b.rays_traced()
    tuned_film, tuned_prim = b.output(0)
    b.close()
    res = {"workload": "instanced displaced spheres (5 x 1,310,720 + 2 tris), 1920x1080, 64 spp, depth 8, NEE",
           "samples": samples, "rays": int(rays),
           "plain": {"ms": round(plain_ms, 2), "msamples_s": round(samples / plain_ms / 1e3, 1), "mrays_s": round(rays / plain_ms / 1e3, 1),
                     "pipeline": "pt_render default (persistent path kernel)"},
           "plain_fused": {"ms": round(fused_ms, 2), "msamples_s": round(samples / fused_ms / 1e3, 1),
                           "mrays_s": round(rays / fused_ms / 1e3, 1), "pipeline": "PT_RENDER_FUSED",
                           "film_equals_plain": bool(np.array_equal(fused_film.view(np.uint32), film.view(np.uint32)))},
           "autotuned": {"ms": round(tuned_ms, 2), "msamples_s": round(samples / tuned_ms / 1e3, 1),
                         "mrays_s": round(rays / tuned_ms / 1e3, 1), "tuning": best.as_dict(), "trials": len(trials)},
           "two_level": two_level,
           "autotuned_equals_plain": bool(np.array_equal(tuned_film.view(np.uint32), film.view(np.uint32))
                                          and np.array_equal(tuned_prim, prim_ids)),
           "timing": "CUDA events, median of 3 after one warm-up; films stay on the device"}
    if cpu:
        from oracle import pyoracle as po
        threads = threads or os.cpu_count() or 1
        kind = "reference" if po.ref_available() else "port"
        cpu_scene = po.RefScene(meshes, env) if kind == "reference" else po.OracleScene(meshes, env)
        r0 = rd.height // 2 - cpu_rows // 2
        desc = dict(d, flags=pb.RENDER_NEE)
        t0 = time.perf_counter()
        ref_rgb, ref_prim = cpu_scene.render(desc, rows=(r0, r0 + cpu_rows), threads=threads)
        dt = time.perf_counter() - t0
        a = film[r0:r0 + cpu_rows].astype(np.float64)
        r = ref_rgb[r0:r0 + cpu_rows].astype(np.float64)
        rmse = float(np.sqrt(np.mean((a - r) ** 2)) / max(np.sqrt(np.mean(r ** 2)), 1e-30))
        res["vs_cpu"] = {"kind": kind, "rows": [int(r0), int(r0 + cpu_rows)], "rel_rmse": rmse,
                         "mean_abs_pixel_error": float(np.mean(np.abs(a - r))),
                         "bit_exact": bool(np.array_equal(film[r0:r0 + cpu_rows].view(np.uint32), ref_rgb[r0:r0 + cpu_rows].view(np.uint32))),
                         "primary_ids_equal": bool(np.array_equal(prim_ids[r0:r0 + cpu_rows], ref_prim[r0:r0 + cpu_rows])),
                         "cpu_msamples_s": round(rd.width * cpu_rows * rd.spp / dt / 1e6, 4), "cores": threads}
        cpu_scene.close()
    scene.close()
    return res


def serve_requests(pb, n_scenes, n_requests, seed):
    """The request mix of the serving workload: scene uniform, resolution in {128..1024}^2, spp in
    {1, 4, 16}, depth 5, next-event estimation on."""
    from polytope_b200 import workloads as W
    rng = np.random.default_rng(seed)
    unit_arrivals = np.cumsum(rng.exponential(1.0, n_requests))  # divided by the rate
    reqs = []
    for k in range(n_requests):
        res = int(rng.choice([128, 256, 512, 1024]))
        spp = int(rng.choice([1, 4, 16]))
        reqs.append((int(rng.integers(n_scenes)), pb.render_desc(res, res, spp, 5, W.SERVE_CAMERA, k + 1, pb.RENDER_NEE)))
    return reqs, unit_arrivals


def serve_tuning(pb):
    t = pb.default_tuning()
    t.pipeline = pb.PIPELINE_PATHS
    t.queue_chunk = 128  # the persistent path kernel's best chunk with 32 M-path waves (as pt_render's default)
    return t


def make_server(pb, wave=1 << 25, policy=0, tuning=None):
    return pb.Server(max_inflight=64, wave_pixels=wave, tuning=tuning or serve_tuning(pb), policy=policy,
                     host_budget=2 << 30)


def film_buffers(reqs):
    """One reusable host film buffer per resolution (a serving client keeps its buffers), for both
    arms, so neither pays for page-faulting fresh memory per request."""
    return {rd.width * rd.height: np.zeros((rd.height, rd.width, 3), np.float32) for _, rd in reqs}


def run_served(pb, srv, scenes, reqs, arrivals, films=None):
    """Submits each request at its arrival time while a client thread waits for the results in
    submission order and copies each film out.  Returns (latencies ms, makespan s, rays): latency
    is the server's completion (film in host memory) minus submission, and the makespan runs from
    the first arrival to the last completion."""
    import queue
    import threading
    films = films or film_buffers(reqs)
    rays0 = srv.stats()["rays_traced"]
    lats = np.zeros(len(reqs))
    run_served.admission_ms = adm = np.zeros(len(reqs))  # submission -> admission, per request
    q = queue.Queue()

    def client():
        for k in range(len(reqs)):
            t = q.get()
            srv.wait(t, 600000)
            lats[k] = srv.poll(t)[1]
            adm[k] = srv.timing(t)["admitted_ms"]
            rd = reqs[k][1]
            pb.check(pb.lib.pt_server_fetch(srv.handle, t, films[rd.width * rd.height].ctypes.data, None))

    th = threading.Thread(target=client)
    th.start()
    t0 = time.perf_counter()
    submit = np.zeros(len(reqs))
    for k, ((si, rd), at) in enumerate(zip(reqs, arrivals)):
        now = time.perf_counter() - t0
        if at > now:
            time.sleep(at - now)
        submit[k] = time.perf_counter() - t0
        q.put(srv.submit(scenes[si], rd))
    th.join()
    span = float(np.max(submit + lats / 1000.0))
    return lats, span, srv.stats()["rays_traced"] - rays0


def with_flags(pb, reqs, extra):
    """The same requests with extra render flags (a pipeline choice for the plain arm)."""
    out = []
    for si, rd in reqs:
        r2 = pb.RenderDesc.from_buffer_copy(rd)
        r2.flags = rd.flags | extra
        out.append((si, r2))
    return out


def run_plain(pb, scenes, reqs, arrivals, films=None):
    """One pt_render per request in arrival order (host film out, pt_render's default pipeline
    unless the requests carry another); returns (latencies ms, makespan s)."""
    films = films or film_buffers(reqs)
    done = np.zeros(len(reqs))
    t0 = time.perf_counter()
    for k, (si, rd) in enumerate(reqs):
        now = time.perf_counter() - t0
        if arrivals[k] > now:
            time.sleep(arrivals[k] - now)
        rgb = films[rd.width * rd.height]
        pb.check(pb.lib.pt_render(scenes[si].handle, ctypes.byref(rd), rgb.ctypes.data, None, 0, None))
        done[k] = time.perf_counter() - t0
    return (done - arrivals) * 1000.0, float(done[-1])


def bench_served(pb, torch, n_scenes=32, n_requests=300, rates=(50.0, 200.0, 2000.0), seed=19, repeats=3):
    """Resident scene pool, Poisson request arrivals at each rate: the serving loop vs one
    pt_render per request in arrival order.  Latency = completion - arrival."""
    from polytope_b200 import workloads as W
    pool = W.serving_pool(n_scenes)
    scenes = build_scenes(pb, pool)
    reqs, unit = serve_requests(pb, n_scenes, n_requests, seed)
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(8) as ex:
        two_bytes = sum(ex.map(lambda sp: pb.two_level_plan(sp[0], sp[1])["device_bytes"], pool))
    # one long-running service for every rate; both arms are warmed on the whole request list
    # (memory pools, host arena, lazily loaded kernels), submitted at once
    srv = make_server(pb)
    films = film_buffers(reqs)
    run_served(pb, srv, scenes, reqs, np.zeros(len(reqs)), films)
    run_plain(pb, scenes, reqs, np.zeros(len(reqs)), films)
    pct = lambda a, q: round(float(np.percentile(a, q)), 2)
    out = {"workload": f"{n_scenes} resident scenes (instanced displaced spheres, 100k-4M tris), {n_requests} Poisson requests per rate, "
                       "128^2-1024^2, 1/4/16 spp, depth 5, NEE",
           "server": "one server for every rate: path-wave pipeline, oldest-first waves of up to 33,554,432 paths, 2 waves queued, "
                     "films by DMA into a 2 GiB pinned arena; a client thread copies results out in submission order "
                     "into reused buffers (the plain arm renders into the same reused buffers)",
           "timing": "host steady clock from the first arrival to the last completion (film in host memory); latency = completion - arrival; "
                     "each arm's run with the median makespan of 3 (runs: [Mrays/s, p99 ms(, GPU busy ms of the waves, scheduler planning ms)] of each)",
           "rates": [],
           "pool": {"faces": int(sum(sum(len(m.faces) for m in sp[0]) for sp in pool)),
                    "device_bytes": int(sum(sc.info().device_bytes for sc in scenes)),
                    "two_level_device_bytes": int(two_bytes)}}
    def summary(lat, span, rays):
        return {"mrays_s": round(rays / span / 1e6, 1), "p50_ms": pct(lat, 50), "p95_ms": pct(lat, 95),
                "p99_ms": pct(lat, 99), "makespan_s": round(span, 3)}

    fused_reqs = with_flags(pb, reqs, pb.RENDER_FUSED)
    run_plain(pb, scenes, fused_reqs, np.zeros(len(reqs)), films)
    for rate in rates:
        # both arms are host-clocked, so each rate runs `repeats` times, arms alternating, and the
        # run with the median makespan of each arm is reported (all runs listed beside it); at the
        # highest rate the plain arm also runs with the one-thread-per-path fused kernel
        arrivals = unit / rate
        top = rate == max(rates)
        served, plain, plain_fused = [], [], []
        for _ in range(repeats):
            s0 = srv.stats()
            lat_s, span_s, rays = run_served(pb, srv, scenes, reqs, arrivals, films)
            s1 = srv.stats()
            served.append(summary(lat_s, span_s, rays))
            served[-1]["gpu_busy_ms"] = round(s1["busy_ms"] - s0["busy_ms"], 1)
            served[-1]["waves"] = int(s1["waves"] - s0["waves"])
            served[-1]["blocked_admission_ms"] = round(s1["blocked_ms"] - s0["blocked_ms"], 1)
            served[-1]["scheduler_plan_ms"] = round(s1["plan_ms"] - s0["plan_ms"], 1)
            served[-1]["scheduler_retire_wait_ms"] = round(s1["retire_wait_ms"] - s0["retire_wait_ms"], 1)
            served[-1]["admission_wait_ms"] = {"p50": pct(run_served.admission_ms, 50), "p99": pct(run_served.admission_ms, 99)}
            lat_p, span_p = run_plain(pb, scenes, reqs, arrivals, films)
            plain.append(summary(lat_p, span_p, rays))
            if top:
                lat_f, span_f = run_plain(pb, scenes, fused_reqs, arrivals, films)
                plain_fused.append(summary(lat_f, span_f, rays))
        med = lambda runs: sorted(runs, key=lambda r: r["makespan_s"])[len(runs) // 2]
        out["rays"] = int(rays)
        entry = {"rate_per_s": rate, "served": med(served), "plain_per_request": med(plain),
                 "runs": {"served": [(r["mrays_s"], r["p99_ms"], r["gpu_busy_ms"], r["scheduler_plan_ms"]) for r in served],
                          "plain_per_request": [(r["mrays_s"], r["p99_ms"]) for r in plain]}}
        entry["served_over_plain"] = round(entry["served"]["mrays_s"] / entry["plain_per_request"]["mrays_s"], 3)
        if top:
            entry["plain_per_request_fused"] = med(plain_fused)
            entry["runs"]["plain_per_request_fused"] = [(r["mrays_s"], r["p99_ms"]) for r in plain_fused]
            entry["served_over_plain_fused"] = round(entry["served"]["mrays_s"] / entry["plain_per_request_fused"]["mrays_s"], 3)
        out["rates"].append(entry)
    srv.close()
    # admission by device memory: the same requests at the highest rate under a request-memory
    # budget of 256 MiB (about nine 1024x1024 requests), so admissions wait for memory to free up
    budget = 256 << 20
    bsrv = pb.Server(max_inflight=64, memory_budget=budget, wave_pixels=1 << 25, tuning=serve_tuning(pb),
                     host_budget=2 << 30)
    run_served(pb, bsrv, scenes, reqs, np.zeros(len(reqs)), films)
    s0 = bsrv.stats()
    lat_b, span_b, rays_b = run_served(pb, bsrv, scenes, reqs, unit / max(rates), films)
    s1 = bsrv.stats()
    out["memory_budgeted"] = dict(summary(lat_b, span_b, rays_b), rate_per_s=max(rates), memory_budget_bytes=budget,
                                  blocked_admission_ms=round(s1["blocked_ms"] - s0["blocked_ms"], 1),
                                  admission_wait_ms={"p50": pct(run_served.admission_ms, 50),
                                                     "p99": pct(run_served.admission_ms, 99)},
                                  gpu_busy_ms=round(s1["busy_ms"] - s0["busy_ms"], 1),
                                  note="blocked_admission_ms counts scheduler time idle with requests queued and no room; "
                                       "admission_wait_ms is each request's submission-to-admission time")
    bsrv.close()
    return out


def l2_roofline(torch, dev, achieved_gbs):
    """The same algorithmic bytes against an L2 bandwidth measured here: a device-to-device copy of
    24 MiB into 24 MiB (both resident in the 126 MB L2), read + write bytes, best of 5 x 50 copies."""
    src = torch.empty(24 << 20, dtype=torch.uint8, device=dev)
    dst = torch.empty_like(src)
    src.fill_(1)
    for _ in range(10):
        dst.copy_(src)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    best = 0.0
    for _ in range(5):
        e0.record()
        for _ in range(50):
            dst.copy_(src)
        e1.record()
        e1.synchronize()
        best = max(best, 2 * src.numel() * 50 / (e0.elapsed_time(e1) * 1e-3) / 1e9)
    return {"achieved": round(achieved_gbs, 1), "peak": round(best, 1), "unit": "GB/s",
            "frac": round(achieved_gbs / best, 4),
            "note": "algorithmic bytes per second against an L2-resident copy (24 MiB -> 24 MiB) measured in this run; "
                    "the tree and faces (113 MB) are L2-resident, so most node and face reads are L2 traffic"}


def max_over_ranks(values, dist, device):
    """Each value's maximum over all ranks (the slowest rank's time); unchanged on one rank."""
    if dist is None:
        return [float(v) for v in values]
    import torch
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t]


def t_error_vs_f64(mesh, rays, hits, limit=1_000_000):
    """Relative error of the FP32 t of closest hits against the FP64 ray-plane distance of the
    same triangle (the microbench mesh has an identity transform, so its vertices are world space)."""
    import polytope_b200 as pb
    sel = np.nonzero((hits["prim"] != pb.PRIM_NONE) & (rays["flags"] == 0))[0][:limit]
    vx = np.stack([mesh.x, mesh.y, mesh.z], 1).astype(np.float64)
    f = np.asarray(mesh.faces)[hits["prim"][sel]]
    v0, v1, v2 = vx[f[:, 0]], vx[f[:, 1]], vx[f[:, 2]]
    org, d = rays["org"][sel].astype(np.float64), rays["dir"][sel].astype(np.float64)
    nrm = np.cross(v1 - v0, v2 - v0)
    t64 = ((v0 - org) * nrm).sum(1) / (d * nrm).sum(1)
    rel = np.abs(hits["t"][sel] - t64) / np.abs(t64)
    return {"closest_hits_checked": int(len(sel)), "max_rel": float(rel.max()), "mean_rel": float(rel.mean())}


def make_workload(n_rays):
    from polytope_b200 import workloads as W
    return W.microbench(n_rays=n_rays)


def cpu_reference(meshes, rays, sample, threads):
    """Time the reference's own closest/any-hit queries (oracle/_ref, else the restatement)."""
    from oracle import pyoracle as po
    if po.ref_available():
        scene, kind = po.RefScene(meshes), "reference"
    else:
        scene, kind = po.OracleScene(meshes), "port"
    sub = rays[:sample]
    t0 = time.perf_counter()
    scene.trace(sub, threads=threads)
    dt = time.perf_counter() - t0
    return sample / dt / 1e6, kind, dt


def run_reference(args, rank, world):
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    meshes, rays = make_workload(N_RAYS)
    sample = args.ref_sample
    for _ in range(max(0, args.warmup)):
        cpu_reference(meshes, rays, min(sample, 65536), threads)
    vals = []
    for _ in range(args.steps):
        v, kind, dt = cpu_reference(meshes, rays, sample, threads)
        vals.append(v)
    value = statistics.median(vals)
    line = {
        "impl": "reference", "metric": "Mrays/s", "value": round(value, 4), "unit": "Mrays/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "rays_per_gpu": N_RAYS, "faces": int(sum(len(m.faces) for m in meshes)),
                   "launch": f"the reference's own bvh::intersect_compact + Mesh::intersect ({kind}), host threads",
                   "parallelism": f"host threads x{threads}", "sample_rays_per_step": sample},
        "cpu_baseline": {"value": round(value, 4), "unit": "Mrays/s", "cores": threads, "kind": kind,
                         "sample": f"first {sample} rays of the {N_RAYS}-ray set per step, all host threads"},
        "e2e": {"value": round(value, 4), "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--rays", type=int, default=N_RAYS)
    ap.add_argument("--ref-sample", type=int, default=N_RAYS)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--no-served", action="store_true")
    ap.add_argument("--no-render", action="store_true")
    ap.add_argument("--render-probe", action="store_true",
                    help="render the instanced scene at 480x270, 16 spp once with the fused kernel (PT_RENDER_FUSED) "
                         "and once with pt_render's default persistent path kernel, then exit (a small case for profilers)")
    ap.add_argument("--batch-probe", action="store_true",
                    help="run the first 32 scenes of the 256-scene batch once through the wavefront pipeline with "
                         "the tuning the autotuner picks for the full batch, then exit (a small case for profilers)")
    ap.add_argument("--no-autotune", action="store_true")
    args = ap.parse_args()

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if args.render_probe:
        import polytope_b200 as pb
        from polytope_b200 import workloads as W
        meshes, env = W.instanced_scene()
        scene = pb.Scene(meshes, env)
        d = W.INSTANCED_RENDER
        for fl in (pb.RENDER_FUSED, 0):
            rgb, _ = pb.render(scene, 480, 270, 16, d["max_depth"], d["camera"], d["seed"], pb.RENDER_NEE | fl)
            print(json.dumps({"render_probe": "480x270x16", "flags": pb.RENDER_NEE | fl, "mean": float(rgb.mean())}))
        return

    if args.batch_probe:
        import polytope_b200 as pb
        from polytope_b200 import workloads as W
        work = W.batched_workload(256)[:32]
        scenes = build_scenes(pb, [(w[0], w[1]) for w in work])
        jobs = [(sc, pb.render_desc(d["width"], d["height"], d["spp"], d["max_depth"], d["camera"], d["seed"], pb.RENDER_NEE))
                for sc, (_, _, d) in zip(scenes, work)]
        t = pb.default_tuning()
        t.pipeline, t.wave_pixels, t.threads_per_block, t.stack_depth, t.queue_chunk = pb.PIPELINE_WAVEFRONT, 1 << 25, 256, 32, 32
        b = pb.Batch(jobs, t)
        b.run()
        print(json.dumps({"batch_probe": "32 scenes, wavefront pipeline", "rays": int(b.rays_traced())}))
        b.close()
        return

    import torch
    import polytope_b200 as pb

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)

    meshes, rays = make_workload(args.rays)
    n = len(rays)
    scene = pb.Scene(meshes)
    stream = torch.cuda.Stream(device=dev)

    # counted pass (untimed): per-ray node / face tests for the algorithmic-bytes numerator
    hits_np, nt, tt = scene.intersect(rays, counts=True)
    alg_bytes = float(32 * nt.sum(dtype=np.uint64) + 44 * tt.sum(dtype=np.uint64) + (28 + 16) * n)
    t_err = t_error_vs_f64(meshes[0], rays, hits_np)

    d_rays = torch.from_numpy(rays.view(np.uint8)).to(dev)
    d_hits = torch.zeros(n * 16, dtype=torch.uint8, device=dev)

    def step():
        pb.check(pb.lib.pt_trace(scene.handle, d_rays.data_ptr(), n, d_hits.data_ptr(), pb.MEM_DEVICE, stream.cuda_stream))

    if not args.no_autotune:  # launch shape of the ray-query kernel, picked before the timed region
        scene.autotune_trace(d_rays, d_hits, n)
    trace_tuning = scene.trace_tuning()

    with torch.cuda.stream(stream):
        for _ in range(max(3, args.warmup)):
            step()
    stream.synchronize()
    assert d_hits.cpu().numpy().tobytes() == hits_np.tobytes(), "device-resident hits differ from the counted pass"

    sampler = clocks_sampler()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    with torch.cuda.stream(stream):
        ev[0].record(stream)
        for k in range(args.steps):
            step()
            ev[k + 1].record(stream)
    stream.synchronize()
    torch.cuda.synchronize()
    per = [ev[k].elapsed_time(ev[k + 1]) for k in range(args.steps)]
    total_ms = ev[0].elapsed_time(ev[-1])

    # end to end through the C ABI with pinned host buffers (H2D + kernel + D2H per step)
    h_rays = torch.from_numpy(rays.view(np.uint8)).pin_memory()
    h_hits = torch.zeros(n * 16, dtype=torch.uint8).pin_memory()
    for _ in range(2):
        pb.check(pb.lib.pt_trace(scene.handle, h_rays.data_ptr(), n, h_hits.data_ptr(), 0, None))
    if dist:
        dist.barrier()
    e2e_steps = max(3, min(args.steps, 10))
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(e2e_steps):
        pb.check(pb.lib.pt_trace(scene.handle, h_rays.data_ptr(), n, h_hits.data_ptr(), 0, None))
    e1.record()
    e1.synchronize()
    e2e_ms = e0.elapsed_time(e1) / e2e_steps
    assert h_hits.numpy().tobytes() == hits_np.tobytes(), "e2e hits differ"
    # the link bound of the end-to-end number: the same rays copied host -> device alone
    h2d_ms = 1e30
    for _ in range(3):
        e0.record()
        d_rays.copy_(h_rays, non_blocking=True)
        e1.record()
        e1.synchronize()
        h2d_ms = min(h2d_ms, e0.elapsed_time(e1))
    # and both directions at once, as a step moves them: the rays in and the hits out on two streams
    d_out = torch.empty(n * 16, dtype=torch.uint8, device=dev)
    h_out = torch.empty(n * 16, dtype=torch.uint8).pin_memory()
    cur, s_in, s_out = torch.cuda.current_stream(), torch.cuda.Stream(), torch.cuda.Stream()
    both_ms = 1e30
    for _ in range(3):
        e0.record()
        s_in.wait_stream(cur)
        s_out.wait_stream(cur)
        with torch.cuda.stream(s_in):
            d_rays.copy_(h_rays, non_blocking=True)
        with torch.cuda.stream(s_out):
            h_out.copy_(d_out, non_blocking=True)
        cur.wait_stream(s_in)
        cur.wait_stream(s_out)
        e1.record()
        e1.synchronize()
        both_ms = min(both_ms, e0.elapsed_time(e1))
    clk = clocks_summary(sampler)

    ms, e2e_ms = max_over_ranks([total_ms / args.steps, e2e_ms], dist, dev)
    if rank == 0:
        value = n * world / (ms * 1e-3) / 1e6
        e2e = n * world / (e2e_ms * 1e-3) / 1e6
        peak, peak_kind = peaks()
        achieved = alg_bytes / (ms * 1e-3) / 1e9
        traffic = profiled_traffic()
        line = {
            "metric": "Mrays/s", "value": round(value, 3), "unit": "Mrays/s", "n_gpus": world,
            "steps": args.steps, "warmup": max(3, args.warmup), "ms_per_step": round(ms, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded generators)",
            "config": {"workload": WORKLOAD, "rays_per_gpu": n, "faces": int(sum(len(m.faces) for m in meshes)),
                       "launch": "plain per-frame launch (one trace kernel over all rays)",
                       "l2": "inputs larger than L2 (rays 512 MiB + hits 256 MiB per step); BVH + faces (113 MB) stay L2-resident",
                       "parallelism": f"replicas x{world}", "trace_tuning": trace_tuning},
            "gpu_launches": args.steps,
            "e2e": {"value": round(e2e, 3), "unit": "Mrays/s", "h2d_bytes_per_step": 32 * n, "d2h_bytes_per_step": 16 * n,
                    "ms_per_step": round(e2e_ms, 4),
                    "h2d_copy_alone_ms": round(h2d_ms, 4), "h2d_gbs": round(32 * n / (h2d_ms * 1e-3) / 1e9, 1),
                    "h2d_and_d2h_concurrent_ms": round(both_ms, 4),
                    "note": "the step's copies alone (rays in and hits out at once, no kernel) bound the end-to-end "
                            "step from below"},
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "traffic": traffic,
                         "note": f"algorithmic bytes {alg_bytes / 1e9:.2f} GB per launch (reference node/face test counts); peak {peak_kind}"},
            "roofline_l2": l2_roofline(torch, dev, achieved),
            "clocks": clk,
            "t_error_vs_fp64": t_err,
            "step_ms": {"min": round(min(per), 4), "median": round(statistics.median(per), 4), "max": round(max(per), 4)},
        }
        # the serving measurement is host-clocked (arrivals, latencies), so it runs first, before
        # the batched and full-frame sections have churned the device and host memory
        if not args.no_served and world == 1:
            line["served"] = bench_served(pb, torch)
        if not args.no_batched and world == 1:
            line["batched"] = bench_batched(pb, torch)
        if not args.no_render and world == 1:
            line["render"] = bench_render(pb, torch, cpu=not args.no_cpu_baseline)
        if not args.no_cpu_baseline and world == 1:  # the host baseline is an N=1 figure
            threads = os.cpu_count() or 1
            v, kind, dt = cpu_reference(meshes, rays, args.ref_sample, threads)
            line["cpu_baseline"] = {"value": round(v, 4), "unit": "Mrays/s", "cores": threads, "kind": kind,
                                    "sample": f"first {args.ref_sample} rays of the ray set ({dt:.1f} s)"}
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
