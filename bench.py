#!/usr/bin/env python
"""Benchmark of the B200 wavefront path tracer on the 1M-triangle sphere-field workload.

Workload (one step = one full frame): 64 displaced icospheres (20,480 triangles each)
over a 2-triangle ground plane plus 256 emissive triangles (1,310,978 triangles),
40/40/20 % Lambert/GGX/mirror, rendered at 1920x1080, 64 spp, path depth 12, NEE.
Synthetic, seeded (scene seed 2, Philox seed 1234).

Arms:
  default           the sm_100a path through the C ABI (libgpt_b200.so)
  --impl reference  the reference's renderer restated on the CPU (oracle/), all host threads,
                    on a bounded sample of the same workload per step
Multi-GPU (torchrun, one process per GPU): every rank renders its own frame of the same
workload on distinct Philox subsequences (weak scaling); the per-pixel accumulation buffers
are summed across ranks with an NCCL all-reduce after each frame (the combined image).

On one GPU the line also carries (--sections, default all):
  plain      the plain single-job FP32 form on the same frame: binary FP32 BVH, warps refilled only
             when all lanes are idle, host-driven iteration loop, 1,048,576 path slots, no autotuning
  cornell    the Cornell box at 512x512, 16 spp, depth 8, NEE
  batched    64 uneven jobs over 4 resident scenes (10k-2M triangles) through the job server in one
             device loop, against the same jobs one at a time (server, frame renderer, plain form)
  serving    open-loop Poisson arrivals (20, 50, 100 jobs/s; 200 per rate) over 8 resident scenes
             (50k-4M triangles): p50/p99 latency, per-job slowdown, paths/s and admitted-bytes
             high-water mark, served (continuous batching: short jobs first, then the others in
             submission order; with --serve-shortest-first also shortest remaining work first) against
             one job at a time in submission order
  precision  8M-triangle scene at 3840x2160, 16 spp, depth 10: BVH8 with 8-bit quantised boxes
             against the binary FP32 BVH (node bytes per ray, traversal Mrays/s), and the FP32 Kahan
             accumulation against FP64 accumulation of the same per-sample radiance (RMSE)
  lights     power-weighted against area-weighted light selection at equal paths (RMSE)
  bvh        the BVH8 built on the host against the same format built on the device: build seconds,
             traversal work and frame time on the C2 and C4 frames, identical images
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
for sub in ("gpu-path-tracer_b200", "oracle"):
    p = os.path.join(ROOT, sub)
    if p not in sys.path:
        sys.path.insert(0, p)

import numpy as np  # noqa: E402

WORKLOAD = dict(workload="spheres-1m", scene="spheres-1m", triangles=1310978, width=1920, height=1080, spp=64,
                depth=12, nee=True, lights=256, pool=1 << 20)
TRACE_ALGO_BYTES_PER_RAY = 32 + 48   # ray record read, material-queue entry (ray and hit) written; a miss writes none
NODE_BYTES = 64 + 4   # a BVH8 node visit reads the 64-byte header (boxes, origin, scales, masks) and its 4-byte reference
TRIANGLE_BYTES = 48


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--pool", type=int, default=0, help="path slots; 0 = autotuned")
    ap.add_argument("--no-autotune", action="store_true", help="use the library defaults instead of gpt_autotune")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="target CPU time of the bounded CPU sample")
    ap.add_argument("--loop", default="graph", choices=["graph", "host"],
                    help="frame loop: one CUDA graph per frame (default) or host-launched iterations (for ncu)")
    ap.add_argument("--profile-case", action="store_true",
                    help="small frame (640x360, 16 spp) of the same scene for ncu captures; not a bench line")
    ap.add_argument("--trace-occupancy", type=int, default=0, help="with --no-autotune: traversal variant (1, 10, 12)")
    ap.add_argument("--trace-refill", type=int, default=0, help="with --no-autotune: idle lanes before a warp refills")
    ap.add_argument("--trace-block", type=int, default=0, help="with --no-autotune: traversal threads per block")
    ap.add_argument("--sections", default="all",
                    help="comma list of extra one-GPU sections: plain,cornell,batched,serving,precision,lights (all/none)")
    ap.add_argument("--serve-jobs", type=int, default=200,
                    help="jobs per arrival rate in the serving section (p99 of fewer than 100 jobs is their maximum)")
    ap.add_argument("--serve-shortest-first", action="store_true",
                    help="serving section: also run the server ordering every job by samples left")
    ap.add_argument("--no-reference-build", action="store_true",
                    help="skip timing the reference's own kernels (oracle/_ref) on the same frame")
    ap.add_argument("--serve-rates", default="20,50,100", help="Poisson arrival rates (jobs/s) of the serving section")
    ap.add_argument("--serve-short-seconds", type=float, default=0.0,
                    help="render time alone below which the served server treats a job as short (0 = the server's default)")
    ap.add_argument("--serve-pool", type=int, default=1 << 23,
                    help="most path slots of the serving section's servers (latency of small jobs grows with the pool)")
    return ap.parse_args()


SECTIONS = ("plain", "cornell", "batched", "serving", "precision", "lights", "bvh")


def wanted_sections(args):
    if args.sections == "all":
        return set(SECTIONS)
    if args.sections in ("", "none"):
        return set()
    out = {x.strip() for x in args.sections.split(",") if x.strip()}
    unknown = out - set(SECTIONS)
    if unknown:
        raise SystemExit(f"unknown sections: {sorted(unknown)}")
    return out


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        d = json.load(open(path))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profile_dram_bytes_per_ray():
    """DRAM bytes per ray of the closest-hit traversal kernel, from the committed ncu capture of one
    full-pool launch of this workload (dram__bytes_read.sum + dram__bytes_write.sum over its rays)."""
    path = os.path.join(ROOT, "profiles", "trace_closest_spheres1m.json")
    if os.path.exists(path):
        return json.load(open(path)).get("dram_bytes_per_ray")
    return None


class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""

    FIELDS = "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown," \
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"

    def __init__(self, device):
        self.device = device
        self.lines = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.device)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        time.sleep(0.05)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "reasons": sorted(reasons), "samples": len(sm)}


def cpu_sample_config(scene_name, seconds, threads):
    """Bounded CPU sample of the workload: the whole image at a reduced resolution (so every part
    of the scene is represented), 4 spp, sized to about `seconds` of CPU time."""
    import oracle
    import scenes
    s = scenes.config_scene(scene_name)
    o = oracle.OracleScene(s)
    w, h = 192, 108
    cam = scenes.scene_camera(s, w, h)
    t0 = time.perf_counter()
    trial = o.render(cam, w, h, 4, WORKLOAD["depth"], True, threads=threads)
    dt = time.perf_counter() - t0
    rate = trial["total_samples"] / dt
    target = max(1, int(rate * seconds))
    scale = max(1.0, np.sqrt(target / (w * h * 4)))
    w2, h2 = int(w * scale) // 2 * 2, int(h * scale) // 2 * 2
    return s, o, (w2, h2, 4)


def run_cpu(scene_name, seconds, threads, steps=1):
    import scenes
    s, o, (w, h, spp) = cpu_sample_config(scene_name, seconds, threads)
    cam = scenes.scene_camera(s, w, h)
    times = []
    total = 0
    for _ in range(steps):
        t0 = time.perf_counter()
        res = o.render(cam, w, h, spp, WORKLOAD["depth"], True, threads=threads)
        times.append(time.perf_counter() - t0)
        total = res["total_samples"]
    return total, times, f"{w}x{h} at {spp} spp of the same scene, camera and depth ({total} paths, whole image)"


def reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    import oracle
    threads = oracle.default_threads()
    steps = args.warmup + args.steps
    per_step = max(3.0, min(15.0, 150.0 / steps))
    total, times, sample = run_cpu(WORKLOAD["scene"], per_step, threads, steps=steps)
    timed = times[args.warmup:] if len(times) > args.warmup else times
    value = total * len(timed) / sum(timed)
    line = {
        "impl": "reference", "metric": "paths_per_second", "value": value, "unit": "paths/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * sum(timed) / len(timed),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD["workload"], "triangles": WORKLOAD["triangles"], "resolution": "1920x1080",
                   "spp": WORKLOAD["spp"], "depth": WORKLOAD["depth"], "nee": True, "l2": "inputs larger than L2 (CPU)"},
        "cpu_baseline": {"value": value, "unit": "paths/s", "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": "paths/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def traversal_summary(st, node_bytes):
    """Per-ray traversal work and rates of one frame's statistics."""
    rays, shadow = st["rays"], st["shadow_rays"]
    out = {"rays": rays, "shadow_rays": shadow, "node_bytes": node_bytes}
    for k, name, n, phase in ((0, "closest", rays, "trace"), (1, "shadow", shadow, "shadow")):
        if n == 0:
            continue
        visits, tests = st["node_visits"][k] / n, st["triangle_tests"][k] / n
        out[name] = {"node_visits_per_ray": visits, "triangle_tests_per_ray": tests,
                     "node_bytes_per_ray": visits * node_bytes, "bvh_bytes_per_ray": visits * node_bytes + tests * TRIANGLE_BYTES,
                     "traversal_mrays_per_second": n / (st["phase_ms"][phase] / 1000.0) / 1e6 if st["phase_ms"][phase] > 0 else None}
    return out


def plain_form(renderer, cam, W, H, spp, depth, frames=2):
    """The plain single-job FP32 wavefront form of a frame: the reference's wavefront structure on this
    project's kernels. Binary FP32 BVH (64-B nodes, local-memory stack), warps refilled only when all
    32 lanes are idle, finished paths regenerated from a queue in finishing order, shading kernels one
    after another, host-driven iteration loop with a flag read per iteration, 1,048,576 path slots (the
    reference's pool), no autotuning. Same images bit for bit as the optimised form."""
    import pathtracer
    settings = dict(pool_size=1 << 20, trace_occupancy=1, trace_refill=32 | (32 << 8), trace_block=128,
                    loop_mode=pathtracer.LOOP_HOST, bvh_format=pathtracer.BVH2_FP32,
                    wavefront_layout=pathtracer.WAVEFRONT_QUEUES)
    renderer.render_frame(cam, W, H, spp, depth, True, **settings)
    stats = [renderer.render_frame(cam, W, H, spp, depth, True, **settings) for _ in range(frames)]
    ms = sum(s["device_ms"] for s in stats) / frames
    return {"value": stats[0]["samples"] / (ms / 1000.0), "unit": "paths/s", "ms_per_frame": ms,
            "iterations": stats[0]["iterations"], "settings": {k: v for k, v in settings.items()},
            "traversal": traversal_summary(stats[-1], pathtracer.NODE_BYTES[pathtracer.BVH2_FP32]),
            "what": "binary FP32 BVH, warps refilled only when all lanes are idle, regeneration queue, shading in sequence, "
                    "host-driven loop, 1,048,576 slots, no autotune"}


def cornell_section(knobs):
    """Cornell box, 512x512, 16 spp, depth 8, NEE (36 triangles, 2-entry alias table)."""
    import pathtracer
    import scenes
    s = scenes.config_scene("cornell")
    r = pathtracer.Renderer(0)
    try:
        r.upload_scene(s)
        W, H, spp, depth = 512, 512, 16, 8
        cam = scenes.scene_camera(s, W, H)
        tuned = r.autotune(cam, W, H, spp, depth, True)
        kn = {k: tuned[k] for k in ("pool_size", "trace_occupancy", "trace_refill", "trace_block")}
        for _ in range(3):
            r.render_frame(cam, W, H, spp, depth, True, **kn)
        stats = [r.render_frame(cam, W, H, spp, depth, True, **kn) for _ in range(10)]
        ms = sum(x["device_ms"] for x in stats) / len(stats)
        rays = sum(x["rays"] + x["shadow_rays"] for x in stats) / len(stats)
        plain = plain_form(r, cam, W, H, spp, depth)
    finally:
        r.close()
    return {"value": W * H * spp / (ms / 1000.0), "unit": "paths/s", "ms_per_frame": ms,
            "mrays_per_second": rays / (ms / 1000.0) / 1e6, "knobs": kn, "plain_form_paths_per_second": plain["value"],
            "config": "cornell box (36 triangles), 512x512, 16 spp, depth 8, NEE"}


def _server_knobs(knobs):
    return dict(trace_block=knobs["trace_block"], trace_refill=knobs["trace_refill"],
                trace_occupancy=knobs["trace_occupancy"])


def _run_jobs_on_server(srv, ids, jobs, open_loop):
    """Submits the jobs (at their arrival times when open_loop, else all at once), waits for all and
    reads every image back. Returns (wall seconds, per-job latency seconds)."""
    t0 = time.perf_counter()
    jids = []
    for j in jobs:
        if open_loop:
            delay = j.arrival_s - (time.perf_counter() - t0)
            if delay > 0:
                time.sleep(delay)
        jids.append(srv.submit(ids[j.scene], j.camera, j.width, j.height, j.spp, j.depth, True))
    lat = []
    service = []
    for jid in jids:
        st = srv.wait(jid, 3600.0)
        if st["state"] != "done":
            raise RuntimeError(f"job {jid} ended as {st['state']}: {srv.last_error()}")
        srv.result(jid)
        lat.append(st["done_s"] - st["submit_s"])
        service.append(st["done_s"] - st["admit_s"])
        srv.release(jid)
    _run_jobs_on_server.service = service
    return time.perf_counter() - t0, lat


def batched_section(knobs):
    """64 uneven jobs over 4 resident scenes: one device loop for all (job server) against one job at
    a time (server with max_active_jobs=1, the optimised frame renderer, and the plain form). Every
    mode renders the job list once untimed, then once timed (steady state: buffers and host image
    memory in place)."""
    import pathtracer
    import scenes
    import workloads
    jobs = workloads.batched_jobs()
    resident = {n: scenes.config_scene(n) for n in workloads.BATCH_SCENES}
    total = sum(j.paths for j in jobs)
    out = {"jobs": len(jobs), "paths": total, "scenes": {n: s.triangle_count for n, s in resident.items()},
           "config": "64 jobs, resolution log-uniform 256x256..1920x1080, spp in {1,4,16,64}, depth 8..12, seeded orbit cameras"}
    warm = [workloads.Job(n, 64, 64, 1, 8, scenes.scene_camera(s, 64, 64)) for n, s in resident.items()]
    for mode, active, schedule in (("batched", 0, 0), ("server_one_at_a_time", 1, pathtracer.SCHEDULE_OLDEST_FIRST)):
        srv = pathtracer.Server(0, pool_size=knobs["pool_size"], max_active_jobs=active, hbm_budget_bytes=32 << 30,
                                schedule=schedule, **_server_knobs(knobs))
        try:
            ids = {n: srv.add_scene(s) for n, s in resident.items()}
            _run_jobs_on_server(srv, ids, warm, False)
            _run_jobs_on_server(srv, ids, jobs, False)  # steady state: one untimed pass over the same jobs
            before = srv.stats()
            wall, _ = _run_jobs_on_server(srv, ids, jobs, False)
            st = srv.stats()
        finally:
            srv.close()
        dev_ms = st["device_ms"] - before["device_ms"]
        out[mode] = {"paths_per_second": total / wall, "device_paths_per_second": total / (dev_ms / 1000.0),
                     "wall_s": wall, "device_s": dev_ms / 1000.0, "slices": st["slices"] - before["slices"],
                     "iterations": st["iterations"] - before["iterations"],
                     "phase_ms": {k: st["phase_ms"][k] - before["phase_ms"][k] for k in st["phase_ms"]},
                     "admitted_high_water_bytes": st["admitted_high_water"]}
    # one frame at a time through gpt_render_frame: optimised (BVH8, graph loop) and plain form
    renderers = {}
    try:
        for n, s in resident.items():
            renderers[n] = pathtracer.Renderer(0)
            renderers[n].upload_scene(s)
        plain_settings = dict(pool_size=1 << 20, trace_occupancy=1, trace_refill=32 | (32 << 8), trace_block=128,
                              loop_mode=pathtracer.LOOP_HOST, bvh_format=pathtracer.BVH2_FP32,
                              wavefront_layout=pathtracer.WAVEFRONT_QUEUES)
        for mode, settings in (("frames_one_at_a_time", dict(knobs)), ("plain_form_one_at_a_time", plain_settings)):
            for j in warm + jobs:  # steady state: one untimed pass over the same jobs
                renderers[j.scene].render_frame(j.camera, j.width, j.height, j.spp, j.depth, True, **settings)
            t0 = time.perf_counter()
            dev = 0.0
            for j in jobs:
                st = renderers[j.scene].render_frame(j.camera, j.width, j.height, j.spp, j.depth, True, **settings)
                dev += st["device_ms"]
            wall = time.perf_counter() - t0
            out[mode] = {"paths_per_second": total / wall, "device_paths_per_second": total / (dev / 1000.0),
                         "wall_s": wall, "device_s": dev / 1000.0}
    finally:
        for r in renderers.values():
            r.close()
    out["speedup_vs_plain_form"] = out["batched"]["paths_per_second"] / out["plain_form_one_at_a_time"]["paths_per_second"]
    out["speedup_vs_frames_one_at_a_time"] = out["batched"]["paths_per_second"] / out["frames_one_at_a_time"]["paths_per_second"]
    out["timing"] = "wall clock from the first submit (or frame) to the last image read back to host memory"
    return out


def serving_section(knobs, rates, n_jobs, max_pool, schedule_served=0, short_seconds=0.0, shortest_first=False):
    """Open-loop Poisson arrivals over 8 resident scenes: continuous batching against one job at a time.
    Both servers hold at most max_pool path slots: an iteration's time grows with the slots in flight,
    and a small job needs a fixed number of iterations, so its latency grows with the pool."""
    import pathtracer
    import scenes
    import workloads
    resident = {n: scenes.config_scene(n) for n in workloads.SERVE_SCENES}
    out = {"scenes": {n: s.triangle_count for n, s in resident.items()}, "jobs_per_rate": n_jobs,
           "budget_bytes": 16 << 30,
           "config": "Poisson arrivals; resolution log-uniform 128x128..2048x2048, spp in {4,16,64,256}, depth 8..12, "
                     "seeded orbit cameras; admission: 64 B per in-flight path + framebuffers within the budget",
           "latency": "server done_s - submit_s per job (submission at the scheduled arrival time)"}
    warm = [workloads.Job(n, 64, 64, 4, 8, scenes.scene_camera(s, 64, 64)) for n, s in resident.items()]
    pool = min(knobs["pool_size"], max_pool)
    out["pool_size"] = pool
    latencies, alone = {}, {}
    # served: continuous batching in the server's default order (short jobs first, shortest remaining
    # work first among them, the other jobs in submission order); shortest_first: the same server
    # ordering every job by samples left; plain: one job at a time in submission order
    modes = (("served", 0, schedule_served),) + (
        (("shortest_first", 0, pathtracer.SCHEDULE_SHORTEST_FIRST),) if shortest_first else ()) + (
        ("plain", 1, pathtracer.SCHEDULE_OLDEST_FIRST),)
    for mode, active, schedule in modes:
        srv = pathtracer.Server(0, pool_size=pool, max_active_jobs=active, hbm_budget_bytes=16 << 30, schedule=schedule,
                                short_job_seconds=short_seconds, **_server_knobs(knobs))
        res = {}
        try:
            ids = {n: srv.add_scene(s) for n, s in resident.items()}
            _run_jobs_on_server(srv, ids, warm, False)
            for rate in rates:
                jobs = workloads.served_jobs(rate, n_jobs)
                before = srv.stats()
                wall, lat = _run_jobs_on_server(srv, ids, jobs, True)
                st = srv.stats()
                paths = sum(j.paths for j in jobs)
                latencies[(mode, rate)] = lat
                if mode == "plain":  # one job at a time: admission to completion is the job's time alone
                    alone[rate] = list(_run_jobs_on_server.service)
                res[f"{rate:g}_jobs_per_s"] = {
                    "p50_latency_s": workloads.percentile(lat, 50), "p99_latency_s": workloads.percentile(lat, 99),
                    "mean_latency_s": sum(lat) / len(lat), "paths_per_second": paths / wall, "wall_s": wall,
                    "device_paths_per_second": paths / ((st["device_ms"] - before["device_ms"]) / 1000.0),
                    "device_busy_fraction": (st["device_ms"] - before["device_ms"]) / 1000.0 / wall,
                    "offered_paths_per_second": paths / jobs[-1].arrival_s,
                    "slices": st["slices"] - before["slices"], "iterations": st["iterations"] - before["iterations"]}
            res["admitted_high_water_bytes"] = srv.stats()["admitted_high_water"]
        finally:
            srv.close()
        out[mode] = res
    # per-job slowdown: latency over the job's own render time alone (one-at-a-time server, admission
    # to completion)
    for rate in rates:
        key = f"{rate:g}_jobs_per_s"
        for mode, _, _ in modes:
            sd = sorted(l / max(a, 1e-6) for l, a in zip(latencies[(mode, rate)], alone[rate]))
            out[mode][key]["p50_slowdown"] = workloads.percentile(sd, 50)
            out[mode][key]["p99_slowdown"] = workloads.percentile(sd, 99)
        for mode in [m for m, _, _ in modes if m != "plain"]:
            out[mode][key]["device_speedup_vs_plain"] = (out[mode][key]["device_paths_per_second"]
                                                         / out["plain"][key]["device_paths_per_second"])
    return out


def bvh_build_section(knobs, cases=(("spheres-1m", 1920, 1080, 64, 12), ("spheres-8m", 3840, 2160, 16, 10)), frames=2):
    """The BVH8 built on the host (binned SAH on all host threads) against the same format built on the
    device (Morton order, clustering, the same 8-wide collapse): build seconds, tree size, traversal
    work and frame time on the headline frame of each scene, and whether the images are identical."""
    import pathtracer
    import scenes
    out = {"what": "host: binned SAH + surface-area-optimal collapse on all host threads; device: Morton order, "
                   "PLOC clustering (radius 16), the same collapse and quantisation on the GPU"}
    for name, W, H, spp, depth in cases:
        s = scenes.config_scene(name)
        cam = scenes.scene_camera(s, W, H)
        res, images = {}, {}
        for label, build in (("host", pathtracer.BVH_BUILD_HOST), ("device", pathtracer.BVH_BUILD_DEVICE)):
            r = pathtracer.Renderer(0)
            try:
                r.set_bvh_build(build)
                r.upload_scene(s)
                times = r.upload_times()
                info = r.scene_info()
                r.render_frame(cam, W, H, spp, depth, True, **knobs)
                stats = [r.render_frame(cam, W, H, spp, depth, True, **knobs) for _ in range(frames)]
                ms = sum(st["device_ms"] for st in stats) / frames
                images[label] = r.framebuffer()
                res[label] = {"bvh_build_s": times["bvh_build_s"], "upload_s": times["upload_s"], "nodes": info["nodes"],
                              "depth": info["depth"], "ms_per_frame": ms, "paths_per_second": stats[-1]["samples"] / (ms / 1000.0),
                              "traversal": traversal_summary(stats[-1], pathtracer.NODE_BYTES[pathtracer.BVH8_Q8])}
            finally:
                r.close()
        res["identical_images"] = bool(np.array_equal(images["host"], images["device"]))
        res["build_speedup"] = res["host"]["bvh_build_s"] / res["device"]["bvh_build_s"]
        res["config"] = f"{s.triangle_count} triangles, {W}x{H}, {spp} spp, depth {depth}, NEE"
        out[name] = res
    return out


def precision_section(knobs):
    """8M-triangle scene, 3840x2160, 16 spp, depth 10: quantised BVH8 against binary FP32 BVH, and
    FP32 Kahan accumulation against FP64 accumulation of the same per-sample radiance."""
    import pathtracer
    import scenes
    s = scenes.config_scene("spheres-8m")
    W, H, spp, depth = 3840, 2160, 16, 10
    r = pathtracer.Renderer(0)
    out = {"config": "spheres-8m (400 displaced icospheres + ground, 4,096 emissive triangles), 3840x2160, 16 spp, depth 10, NEE"}
    try:
        t0 = time.perf_counter()
        r.upload_scene(s)
        out["scene_upload_s"] = time.perf_counter() - t0
        out["scene_upload_breakdown_s"] = r.upload_times()
        info = r.scene_info()
        out["triangles"], out["lights"] = info["triangles"], info["lights"]
        cam = scenes.scene_camera(s, W, H)
        formats = {}
        for name, fmt in (("bvh8_q8", pathtracer.BVH8_Q8), ("bvh2_fp32", pathtracer.BVH2_FP32)):
            r.render_frame(cam, W, H, spp, depth, True, bvh_format=fmt, **knobs)
            st = r.render_frame(cam, W, H, spp, depth, True, bvh_format=fmt, **knobs)
            formats[name] = {"paths_per_second": st["samples"] / (st["device_ms"] / 1000.0), "ms_per_frame": st["device_ms"],
                             "nodes": info["nodes"] if fmt == pathtracer.BVH8_Q8 else info["binary_nodes"],
                             "depth": info["depth"] if fmt == pathtracer.BVH8_Q8 else info["binary_depth"],
                             "traversal": traversal_summary(st, pathtracer.NODE_BYTES[fmt])}
            if fmt == pathtracer.BVH8_Q8:
                fb8 = r.framebuffer()
            else:
                formats["identical_images"] = bool(np.array_equal(fb8, r.framebuffer()))
        out["bvh"] = formats
        # the BVH8 frame again for its buffers: per-pixel Kahan sums and the per-sample radiance
        r.render_frame(cam, W, H, spp, depth, True, **knobs)
        kahan = r.accumulation()[:, :3].astype(np.float64)
        fp64 = r.accumulation_fp64()  # FP64 sums of the same samples, on the device
        rad = r.sample_radiance().reshape(W * H, spp, 3)
        naive = np.zeros((W * H, 3), dtype=np.float32)
        for k in range(spp):  # plain FP32 summation in sample order, for comparison
            naive += rad[:, k, :]
        del rad
        ref = fp64 / spp
        rms_ref = float(np.sqrt(np.mean(ref ** 2)))
        acc = {}
        for name, img in (("fp32_kahan", kahan / spp), ("fp32_naive", naive.astype(np.float64) / spp)):
            err = img - ref
            per_pixel = np.sqrt(np.mean(err ** 2, axis=1))
            acc[name] = {"image_rmse": float(np.sqrt(np.mean(err ** 2))),
                         "image_rmse_relative": float(np.sqrt(np.mean(err ** 2))) / rms_ref if rms_ref > 0 else None,
                         "per_pixel_rmse_max": float(per_pixel.max()),
                         "per_pixel_rmse_p99": float(np.percentile(per_pixel, 99)),
                         "pixels_exact": float(np.mean(np.all(err == 0.0, axis=1)))}
        out["accumulation_vs_fp64"] = acc
        out["fp64_image_rms"] = rms_ref
    finally:
        r.close()
    return out


def summary(line):
    """The line's comparisons in a few numbers: headline, plain form, the reference's own kernels on the
    same GPU, the batched mix, and serving latency per arrival rate."""
    def get(d, *keys):
        for k in keys:
            if not isinstance(d, dict) or k not in d:
                return None
            d = d[k]
        return d
    out = {"value": line["value"], "e2e": line["e2e"]["value"], "roofline_frac": line["roofline"]["frac"],
           "dram_frac": line["roofline"].get("dram_frac"),
           "plain_form_speedup_of_value": get(line, "plain_form", "speedup_of_value"),
           "reference_build_b200_value": get(line, "reference_build_b200", "value"),
           "reference_build_b200_speedup_of_value": get(line, "reference_build_b200", "speedup_of_value"),
           "batched_speedup_vs_plain_form": get(line, "batched", "speedup_vs_plain_form"),
           "power_sampling_samples_for_equal_rmse_c2": get(line, "light_sampling", "spheres-1m", "power", "samples_for_equal_rmse_vs_area"),
           "power_sampling_samples_for_equal_rmse_c4": get(line, "light_sampling", "spheres-8m", "power", "samples_for_equal_rmse_vs_area"),
           "cpu_baseline_value": get(line, "cpu_baseline", "value"),
           "bvh_build_s_host_device": {n: [get(line, "bvh_build", n, "host", "bvh_build_s"), get(line, "bvh_build", n, "device", "bvh_build_s")]
                                       for n in ("spheres-1m", "spheres-8m") if get(line, "bvh_build", n) is not None}}
    serving = line.get("serving")
    if isinstance(serving, dict) and isinstance(serving.get("served"), dict):
        out["serving_latency_s"] = {
            rate: {k: x for k, x in (("served_p50", v.get("p50_latency_s")), ("served_p99", v.get("p99_latency_s")),
                                      ("shortest_first_p50", get(serving, "shortest_first", rate, "p50_latency_s")),
                                      ("shortest_first_p99", get(serving, "shortest_first", rate, "p99_latency_s")),
                                      ("plain_p50", get(serving, "plain", rate, "p50_latency_s")),
                                      ("plain_p99", get(serving, "plain", rate, "p99_latency_s"))) if x is not None}
            for rate, v in serving["served"].items() if isinstance(v, dict)}
        out["serving_jobs_per_rate"] = serving.get("jobs_per_rate")
    return out


def light_sampling_section(knobs, scene_names=("spheres-1m", "spheres-8m"), res=(480, 270), spp=64, ref_spp=4096, trials=3):
    """Power-weighted against area-weighted light selection (and PCG32 against Philox) at equal paths.
    Per scene and mode: the RMSE of a spp-sample frame against a converged ref_spp-sample frame of the
    same mode, accumulated in FP64 and rendered by the deterministic build (whose arithmetic equals the
    CPU oracle's bit for bit), averaged over `trials` independent frames (distinct stream offsets); and
    the product's paths/s on the full-size frame of the headline workload in each mode. "Paths/s at
    equal RMSE" scales a mode's paths/s by (RMSE area / RMSE mode)^2, the factor by which the area mode
    needs more samples for the same error. The shadow-radiance clamp (Intersect.cu:178) makes the two
    modes' converged images differ slightly; that difference is reported too."""
    import pathtracer
    import scenes
    W, H = res
    out = {"config": f"{W}x{H}, {spp} spp vs a {ref_spp}-spp FP64-accumulated frame of the same mode (deterministic build), "
                     f"{trials} trials, depth per workload, NEE",
           "modes": {"area": "LightSampler.cpp:16-19 weights (the reference's)", "power": "area x luminance(emission), FP64 prefix sums",
                     "power_pcg32": "power weights, PCG32 streams"}}
    modes = {"area": (pathtracer.LIGHTS_AREA, pathtracer.RNG_PHILOX), "power": (pathtracer.LIGHTS_POWER, pathtracer.RNG_PHILOX),
             "power_pcg32": (pathtracer.LIGHTS_POWER, pathtracer.RNG_PCG32)}
    for name in scene_names:
        s = scenes.config_scene(name)
        depth = 12 if name == "spheres-1m" else 10
        cam = scenes.scene_camera(s, W, H)
        det = pathtracer.Renderer(0, variant="det")
        prod = pathtracer.Renderer(0)
        res_out = {}
        try:
            det.upload_scene(s)
            prod.upload_scene(s)
            refs = {}
            for m, (lights, rng) in modes.items():
                if m == "power_pcg32":
                    refs[m] = refs["power"]
                    continue
                det.render_frame(cam, W, H, ref_spp, depth, True, light_sampling=lights, rng_offset=1 << 44)
                refs[m] = det.accumulation_fp64() / ref_spp
            for m, (lights, rng) in modes.items():
                errs = []
                for k in range(trials):
                    prod.render_frame(cam, W, H, spp, depth, True, light_sampling=lights, rng_policy=rng, rng_offset=k * W * H * spp,
                                      **knobs)
                    img = prod.accumulation()[:, :3].astype(np.float64) / spp
                    errs.append(float(np.sqrt(np.mean((img - refs[m]) ** 2))))
                res_out[m] = {"rmse": float(np.mean(errs)), "rmse_trials": errs}
            base = res_out["area"]["rmse"]
            for m in res_out:
                res_out[m]["samples_for_equal_rmse_vs_area"] = (res_out[m]["rmse"] / base) ** 2
            res_out["converged_difference_rmse_power_vs_area"] = float(np.sqrt(np.mean((refs["power"] - refs["area"]) ** 2)))
            res_out["converged_rms"] = float(np.sqrt(np.mean(refs["area"] ** 2)))
            if name == WORKLOAD["scene"]:
                fw, fh, fspp = WORKLOAD["width"], WORKLOAD["height"], WORKLOAD["spp"]
                fcam = scenes.scene_camera(s, fw, fh)
                for m, (lights, rng) in modes.items():
                    prod.render_frame(fcam, fw, fh, fspp, depth, True, light_sampling=lights, rng_policy=rng, **knobs)
                    st = [prod.render_frame(fcam, fw, fh, fspp, depth, True, light_sampling=lights, rng_policy=rng, **knobs) for _ in range(2)]
                    ms = sum(x["device_ms"] for x in st) / len(st)
                    pps = st[0]["samples"] / (ms / 1000.0)
                    res_out[m]["full_frame_paths_per_second"] = pps
                    res_out[m]["full_frame_ms"] = ms
                    res_out[m]["paths_per_second_at_equal_rmse"] = pps / res_out[m]["samples_for_equal_rmse_vs_area"]
        finally:
            det.close()
            prod.close()
        out[name] = res_out
    return out


def b200_arm(args):
    import torch
    import pathtracer
    import scenes
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=torch.device("cuda", local))

    W, H, spp, depth = WORKLOAD["width"], WORKLOAD["height"], WORKLOAD["spp"], WORKLOAD["depth"]
    if args.profile_case:
        W, H, spp = 640, 360, 16
        args.no_cpu_baseline = True
    scene = scenes.config_scene(WORKLOAD["scene"])
    renderer = pathtracer.Renderer(local)
    t0 = time.perf_counter()
    renderer.upload_scene(scene)
    upload_s = time.perf_counter() - t0
    upload_breakdown = renderer.upload_times()
    info = renderer.scene_info()
    cam = scenes.scene_camera(scene, W, H)
    import multigpu
    samples_per_frame = spp * W * H
    rng_offset = multigpu.rank_rng_offset(rank, samples_per_frame)
    accum = torch.zeros((W * H, 4), dtype=torch.float32, device="cuda") if world > 1 else None

    loop_mode = pathtracer.LOOP_HOST if args.loop == "host" else pathtracer.LOOP_GRAPH
    tuned = {}
    if not args.no_autotune:
        t0 = time.perf_counter()
        tuned = renderer.autotune(cam, W, H, spp, depth, True)
        tuned["seconds"] = time.perf_counter() - t0
    knobs = dict(pool_size=args.pool or tuned.get("pool_size", WORKLOAD["pool"]),
                 trace_occupancy=tuned.get("trace_occupancy", args.trace_occupancy),
                 trace_refill=tuned.get("trace_refill", args.trace_refill),
                 trace_block=tuned.get("trace_block", args.trace_block))

    exchange = [torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)] if world > 1 else None

    def step():
        st = renderer.render_frame(cam, W, H, spp, depth, True, rng_offset=rng_offset, loop_mode=loop_mode, **knobs)
        if world > 1:
            # the frame's accumulation straight into the collective's buffer (device to device), then one
            # all-reduce over NCCL; both timed with CUDA events on torch's stream and added to the step
            cur = torch.cuda.current_stream()
            exchange[0].record(cur)
            renderer.copy_accumulation_to(accum, stream=cur.cuda_stream)
            multigpu.combine_accumulation(accum, dist)
            exchange[1].record(cur)
            exchange[1].synchronize()
            st["device_ms"] += exchange[0].elapsed_time(exchange[1])
        return st

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    torch.cuda.synchronize()
    wall0 = time.perf_counter()
    stats = [step() for _ in range(args.steps)]
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    wall = time.perf_counter() - wall0
    clocks = sampler.stop()
    # CUDA-event timing of the closest-hit traversal launches: one more frame of the same workload
    # with host-launched iterations (events cannot bracket a node inside the graph's WHILE loop).
    ev = renderer.render_frame(cam, W, H, spp, depth, True, rng_offset=rng_offset, loop_mode=pathtracer.LOOP_HOST, **knobs)

    device_s = sum(s["device_ms"] for s in stats) / 1000.0
    if dist:
        device_s, wall = multigpu.max_over_ranks([device_s, wall], dist, device="cuda")
    paths = sum(s["samples"] for s in stats) * world
    value = paths / device_s
    e2e = paths / wall
    rays = sum(s["rays"] for s in stats)
    shadow = sum(s["shadow_rays"] for s in stats)
    iters = sum(s["iterations"] for s in stats)
    trace_ms = sum(s["phase_ms"]["trace"] for s in stats)
    visits = sum(s["node_visits"][0] for s in stats)
    tests = sum(s["triangle_tests"][0] for s in stats)
    algo_bytes = rays * TRACE_ALGO_BYTES_PER_RAY + visits * NODE_BYTES + tests * TRIANGLE_BYTES
    per_launch_bytes = algo_bytes / iters
    per_launch_s_globaltimer = trace_ms / 1000.0 / iters
    per_launch_s = ev["trace_event_ms"] / 1000.0 / ev["iterations"]
    achieved = per_launch_bytes / per_launch_s / 1e9
    peak, peak_kind = measured_peaks()
    dram_per_ray = profile_dram_bytes_per_ray()
    traffic = dram_per_ray * rays / iters if dram_per_ray else None
    launches = sum(s["kernel_launches"] for s in stats)

    if dist:
        dist.barrier()
    if rank != 0:
        dist.destroy_process_group()
        return 0

    line = {
        "metric": "paths_per_second", "value": value, "unit": "paths/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1000.0 * device_s / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD["workload"], "triangles": info["triangles"], "bvh8_nodes": info["nodes"],
                   "bvh8_depth": info["depth"], "lights": info["lights"], "resolution": f"{W}x{H}", "spp": spp,
                   "depth": depth, "nee": True, "pool": knobs["pool_size"], "knobs": knobs, "autotune": tuned,
                   "l2": "inputs larger than L2 (1.31M-triangle scene, 189 MB shading records, 1.6 GB per-sample radiance)",
                   "parallelism": f"{world} independent frames (distinct Philox subsequences) + NCCL all-reduce of the accumulation" if world > 1 else "1 GPU"},
        "mrays_per_second": (rays + shadow) * world / device_s / 1e6,
        "rays_per_step": (rays + shadow) / args.steps,
        "iterations_per_step": iters / args.steps,
        "phase_ms_per_step": {k: sum(s["phase_ms"][k] for s in stats) / args.steps for k in ("trace", "shade", "shadow", "regen")},
        "scene_upload_s": upload_s,
        "scene_upload_breakdown_s": upload_breakdown,
        "traversal": traversal_summary(stats[-1], NODE_BYTES),
        "roofline": {"kernel": "trace_kernel<closest> (BVH8 closest hit)", "bound": "latency", "achieved": achieved,
                     "peak": peak, "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                     "dram_frac": (traffic / per_launch_s / 1e9 / peak) if traffic else None,
                     "bound_note": "load latency and lane divergence: the algorithmic node/triangle bytes (frac) are served mostly "
                                   "by L1/L2; dram_frac is the DRAM traffic of a launch over its duration against the same peak",
                     "peak_source": peak_kind,
                     "algorithmic_bytes_per_launch": per_launch_bytes,
                     "bytes_model": f"{TRACE_ALGO_BYTES_PER_RAY} B/ray (ray in, material-queue entry out, every ray counted as a hit) + {NODE_BYTES} B/node visited + {TRIANGLE_BYTES} B/triangle tested",
                     "traffic_source": "ncu DRAM bytes per ray of a full-pool launch (profiles/trace_closest_spheres1m.json) x this run's rays per launch",
                     "rays_per_launch": rays / iters,
                     "node_visits_per_ray": visits / max(rays, 1), "triangle_tests_per_ray": tests / max(rays, 1),
                     "avg_launch_ms": per_launch_s * 1000.0,
                     "avg_launch_ms_source": "CUDA events around each closest-hit launch of one host-looped frame of the same workload",
                     "avg_launch_ms_in_graph": per_launch_s_globaltimer * 1000.0,
                     "avg_launch_ms_in_graph_source": "first-block start to last-block end (%globaltimer) of every launch in the timed graph frames"},
        "gpu_launches": launches,
        "loop": args.loop,
        "host_loop_frame_ms": ev["device_ms"],
        "e2e": {"value": e2e, "unit": "paths/s", "h2d_bytes_per_step": 128,
                "d2h_bytes_per_step": W * H * 4 + 256,
                "note": "gpt_render_frame per step: job parameters host->device, frame graph, RGBA8 frame and counters device->host"},
    }
    if clocks:
        line["clocks"] = clocks
    if world == 1 and not args.profile_case and not args.no_reference_build:
        try:
            import ref_harness
        except ImportError:
            ref_harness = None
        if ref_harness is not None and ref_harness.available():
            # The reference's own kernels (oracle/_ref, built from its sources for sm_100a) on the same
            # GPU, driven through its launchers with its host-synchronised loop, pool of 1,048,576 slots.
            R = ref_harness.RefScene(scene)
            frames = [R.render(cam, W, H, spp, depth, True) for _ in range(2)]
            R.close()
            ref_ms = min(f["frame_ms"] for f in frames)
            line["reference_build_b200"] = {"value": samples_per_frame / (ref_ms / 1000.0), "unit": "paths/s",
                                            "ms_per_frame": ref_ms, "iterations": frames[-1]["iterations"],
                                            "speedup_of_value": value / (samples_per_frame / (ref_ms / 1000.0)),
                                            "what": "reference kernels (Intersect/PathGeneration/MaterialEval/Iteration.cu) compiled for sm_100a, replayed RenderFrame loop"}
    sections = wanted_sections(args) if (world == 1 and not args.profile_case) else set()
    per_scene = {WORKLOAD["workload"]: {"value": value, "unit": "paths/s", "mrays_per_second": line["mrays_per_second"],
                                        "config": "1920x1080, 64 spp, depth 12, NEE"}}
    timings = {}

    def run_section(name, fn):
        t0 = time.perf_counter()
        try:
            return fn()
        except Exception as e:  # a failed section is reported, the rest of the line stands
            return {"error": f"{type(e).__name__}: {e}"}
        finally:
            timings[name] = time.perf_counter() - t0

    if "plain" in sections:
        pf = run_section("plain", lambda: plain_form(renderer, cam, W, H, spp, depth))
        if "value" in pf:
            pf["speedup_of_value"] = value / pf["value"]
        line["plain_form"] = pf
    renderer.close()
    if "cornell" in sections:
        per_scene["cornell"] = run_section("cornell", lambda: cornell_section(knobs))
    if "batched" in sections:
        line["batched"] = run_section("batched", lambda: batched_section(knobs))
    if "serving" in sections:
        rates = [float(x) for x in args.serve_rates.split(",") if x.strip()]
        line["serving"] = run_section("serving", lambda: serving_section(knobs, rates, args.serve_jobs, args.serve_pool,
                                                                           short_seconds=args.serve_short_seconds,
                                                                           shortest_first=args.serve_shortest_first))
    if "precision" in sections:
        pr = run_section("precision", lambda: precision_section(knobs))
        line["precision"] = pr
        if "bvh" in pr:
            per_scene["spheres-8m"] = {"value": pr["bvh"]["bvh8_q8"]["paths_per_second"], "unit": "paths/s",
                                       "config": "3840x2160, 16 spp, depth 10, NEE"}
    if "lights" in sections:
        line["light_sampling"] = run_section("lights", lambda: light_sampling_section(knobs))
    if "bvh" in sections:
        line["bvh_build"] = run_section("bvh", lambda: bvh_build_section(knobs))
    if sections:
        line["per_scene"] = per_scene
        line["section_seconds"] = timings
    if world == 1 and not args.no_cpu_baseline:
        import oracle
        threads = oracle.default_threads()
        total, times, sample = run_cpu(WORKLOAD["scene"], args.cpu_seconds, threads, steps=1)
        line["cpu_baseline"] = {"value": total / times[0], "unit": "paths/s", "cores": threads, "kind": "port",
                                "sample": sample}
    line["summary"] = summary(line)  # last key: a truncated tail of the line still carries it
    print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return reference_arm(args)
    return b200_arm(args)


if __name__ == "__main__":
    sys.exit(main())
