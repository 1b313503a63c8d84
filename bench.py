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
TRACE_ALGO_BYTES_PER_RAY = 32 + 16 + 4   # ray record read, hit record write, queue index write
NODE_BYTES = 128
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
    return ap.parse_args()


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        d = json.load(open(path))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profile_traffic():
    """DRAM bytes per launch of the closest-hit traversal kernel from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "trace_closest_spheres1m.json")
    if os.path.exists(path):
        d = json.load(open(path))
        return d.get("dram_bytes_per_launch_full_size")
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
                 trace_occupancy=tuned.get("trace_occupancy", 0), trace_refill=tuned.get("trace_refill", 0),
                 trace_block=tuned.get("trace_block", 0))

    def step():
        st = renderer.render_frame(cam, W, H, spp, depth, True, rng_offset=rng_offset, loop_mode=loop_mode, **knobs)
        if world > 1:
            host = renderer.accumulation()
            accum.copy_(torch.from_numpy(host))
            multigpu.combine_accumulation(accum, dist)
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
    traffic = profile_traffic()
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
        "roofline": {"kernel": "trace_kernel<closest> (BVH8 closest hit)", "bound": "hbm", "achieved": achieved,
                     "peak": peak, "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                     "peak_source": peak_kind,
                     "algorithmic_bytes_per_launch": per_launch_bytes,
                     "bytes_model": f"{TRACE_ALGO_BYTES_PER_RAY} B/ray (ray in, hit out, queue index) + {NODE_BYTES} B/node visited + {TRIANGLE_BYTES} B/triangle tested",
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
    if world == 1 and not args.profile_case:
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
    if world == 1 and not args.no_cpu_baseline:
        import oracle
        threads = oracle.default_threads()
        total, times, sample = run_cpu(WORKLOAD["scene"], args.cpu_seconds, threads, steps=1)
        line["cpu_baseline"] = {"value": total / times[0], "unit": "paths/s", "cores": threads, "kind": "port",
                                "sample": sample}
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
