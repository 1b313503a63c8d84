"""Parity of the sm_100a path (through the C ABI) with the oracle, on the same seeded inputs.

Bar: bit-exact hit triangle ids, queue counts and alias-table entries; per-path (per-sample)
radiance within 1e-4 relative (the kernels and the oracle follow the same IEEE operation order,
so they are expected to agree bit for bit; the tolerance is the stated bar); converged image
within a stated RMSE of the FP64-accumulated oracle.
"""
import ctypes
import json
import os
import tempfile
import time

import numpy as np
import pytest

import oracle
import pathtracer
import scenes

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
INVALID = 0xFFFFFFFF
RADIANCE_RTOL = 1e-4


def kat_lib():
    path = os.path.join(HERE, "kat", "libphilox_kat.so")
    if not os.path.exists(path):
        import subprocess
        subprocess.run(["make", "-s", "-C", os.path.join(HERE, "kat")], check=True)
    L = ctypes.CDLL(path)
    L.philox_kat.restype = ctypes.c_int
    L.philox_kat.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                             ctypes.c_void_p, ctypes.c_void_p]
    return L


def run_kat(subseq, offsets):
    import torch
    s = torch.tensor(np.asarray(subseq, dtype=np.uint64).view(np.int64), device="cuda")
    o = torch.tensor(np.asarray(offsets, dtype=np.uint32).view(np.int32), device="cuda")
    n, k = len(subseq), len(offsets)
    sched = torch.zeros((n, 14), dtype=torch.float32, device="cuda")
    reinit = torch.zeros((n, k, 4), dtype=torch.float32, device="cuda")
    words = torch.zeros((n, 8), dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    rc = kat_lib().philox_kat(s.data_ptr(), n, o.data_ptr(), k, sched.data_ptr(), reinit.data_ptr(), words.data_ptr())
    assert rc == 0
    return sched.cpu().numpy(), reinit.cpu().numpy(), words.cpu().numpy().view(np.uint32)


def test_oracle_philox_matches_device_curand():
    subseq = [0, 1, 2, 3, 1000, 123456789, 2**32 + 5, 2**40 + 77]
    sched, _, words = run_kat(subseq, [0])
    for i, s in enumerate(subseq):
        w, u = oracle.philox_words(s, 0, 17)
        assert np.array_equal(words[i], w[:8]), s
        assert np.array_equal(sched[i], u[:14]), s


def test_curand_reinit_at_offset_continues_the_stream():
    # the path slots keep (sample, stream position) instead of the 64-byte curand state
    subseq = list(range(0, 4096, 7))
    offsets = [0, 1, 4, 5, 8, 9, 13, 40, 41, 42, 43]
    _, reinit, _ = run_kat(subseq, offsets)
    for i, s in enumerate(subseq):
        _, u = oracle.philox_words(s, 0, 48)
        for k, off in enumerate(offsets):
            assert np.array_equal(reinit[i, k], u[off:off + 4]), (s, off)


@pytest.fixture(scope="module")
def cornell(gpu_renderer, scene_factory, oracle_scene):
    s = scene_factory("cornell")
    gpu_renderer.upload_scene(s)
    return gpu_renderer, s, oracle_scene("cornell")


def test_hit_ids_cornell_1m_rays_bit_exact(cornell):
    r, s, o = cornell
    rays = scenes.hit_ray_set(s, 1 << 20, seed=11)
    tri_g, uvt_g = r.trace_closest_np(rays)
    tri_o, uvt_o = o.trace_closest(rays)
    assert np.array_equal(tri_g, tri_o)
    hit = tri_o != INVALID
    assert hit.mean() > 0.5
    assert np.array_equal(uvt_g[hit].view(np.uint32), uvt_o[hit].view(np.uint32))


def test_any_hit_cornell_bit_exact(cornell):
    r, s, o = cornell
    rays = scenes.hit_ray_set(s, 1 << 18, seed=12)
    tri, uvt = o.trace_closest(rays)
    t = np.where(tri != INVALID, uvt[:, 2], 10.0)
    rays[0::2, 7] = t[0::2] * 0.999
    rays[1::2, 7] = t[1::2] * 1.001
    occ_g = r.trace_any_np(rays)
    occ_o = o.trace_any(rays)
    assert np.array_equal(occ_g, occ_o)
    assert occ_o[1::2].mean() > 0.5


def test_alias_table_bit_exact(cornell):
    r, s, o = cornell
    assert np.array_equal(r.alias_table(), o.alias_table().view(np.uint32).reshape(-1, 4))


def assert_render_parity(r, o, cam, w, h, spp, depth, nee, pool=1 << 20):
    stats = r.render_frame(cam, w, h, spp, depth, nee, pool_size=pool)
    ref = o.render(cam, w, h, spp, depth, nee, pool_size=pool, accumulation=1)
    assert stats["samples"] == ref["total_samples"]
    assert stats["iterations"] == ref["iterations"]
    log = r.queue_log()
    assert np.array_equal(log, ref["queue_log"])
    rad_g, rad_o = r.sample_radiance(), ref["sample_radiance"]
    assert np.all(np.isfinite(rad_g))
    err = np.abs(rad_g - rad_o)
    assert np.all(err <= RADIANCE_RTOL * np.maximum(np.abs(rad_o), 1e-6)), float(err.max())
    exact = float(np.mean(np.all(rad_g.view(np.uint32) == rad_o.view(np.uint32), axis=1)))
    acc = r.accumulation()
    assert np.all(np.abs(acc - ref["accumulation"]) <= RADIANCE_RTOL * np.maximum(np.abs(ref["accumulation"]), 1e-6))
    fb = r.framebuffer()
    assert np.max(np.abs(fb.view(np.uint8).astype(int) - ref["framebuffer"].view(np.uint8).astype(int))) <= 1
    return stats, exact, ref


def test_render_cornell_c1_parity(cornell):
    """512x512, 16 spp, depth 8, NEE, 2-entry alias table."""
    r, s, o = cornell
    cam = scenes.scene_camera(s, 512, 512)
    stats, exact, ref = assert_render_parity(r, o, cam, 512, 512, 16, 8, True)
    assert exact == 1.0
    assert np.array_equal(r.framebuffer(), ref["framebuffer"])


def test_render_cornell_small_pool_parity(cornell):
    # pool smaller than the frame: exercises regeneration across many iterations
    r, s, o = cornell
    cam = scenes.scene_camera(s, 64, 64)
    _, exact, _ = assert_render_parity(r, o, cam, 64, 64, 16, 8, True, pool=5000)
    assert exact == 1.0


@pytest.mark.parametrize("nee", [True, False])
def test_render_all_shading_models_parity(gpu_renderer, scene_factory, oracle_scene, nee):
    s = scene_factory("cornell-all")
    o = oracle_scene("cornell-all")
    gpu_renderer.upload_scene(s)
    cam = scenes.scene_camera(s, 128, 128)
    _, exact, _ = assert_render_parity(gpu_renderer, o, cam, 128, 128, 16, 10, nee)
    assert exact == 1.0
    assert np.array_equal(gpu_renderer.alias_table(), o.alias_table().view(np.uint32).reshape(-1, 4))


def test_render_spheres_parity(gpu_renderer, scene_factory, oracle_scene):
    s = scene_factory("spheres-small")
    o = oracle_scene("spheres-small")
    gpu_renderer.upload_scene(s)
    cam = scenes.scene_camera(s, 96, 64)
    _, exact, _ = assert_render_parity(gpu_renderer, o, cam, 96, 64, 4, 12, True, pool=3000)
    assert exact == 1.0
    assert np.array_equal(gpu_renderer.alias_table(), o.alias_table().view(np.uint32).reshape(-1, 4))


def test_hit_ids_spheres_200k_bit_exact(gpu_renderer, scene_factory, oracle_scene):
    s = scene_factory("spheres-200k")
    o = oracle_scene("spheres-200k")
    gpu_renderer.upload_scene(s)
    rays = scenes.hit_ray_set(s, 1 << 20, seed=13)
    tri_g, uvt_g = gpu_renderer.trace_closest_np(rays)
    tri_o, uvt_o = o.trace_closest(rays)
    assert np.array_equal(tri_g, tri_o)
    hit = tri_o != INVALID
    assert np.array_equal(uvt_g[hit].view(np.uint32), uvt_o[hit].view(np.uint32))
    assert np.array_equal(gpu_renderer.alias_table(), o.alias_table().view(np.uint32).reshape(-1, 4))


def test_converged_image_rmse_vs_fp64_oracle(gpu_renderer, scene_factory, oracle_scene):
    s = scene_factory("cornell")
    o = oracle_scene("cornell")
    gpu_renderer.upload_scene(s)
    cam = scenes.scene_camera(s, 48, 48)
    gpu_renderer.render_frame(cam, 48, 48, 1024, 8, True)
    ref = o.render(cam, 48, 48, 1024, 8, True, accumulation=2)
    g = gpu_renderer.accumulation()[:, :3] / 1024.0
    f = ref["accumulation"][:, :3].astype(np.float64) / 1024.0
    rmse = float(np.sqrt(np.mean((g - f) ** 2)))
    assert rmse <= 1e-6 * max(1.0, float(np.sqrt(np.mean(f ** 2))))


def test_render_errors_and_clear(gpu_renderer, scene_factory):
    import pathtracer as P
    fresh = P.Renderer(0)
    with pytest.raises(P.GptError) as e:
        fresh.render_frame(np.zeros(12, np.float32), 8, 8, 1, 1)
    assert e.value.code == 5
    fresh.init_rendering_buffers(16, 8)
    fresh.clear(10, 20, 30, 255)
    fb = fresh.lock_frame()
    assert fb.size == 128 and np.all(fb == (10 | 20 << 8 | 30 << 16 | 255 << 24))
    with pytest.raises(P.GptError) as e:
        fresh.upload_times()
    assert e.value.code == 5
    fresh.close()


def test_scene_upload_times(gpu_renderer, scene_factory):
    """The upload reports the host BVH build inside the whole upload's wall time."""
    import time as _time
    s = scene_factory("spheres-200k")
    t0 = _time.perf_counter()
    gpu_renderer.upload_scene(s)
    wall = _time.perf_counter() - t0
    t = gpu_renderer.upload_times()
    assert 0.0 < t["bvh_build_s"] < t["upload_s"] <= wall


def test_simulation_thread_frames_stop_resume(gpu_renderer, scene_factory):
    s = scene_factory("cornell")
    gpu_renderer.upload_scene(s)
    states = [((0.5, 0.5, 2.0 + 0.1 * k), (1.0, 0.0, 0.0, 0.0)) for k in range(3)]
    with tempfile.TemporaryDirectory() as d:
        gpu_renderer.start_simulation(64, 48, np.radians(40.0), states, 4, 6, d, True)
        with pytest.raises(pathtracer.GptError):
            gpu_renderer.start_simulation(64, 48, np.radians(40.0), states, 4, 6, d, True)
        t0 = time.time()
        while gpu_renderer.is_rendering() and time.time() - t0 < 60:
            time.sleep(0.01)
        assert not gpu_renderer.is_rendering()
        p = gpu_renderer.progress()
        assert p["done_frames"] == 3 and p["total_frames"] == 3 and p["total_samples"] == 4 * 64 * 48
        files = sorted(os.listdir(d))
        assert files == ["frame_0000.png", "frame_0001.png", "frame_0002.png"]
        assert open(os.path.join(d, files[0]), "rb").read(8) == b"\x89PNG\r\n\x1a\n"
        frame = gpu_renderer.lock_frame()
        assert frame.size == 64 * 48 and np.any(frame != 0)
        gpu_renderer.resume_simulation(2)
        while gpu_renderer.is_rendering() and time.time() - t0 < 60:
            time.sleep(0.01)
        assert gpu_renderer.progress()["done_frames"] == 3
        with pytest.raises(pathtracer.GptError):
            gpu_renderer.resume_simulation(3)
    # stop mid-run: the device loop ends at the next iteration through the host-mapped flag
    gpu_renderer.start_simulation(256, 256, np.radians(40.0), states * 4, 256, 8, None, True)
    time.sleep(0.05)
    gpu_renderer.stop_rendering()
    assert not gpu_renderer.is_rendering()
    assert gpu_renderer.progress()["done_frames"] < 12
    assert gpu_renderer.last_error() is None
    # a stopped simulation does not cut later frames short
    cam = scenes.scene_camera(s, 32, 32)
    st = gpu_renderer.render_frame(cam, 32, 32, 4, 8, True)
    assert st["samples"] == 4 * 32 * 32
    ref = oracle.OracleScene(s).render(cam, 32, 32, 4, 8, True)
    assert st["iterations"] == ref["iterations"]
    assert np.array_equal(gpu_renderer.sample_radiance().view(np.uint32), ref["sample_radiance"].view(np.uint32))


def test_host_loop_matches_graph_loop(gpu_renderer, scene_factory, oracle_scene):
    """The host-driven iteration loop (the reference's structure) and the device-driven graph
    loop run the same kernels: identical per-sample radiance and queue counts."""
    import pathtracer as P
    s = scene_factory("cornell-all")
    gpu_renderer.upload_scene(s)
    cam = scenes.scene_camera(s, 64, 64)
    a = gpu_renderer.render_frame(cam, 64, 64, 16, 10, True, pool_size=9000, loop_mode=P.LOOP_GRAPH)
    rad_a, log_a = gpu_renderer.sample_radiance(), gpu_renderer.queue_log()
    b = gpu_renderer.render_frame(cam, 64, 64, 16, 10, True, pool_size=9000, loop_mode=P.LOOP_HOST)
    rad_b, log_b = gpu_renderer.sample_radiance(), gpu_renderer.queue_log()
    assert a["iterations"] == b["iterations"]
    assert np.array_equal(log_a, log_b)
    assert np.array_equal(rad_a.view(np.uint32), rad_b.view(np.uint32))
    assert b["trace_event_ms"] > 0.0


def test_autotune_returns_valid_knobs_and_results_do_not_change(gpu_renderer, scene_factory):
    s = scene_factory("spheres-small")
    gpu_renderer.upload_scene(s)
    cam = scenes.scene_camera(s, 128, 96)
    knobs = gpu_renderer.autotune(cam, 128, 96, 16, 12, True)
    assert knobs["candidates"] >= 12 and knobs["trial_ms"] > 0
    assert knobs["pool_size"] in (1 << 20, 2 << 20, 4 << 20, 8 << 20, 16 << 20)
    assert knobs["trace_occupancy"] in (1, 10, 12) and knobs["trace_block"] in (64, 128)
    assert knobs["trace_refill"] & 0xFF in (8, 16) and knobs["trace_refill"] >> 8 in (0, 2, 4, 8, 16)
    gpu_renderer.render_frame(cam, 128, 96, 16, 12, True)
    a = gpu_renderer.sample_radiance()
    gpu_renderer.render_frame(cam, 128, 96, 16, 12, True, pool_size=knobs["pool_size"], trace_occupancy=knobs["trace_occupancy"],
                              trace_refill=knobs["trace_refill"], trace_block=knobs["trace_block"])
    b = gpu_renderer.sample_radiance()
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


def test_rng_offset_shards_match_oracle(gpu_renderer, scene_factory, oracle_scene):
    """A rank's shard (Philox subsequences offset by rank x samples per frame) equals the oracle's."""
    import multigpu
    s = scene_factory("cornell-all")
    o = oracle_scene("cornell-all")
    gpu_renderer.upload_scene(s)
    cam = scenes.scene_camera(s, 48, 48)
    off = multigpu.rank_rng_offset(3, 16 * 48 * 48)
    gpu_renderer.render_frame(cam, 48, 48, 16, 10, True, rng_offset=off)
    ref = o.render(cam, 48, 48, 16, 10, True, rng_offset=off)
    assert np.array_equal(gpu_renderer.sample_radiance().view(np.uint32), ref["sample_radiance"].view(np.uint32))
    assert np.array_equal(gpu_renderer.queue_log(), ref["queue_log"])


def test_copy_accumulation_device_matches_host_read(gpu_renderer, scene_factory):
    """gpt_copy_accumulation_device (the multi-GPU exchange's source) copies the same float4
    accumulation gpt_read_accumulation returns, on the renderer's stream or on a caller's stream."""
    import torch
    s = scene_factory("cornell")
    gpu_renderer.upload_scene(s)
    cam = scenes.scene_camera(s, 40, 30)
    gpu_renderer.render_frame(cam, 40, 30, 4, 6, True)
    host = gpu_renderer.accumulation()
    dev = torch.full((40 * 30, 4), -1.0, dtype=torch.float32, device="cuda")
    gpu_renderer.copy_accumulation_to(dev)
    assert np.array_equal(dev.cpu().numpy().view(np.uint32), host.view(np.uint32))
    dev2 = torch.zeros_like(dev)
    cur = torch.cuda.current_stream()
    gpu_renderer.copy_accumulation_to(dev2, stream=cur.cuda_stream)
    cur.synchronize()
    assert np.array_equal(dev2.cpu().numpy().view(np.uint32), host.view(np.uint32))


def test_fp64_reference_accumulation_on_device(gpu_renderer, scene_factory):
    """gpt_read_accumulation_fp64 sums every pixel's samples in FP64 in sample order: equal, bit for bit,
    to the same sum taken on the host from the per-sample radiance; the FP32 Kahan accumulation stays
    within a few FP32 ulps of it."""
    s = scene_factory("cornell-all")
    gpu_renderer.upload_scene(s)
    cam = scenes.scene_camera(s, 48, 40)
    gpu_renderer.render_frame(cam, 48, 40, 16, 8, True)
    fp64 = gpu_renderer.accumulation_fp64()
    rad = gpu_renderer.sample_radiance().reshape(48 * 40, 16, 3)
    ref = np.zeros((48 * 40, 3), dtype=np.float64)
    for k in range(16):
        ref += rad[:, k, :].astype(np.float64)
    assert np.array_equal(fp64.view(np.uint64), ref.view(np.uint64))
    kahan = gpu_renderer.accumulation()[:, :3].astype(np.float64)
    assert np.all(np.abs(kahan - fp64) <= 4 * np.spacing(np.abs(fp64).astype(np.float32)).astype(np.float64) + 1e-30)


def decode_png_rgba8(path):
    """A PNG's RGBA8 pixels [h, w, 4], rows top to bottom, with every chunk CRC checked (filters 0-4)."""
    import struct
    import zlib
    data = open(path, "rb").read()
    assert data[:8] == b"\x89PNG\r\n\x1a\n"
    pos, idat, w, h = 8, b"", None, None
    while pos < len(data):
        length, ctype = struct.unpack(">I4s", data[pos:pos + 8])
        body = data[pos + 8:pos + 8 + length]
        assert zlib.crc32(ctype + body) & 0xFFFFFFFF == struct.unpack(">I", data[pos + 8 + length:pos + 12 + length])[0]
        if ctype == b"IHDR":
            w, h, bit_depth, color = struct.unpack(">IIBB", body[:10])
            assert (bit_depth, color) == (8, 6)
        elif ctype == b"IDAT":
            idat += body
        elif ctype == b"IEND":
            break
        pos += 12 + length
    raw = zlib.decompress(idat)
    stride = 4 * w
    out = np.zeros((h, stride), np.int64)
    prev = np.zeros(stride, np.int64)
    for y in range(h):
        f = raw[y * (stride + 1)]
        line = np.frombuffer(raw, np.uint8, stride, y * (stride + 1) + 1).astype(np.int64)
        cur = np.zeros(stride, np.int64)
        for i in range(stride):
            a = cur[i - 4] if i >= 4 else 0
            b = prev[i]
            c = prev[i - 4] if i >= 4 else 0
            if f == 0:
                pred = 0
            elif f == 1:
                pred = a
            elif f == 2:
                pred = b
            elif f == 3:
                pred = (a + b) // 2
            else:
                p = a + b - c
                pa, pb, pc = abs(p - a), abs(p - b), abs(p - c)
                pred = a if pa <= pb and pa <= pc else (b if pb <= pc else c)
            cur[i] = (line[i] + pred) & 255
        out[y] = cur
        prev = cur
    return out.astype(np.uint8).reshape(h, w, 4)


def test_simulation_sequence_frames_and_pngs_match_oracle(gpu_renderer, scene_factory, oracle_scene):
    """A recorded camera path resampled to frames (gpt_resample_motion), rendered by the simulation
    thread (StartSimulation, Renderer.cpp:401-466): every saved PNG holds, vertically flipped
    (SaveRenderedFrame, Renderer.cpp:649-675), the oracle's framebuffer for that frame's camera
    (MakeDeviceCamera from the resampled state), bit for bit; the locked frame is the last one."""
    s = scene_factory("cornell-all")
    o = oracle_scene("cornell-all")
    gpu_renderer.upload_scene(s)
    W, H, spp, depth = 40, 30, 4, 8
    fov = np.float32(np.radians(40.0))
    path = [((0.5, 0.5, 2.2), (1.0, 0.0, 0.0, 0.0), 0.0),
            ((0.6, 0.55, 2.0), (0.9962, 0.0, 0.0872, 0.0), 0.5),
            ((0.7, 0.5, 1.9), (0.9848, 0.0, 0.1736, 0.0), 1.2)]
    states = pathtracer.resample_motion(path, 0.4)
    assert len(states) == 4
    with tempfile.TemporaryDirectory() as d:
        gpu_renderer.start_simulation(W, H, float(fov), states, spp, depth, d, True)
        t0 = time.time()
        while gpu_renderer.is_rendering() and time.time() - t0 < 60:
            time.sleep(0.01)
        assert gpu_renderer.progress()["done_frames"] == len(states)
        aspect = float(np.float32(W) / np.float32(H))
        for k, (pos, quat) in enumerate(states):
            cam = pathtracer.make_device_camera(float(fov), aspect, pos, quat)
            ref = o.render(cam, W, H, spp, depth, True)["framebuffer"]
            png = decode_png_rgba8(os.path.join(d, f"frame_{k:04d}.png"))
            expect = ref.view(np.uint8).reshape(H, W, 4)[::-1]
            assert np.array_equal(png, expect), k
        assert np.array_equal(gpu_renderer.lock_frame(), ref)


def test_imported_obj_scene_renders_like_the_oracle(gpu_renderer, tmp_path):
    """An OBJ/MTL file (every shading model, constant materials) through gpt_obj_load: the
    deterministic build renders it as the oracle does, bit for bit."""
    from test_obj_import import write_obj
    s = scenes.cornell_all_models(1)
    imported = pathtracer.load_obj(write_obj(s, str(tmp_path)))
    imported.camera = s.camera
    o = oracle.OracleScene(imported)
    gpu_renderer.upload_scene(imported)
    cam = scenes.scene_camera(s, 64, 48)
    st = gpu_renderer.render_frame(cam, 64, 48, 4, 10, True)
    ref = o.render(cam, 64, 48, 4, 10, True)
    assert st["iterations"] == ref["iterations"]
    assert np.array_equal(gpu_renderer.queue_log(), ref["queue_log"])
    assert np.array_equal(gpu_renderer.sample_radiance().view(np.uint32), ref["sample_radiance"].view(np.uint32))
    assert np.array_equal(gpu_renderer.framebuffer(), ref["framebuffer"])


def test_yaml_scene_file_renders_like_the_oracle(gpu_renderer, tmp_path):
    """A scene file in the reference's YAML format (two OBJ models, a rotated parent, a scaled child,
    a look-at camera) through scene_file.load_scene: the deterministic build renders it as the oracle
    does, bit for bit."""
    import scene_file
    from test_obj_import import write_obj
    root = tmp_path / "Assets"
    for d in ("Models/Room", "Models/Ball", "Scenes"):
        (root / d).mkdir(parents=True)
    write_obj(scenes.cornell_all_models(1), str(root / "Models/Room"))
    write_obj(scenes.sphere_field(1, 2, 2, 3, name="ball"), str(root / "Models/Ball"))
    (root / "Scenes/room.yaml").write_text("""
scene:
    - components:
        - type: Transform
          translation: [0.5, 0.5, 2.2]
          target: [0.5, 0.45, 0.0]
          scale: [1.0, 1.0, 1.0]
        - type: Camera
          fov-y: 40.0
          near-plane: 0.1
          far-plane: 100.0
    - components:
        - type: Transform
          translation: [0.5, 0.0, 0.5]
          euler-degrees: [0.0, 10.0, 0.0]
          scale: [1.0, 1.0, 1.0]
      children:
        - components:
            - type: Transform
              translation: [-0.5, 0.0, -0.5]
              scale: [1.0, 1.0, 1.0]
            - type: Model
              path: Models/Room/scene.obj
        - components:
            - type: Transform
              translation: [-0.2, 0.15, 0.1]
              scale: [0.01, 0.01, 0.01]
            - type: Model
              path: Models/Ball/scene.obj
""")
    s = scene_file.load_scene(str(root / "Scenes/room.yaml"))
    o = oracle.OracleScene(s)
    gpu_renderer.upload_scene(s)
    cam = scene_file.device_camera(s, 64, 48)
    st = gpu_renderer.render_frame(cam, 64, 48, 4, 10, True)
    ref = o.render(cam, 64, 48, 4, 10, True)
    assert st["iterations"] == ref["iterations"]
    assert np.array_equal(gpu_renderer.queue_log(), ref["queue_log"])
    assert np.array_equal(gpu_renderer.sample_radiance().view(np.uint32), ref["sample_radiance"].view(np.uint32))
    assert np.array_equal(gpu_renderer.framebuffer(), ref["framebuffer"])
    assert np.count_nonzero(ref["framebuffer"]) > 0
