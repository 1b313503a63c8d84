"""Parity at the benchmark's scale (deterministic build against the oracle, bit for bit):

* 2^20 closest-hit and any-hit rays on spheres-1m (1.31M triangles, the headline workload) and
  spheres-8m (8.19M triangles, the precision workload), against both BVH formats (the 8-bit quantised
  BVH8 and the FP32 binary BVH). The deepest trees are where quantised boxes would first cull a
  closest hit.
* per-path radiance of a band of the headline frame's camera at spp = 1: the first 1920 x 136
  samples (the bottom rows) of the 1920x1080 frame, depth 12, NEE.
* jobs of the batched mix rendered by the job server, against the oracle.
"""
import numpy as np
import pytest

import pathtracer
import scenes

pytestmark = pytest.mark.gpu

INVALID = 0xFFFFFFFF


@pytest.mark.parametrize("name", ["spheres-1m", "spheres-8m"])
def test_hits_bit_exact_at_benchmark_scale(gpu_renderer, scene_factory, oracle_scene, name):
    s = scene_factory(name)
    o = oracle_scene(name)
    gpu_renderer.upload_scene(s)
    rays = scenes.hit_ray_set(s, 1 << 20, seed=21)
    tri_o, uvt_o = o.trace_closest(rays)
    hit = tri_o != INVALID
    assert hit.mean() > 0.3
    for fmt in (pathtracer.BVH8_Q8, pathtracer.BVH2_FP32):
        tri_g, uvt_g = gpu_renderer.trace_closest_np(rays, bvh_format=fmt)
        assert np.array_equal(tri_g, tri_o), fmt
        assert np.array_equal(uvt_g[hit].view(np.uint32), uvt_o[hit].view(np.uint32)), fmt
    # any hit: segments ending just before / just after the closest hit
    seg = rays[: 1 << 19].copy()
    t = np.where(tri_o[: 1 << 19] != INVALID, uvt_o[: 1 << 19, 2], 50.0)
    seg[0::2, 7] = t[0::2] * 0.999
    seg[1::2, 7] = t[1::2] * 1.001
    occ_o = o.trace_any(seg)
    for fmt in (pathtracer.BVH8_Q8, pathtracer.BVH2_FP32):
        assert np.array_equal(gpu_renderer.trace_any_np(seg, bvh_format=fmt), occ_o), fmt


def test_headline_frame_band_per_path_bit_exact(gpu_renderer, scene_factory, oracle_scene):
    s = scene_factory("spheres-1m")
    o = oracle_scene("spheres-1m")
    gpu_renderer.upload_scene(s)
    W, H = 1920, 1080
    band = W * 136
    cam = scenes.scene_camera(s, W, H)
    st = gpu_renderer.render_frame(cam, W, H, 1, 12, True, max_samples=band)
    ref = o.render(cam, W, H, 1, 12, True, max_samples=band)
    assert st["samples"] == band == ref["total_samples"]
    assert st["iterations"] == ref["iterations"]
    assert np.array_equal(gpu_renderer.queue_log(), ref["queue_log"])
    rad = gpu_renderer.sample_radiance()
    assert np.array_equal(rad.view(np.uint32), ref["sample_radiance"].view(np.uint32))
    assert (rad.sum(1) > 0).mean() > 0.3  # the band sees lit geometry


def test_served_mix_jobs_match_the_oracle(scene_factory, oracle_scene):
    """Jobs of the batched mix (their own orbit cameras) submitted together to the deterministic
    build's job server: each image and accumulation is the oracle's."""
    import workloads
    resident = {n: scene_factory(n) for n in ("spheres-10k", "spheres-200k")}
    srv = pathtracer.Server(0, pool_size=1 << 18, hbm_budget_bytes=2 << 30, variant="det")
    try:
        ids = {n: srv.add_scene(sc) for n, sc in resident.items()}
        jobs = [j for j in workloads.batched_jobs() if j.scene in resident][:4]
        jobs = [workloads.Job(j.scene, min(j.width, 200), min(j.height, 150), min(j.spp, 16), j.depth, j.camera) for j in jobs]
        jids = [srv.submit(ids[j.scene], j.camera, j.width, j.height, j.spp, j.depth, True, keep_accumulation=True) for j in jobs]
        for j, jid in zip(jobs, jids):
            st = srv.wait(jid, 600)
            assert st["state"] == "done"
            fb, acc = srv.result(jid, accumulation=True)
            ref = oracle_scene(j.scene).render(j.camera, j.width, j.height, j.spp, j.depth, True)
            assert np.array_equal(fb, ref["framebuffer"]), j
            assert np.array_equal(acc.view(np.uint32), ref["accumulation"].view(np.uint32)), j
            srv.release(jid)
    finally:
        srv.close()
