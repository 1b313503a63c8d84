"""The two BVH formats of the frame renderer give the same results bit for bit.

GPT_BVH8_Q8 (8-wide, 8-bit quantised child boxes, 128-byte nodes, shared-memory stack) and
GPT_BVH2_FP32 (the binary tree it is collapsed from, FP32 child boxes, 64-byte nodes, local-memory
stack) are both conservative: neither culls a box that holds the closest hit, so closest-hit
triangles, (u, v, t), occlusion bits, per-sample radiance and images agree exactly, and both agree
with the oracle's traversal of the reference's median-split BVH.
"""
import numpy as np
import pytest

import pathtracer as P
import scenes

pytestmark = pytest.mark.gpu

INVALID = 0xFFFFFFFF


@pytest.mark.parametrize("name,seed", [("cornell", 21), ("spheres-200k", 22)])
def test_binary_bvh_closest_hits_bit_exact(gpu_renderer, scene_factory, oracle_scene, name, seed):
    s = scene_factory(name)
    gpu_renderer.upload_scene(s)
    info = gpu_renderer.scene_info()
    assert info["binary_nodes"] > 0 and 0 < info["binary_depth"] <= 64
    rays = scenes.hit_ray_set(s, 1 << 20, seed=seed)
    tri8, uvt8 = gpu_renderer.trace_closest_np(rays, bvh_format=P.BVH8_Q8)
    tri2, uvt2 = gpu_renderer.trace_closest_np(rays, bvh_format=P.BVH2_FP32)
    assert np.array_equal(tri2, tri8)
    hit = tri8 != INVALID
    assert hit.mean() > 0.3
    assert np.array_equal(uvt2[hit].view(np.uint32), uvt8[hit].view(np.uint32))
    tri_o, uvt_o = oracle_scene(name).trace_closest(rays)
    assert np.array_equal(tri2, tri_o)
    assert np.array_equal(uvt2[hit].view(np.uint32), uvt_o[hit].view(np.uint32))


def test_binary_bvh_any_hit_bit_exact(gpu_renderer, scene_factory, oracle_scene):
    s = scene_factory("spheres-200k")
    gpu_renderer.upload_scene(s)
    o = oracle_scene("spheres-200k")
    rays = scenes.hit_ray_set(s, 1 << 18, seed=23)
    tri, uvt = o.trace_closest(rays)
    t = np.where(tri != INVALID, uvt[:, 2], 30.0)
    rays[0::2, 7] = t[0::2] * 0.999
    rays[1::2, 7] = t[1::2] * 1.001
    occ8 = gpu_renderer.trace_any_np(rays, bvh_format=P.BVH8_Q8)
    occ2 = gpu_renderer.trace_any_np(rays, bvh_format=P.BVH2_FP32)
    assert np.array_equal(occ2, occ8)
    assert np.array_equal(occ2, o.trace_any(rays))


@pytest.mark.parametrize("name,w,h,spp,depth,loop", [("cornell-all", 96, 64, 16, 10, P.LOOP_GRAPH),
                                                      ("spheres-small", 96, 64, 4, 12, P.LOOP_HOST)])
def test_binary_bvh_frames_bit_identical(gpu_renderer, scene_factory, oracle_scene, name, w, h, spp, depth, loop):
    s = scene_factory(name)
    gpu_renderer.upload_scene(s)
    cam = scenes.scene_camera(s, w, h)
    a = gpu_renderer.render_frame(cam, w, h, spp, depth, True, pool_size=5000, bvh_format=P.BVH8_Q8)
    rad_a, log_a, fb_a = gpu_renderer.sample_radiance(), gpu_renderer.queue_log(), gpu_renderer.framebuffer()
    # the plain configuration: binary FP32 BVH, warps refilled only when all lanes are idle, the
    # reference's queue structure (regeneration queue, shading in sequence), host loop
    b = gpu_renderer.render_frame(cam, w, h, spp, depth, True, pool_size=5000, bvh_format=P.BVH2_FP32,
                                  trace_refill=32 | (32 << 8), loop_mode=loop, wavefront_layout=P.WAVEFRONT_QUEUES)
    rad_b, log_b, fb_b = gpu_renderer.sample_radiance(), gpu_renderer.queue_log(), gpu_renderer.framebuffer()
    assert a["iterations"] == b["iterations"]
    assert np.array_equal(log_a, log_b)
    assert np.array_equal(rad_a.view(np.uint32), rad_b.view(np.uint32))
    assert np.array_equal(fb_a, fb_b)
    ref = oracle_scene(name).render(cam, w, h, spp, depth, True, pool_size=5000)
    assert np.array_equal(rad_b.view(np.uint32), ref["sample_radiance"].view(np.uint32))
    # the binary tree visits more, smaller nodes than the 8-wide one
    assert b["node_visits"][0] > a["node_visits"][0] > 0


def test_binary_bvh_unknown_format_is_rejected(gpu_renderer, scene_factory):
    s = scene_factory("cornell")
    gpu_renderer.upload_scene(s)
    cam = scenes.scene_camera(s, 8, 8)
    with pytest.raises(P.GptError) as e:
        gpu_renderer.render_frame(cam, 8, 8, 1, 2, True, bvh_format=7)
    assert e.value.code == 1



@pytest.mark.parametrize("loop", [P.LOOP_GRAPH, P.LOOP_HOST])
def test_wavefront_layouts_bit_identical(gpu_renderer, scene_factory, loop):
    """Bitmap regeneration in slot order with concurrent shading (GPT_WAVEFRONT_B200) and the
    reference's queue structure (GPT_WAVEFRONT_QUEUES) hand out the same samples per iteration:
    identical queue sizes, iteration counts and per-sample radiance, with a pool far smaller than
    the frame so that slots are reused many times."""
    s = scene_factory("cornell-all")
    gpu_renderer.upload_scene(s)
    cam = scenes.scene_camera(s, 80, 60)
    a = gpu_renderer.render_frame(cam, 80, 60, 16, 10, True, pool_size=3000, loop_mode=loop, wavefront_layout=P.WAVEFRONT_B200)
    rad_a, log_a = gpu_renderer.sample_radiance(), gpu_renderer.queue_log()
    b = gpu_renderer.render_frame(cam, 80, 60, 16, 10, True, pool_size=3000, loop_mode=loop, wavefront_layout=P.WAVEFRONT_QUEUES)
    rad_b, log_b = gpu_renderer.sample_radiance(), gpu_renderer.queue_log()
    assert a["iterations"] == b["iterations"] > 10
    assert np.array_equal(log_a, log_b)
    assert np.array_equal(rad_a.view(np.uint32), rad_b.view(np.uint32))
    with pytest.raises(P.GptError):
        gpu_renderer.render_frame(cam, 8, 8, 1, 2, True, wavefront_layout=2)
