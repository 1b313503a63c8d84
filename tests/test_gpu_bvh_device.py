"""BVH8 built on the device (gpt_set_bvh_build(GPT_BVH_BUILD_DEVICE)).

The device builder orders triangles by Morton code, clusters nearest neighbours into a binary tree
and collapses it with the host builder's 8-wide collapse and quantisation. Its tree differs from the
host's binned-SAH tree, but the traversal is conservative and closest-hit ties go to the smaller
input index, so hits, per-sample radiance and images must equal those of the host-built BVH (and of
the oracle) bit for bit; only the traversal work may differ.
"""
import dataclasses

import numpy as np
import pytest

import pathtracer as P
import scenes

pytestmark = pytest.mark.gpu

INVALID = 0xFFFFFFFF


@pytest.fixture(scope="module")
def device_renderer():
    r = P.Renderer(0, variant="det")
    r.set_bvh_build(P.BVH_BUILD_DEVICE)
    yield r
    r.close()


@pytest.fixture(scope="module")
def host_renderer():
    r = P.Renderer(0, variant="det")
    yield r
    r.close()


def check(r, s):
    c = r.check_bvh(s)
    assert c["containment_violations"] == 0
    assert c["triangles_not_exactly_once"] == 0
    assert c["leaf_triangles"] == s.triangle_count


@pytest.mark.parametrize("name", ["cornell", "cornell-all", "spheres-small", "spheres-200k"])
def test_device_bvh_is_valid_and_hits_equal_the_host_bvh(device_renderer, host_renderer, scene_factory, oracle_scene, name):
    s = scene_factory(name)
    device_renderer.upload_scene(s)
    host_renderer.upload_scene(s)
    check(device_renderer, s)
    check(host_renderer, s)  # the same checker holds for the host-built tree
    info, host_info = device_renderer.scene_info(), host_renderer.scene_info()
    assert info["binary_nodes"] == 0 and host_info["binary_nodes"] > 0  # no binary FP32 BVH from the device build
    assert 0 < info["depth"] <= 64 and info["nodes"] > 0
    rays = scenes.hit_ray_set(s, 1 << 20, seed=31)
    tri_d, uvt_d = device_renderer.trace_closest_np(rays)
    tri_h, uvt_h = host_renderer.trace_closest_np(rays)
    assert np.array_equal(tri_d, tri_h)
    hit = tri_d != INVALID
    assert hit.mean() > 0.3
    assert np.array_equal(uvt_d[hit].view(np.uint32), uvt_h[hit].view(np.uint32))
    tri_o, _ = oracle_scene(name).trace_closest(rays)
    assert np.array_equal(tri_d, tri_o)
    # shadow rays ending just before and just after the closest hit
    t = np.where(hit, uvt_h[:, 2], 30.0)
    rays = rays[: 1 << 18].copy()
    rays[0::2, 7] = t[: 1 << 18][0::2] * 0.999
    rays[1::2, 7] = t[: 1 << 18][1::2] * 1.001
    assert np.array_equal(device_renderer.trace_any_np(rays), host_renderer.trace_any_np(rays))


@pytest.mark.parametrize("name,w,h,spp,depth", [("cornell-all", 96, 64, 16, 10), ("spheres-small", 96, 64, 4, 12)])
def test_device_bvh_frames_equal_the_host_bvh(device_renderer, host_renderer, scene_factory, oracle_scene, name, w, h, spp, depth):
    s = scene_factory(name)
    device_renderer.upload_scene(s)
    host_renderer.upload_scene(s)
    cam = scenes.scene_camera(s, w, h)
    a = device_renderer.render_frame(cam, w, h, spp, depth, True, pool_size=5000)
    b = host_renderer.render_frame(cam, w, h, spp, depth, True, pool_size=5000)
    assert a["iterations"] == b["iterations"]
    assert np.array_equal(device_renderer.queue_log(), host_renderer.queue_log())
    rad = device_renderer.sample_radiance()
    assert np.array_equal(rad.view(np.uint32), host_renderer.sample_radiance().view(np.uint32))
    assert np.array_equal(device_renderer.framebuffer(), host_renderer.framebuffer())
    ref = oracle_scene(name).render(cam, w, h, spp, depth, True, pool_size=5000)
    assert np.array_equal(rad.view(np.uint32), ref["sample_radiance"].view(np.uint32))
    assert a["node_visits"][0] > 0 and b["node_visits"][0] > 0


def test_device_bvh_refuses_the_binary_format(device_renderer, scene_factory):
    s = scene_factory("cornell")
    device_renderer.upload_scene(s)
    cam = scenes.scene_camera(s, 8, 8)
    with pytest.raises(P.GptError):
        device_renderer.render_frame(cam, 8, 8, 1, 2, True, bvh_format=P.BVH2_FP32)
    device_renderer.render_frame(cam, 8, 8, 1, 2, True)


@pytest.mark.parametrize("count", [1, 2, 3, 9])
def test_device_bvh_of_a_few_triangles(device_renderer, host_renderer, scene_factory, count):
    """Trees of 1 to 9 triangles (a root that is one leaf, one or two wide levels) give the host BVH's hits."""
    full = scene_factory("cornell-all")
    s = dataclasses.replace(full, positions=full.positions[:count].copy(), normals=full.normals[:count].copy(),
                            tangents=full.tangents[:count].copy(), uvs=full.uvs[:count].copy(),
                            material_ids=full.material_ids[:count].copy())
    device_renderer.upload_scene(s)
    host_renderer.upload_scene(s)
    check(device_renderer, s)
    rays = scenes.hit_ray_set(full, 1 << 14, seed=32)
    tri_d, uvt_d = device_renderer.trace_closest_np(rays)
    tri_h, uvt_h = host_renderer.trace_closest_np(rays)
    assert np.array_equal(tri_d, tri_h)
    assert np.array_equal(uvt_d.view(np.uint32), uvt_h.view(np.uint32))


def test_job_server_with_device_built_scenes(host_renderer, scene_factory):
    """The job server building its scenes' BVH8 on the device: jobs over two resident scenes give the
    frame renderer's (host-built BVH) images bit for bit."""
    names = ["cornell-all", "spheres-small"]
    srv = P.Server(0, pool_size=1 << 16, bvh_build=P.BVH_BUILD_DEVICE, hbm_budget_bytes=1 << 30, variant="det")
    try:
        ids = {n: srv.add_scene(scene_factory(n)) for n in names}
        jobs = [("cornell-all", 40, 30, 4, 6), ("spheres-small", 64, 40, 4, 12), ("spheres-small", 31, 29, 1, 10)]
        jids = []
        for name, w, h, spp, depth in jobs:
            cam = scenes.scene_camera(scene_factory(name), w, h)
            jids.append(srv.submit(ids[name], cam, w, h, spp, depth, True, keep_accumulation=True))
        for jid, (name, w, h, spp, depth) in zip(jids, jobs):
            st = srv.wait(jid, 300)
            assert st["state"] == "done", (name, st)
            fb, acc = srv.result(jid, accumulation=True)
            s = scene_factory(name)
            host_renderer.upload_scene(s)
            host_renderer.render_frame(scenes.scene_camera(s, w, h), w, h, spp, depth, True)
            assert np.array_equal(acc.view(np.uint32), host_renderer.accumulation().reshape(-1, 4).view(np.uint32))
            assert np.array_equal(fb, host_renderer.framebuffer().reshape(-1))
    finally:
        srv.close()
    with pytest.raises(P.GptError):
        P.Server(0, bvh_build=2)


@pytest.mark.parametrize("name", ["spheres-1m", "spheres-8m"])
def test_device_bvh_at_benchmark_scale(device_renderer, host_renderer, scene_factory, name):
    """The 1.31M-triangle headline scene and the 8.19M-triangle precision scene: valid trees whose hits
    on 2^20 rays equal the host BVH's."""
    s = scene_factory(name)
    device_renderer.upload_scene(s)
    t_device = device_renderer.upload_times()["bvh_build_s"]
    host_renderer.upload_scene(s)
    t_host = host_renderer.upload_times()["bvh_build_s"]
    check(device_renderer, s)
    rays = scenes.hit_ray_set(s, 1 << 20, seed=33)
    tri_d, uvt_d = device_renderer.trace_closest_np(rays)
    tri_h, uvt_h = host_renderer.trace_closest_np(rays)
    assert np.array_equal(tri_d, tri_h)
    hit = tri_d != INVALID
    assert np.array_equal(uvt_d[hit].view(np.uint32), uvt_h[hit].view(np.uint32))
    assert t_device < t_host
