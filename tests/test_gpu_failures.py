"""Failure paths, tested without faulting the GPU.

* The device loop's bound: a frame whose iteration cap runs out while paths are in flight ends
  promptly with GPT_ERR_DEVICE_FAULT, in the graph loop and in the host loop, and the next frame is
  correct.
* The traversal stack's bound: a stack shallower than the BVH8 overflows on some rays; the kernel
  records it, stops those rays (no access outside the stack) and the frame ends with
  GPT_ERR_DEVICE_FAULT; the next frame is correct.
* Host allocation failures (gpt_inject_allocation_failure, failing before cudaMalloc is called):
  scene upload, frame buffers and the job server fail with GPT_ERR_OUT_OF_MEMORY at every
  allocation and leave the renderer or server usable.
"""
import time

import numpy as np
import pytest

import pathtracer
import scenes

pytestmark = pytest.mark.gpu

DEVICE_FAULT, OUT_OF_MEMORY = 8, 3


def render_matches_oracle(r, o, s, w=32, h=32, spp=4, depth=8):
    cam = scenes.scene_camera(s, w, h)
    st = r.render_frame(cam, w, h, spp, depth, True)
    ref = o.render(cam, w, h, spp, depth, True)
    assert st["iterations"] == ref["iterations"]
    assert np.array_equal(r.queue_log(), ref["queue_log"])
    assert np.array_equal(r.sample_radiance().view(np.uint32), ref["sample_radiance"].view(np.uint32))


@pytest.mark.parametrize("loop", [pathtracer.LOOP_GRAPH, pathtracer.LOOP_HOST])
def test_iteration_cap_ends_the_frame_with_a_device_fault(gpu_renderer, scene_factory, oracle_scene, loop):
    s = scene_factory("cornell")
    gpu_renderer.upload_scene(s)
    cam = scenes.scene_camera(s, 64, 64)
    t0 = time.perf_counter()
    with pytest.raises(pathtracer.GptError) as e:
        gpu_renderer.render_frame(cam, 64, 64, 16, 8, True, pool_size=4096, loop_mode=loop, max_iterations=3)
    assert e.value.code == DEVICE_FAULT
    assert time.perf_counter() - t0 < 10.0
    # a cap above what the frame needs changes nothing
    st = gpu_renderer.render_frame(cam, 64, 64, 16, 8, True, pool_size=4096, loop_mode=loop, max_iterations=100000)
    assert st["samples"] == 64 * 64 * 16
    render_matches_oracle(gpu_renderer, oracle_scene("cornell"), s)


@pytest.mark.parametrize("loop", [pathtracer.LOOP_GRAPH, pathtracer.LOOP_HOST])
def test_traversal_stack_overflow_is_reported(gpu_renderer, scene_factory, oracle_scene, loop):
    s = scene_factory("spheres-200k")
    gpu_renderer.upload_scene(s)
    depth = gpu_renderer.scene_info()["depth"]
    assert depth > 2
    cam = scenes.scene_camera(s, 96, 64)
    # a ray descending below the root with more than one child group pending needs two entries
    with pytest.raises(pathtracer.GptError) as e:
        gpu_renderer.render_frame(cam, 96, 64, 4, 8, True, loop_mode=loop, trace_stack=1)
    assert e.value.code == DEVICE_FAULT
    # the tree's own depth (the default, or an explicit stack at least that deep) renders normally
    a = gpu_renderer.render_frame(cam, 96, 64, 4, 8, True, loop_mode=loop)
    rad_a = gpu_renderer.sample_radiance()
    b = gpu_renderer.render_frame(cam, 96, 64, 4, 8, True, loop_mode=loop, trace_stack=64)
    assert a["iterations"] == b["iterations"]
    assert np.array_equal(rad_a.view(np.uint32), gpu_renderer.sample_radiance().view(np.uint32))
    with pytest.raises(pathtracer.GptError):
        gpu_renderer.render_frame(cam, 8, 8, 1, 2, True, trace_stack=65)
    small = scene_factory("cornell")
    gpu_renderer.upload_scene(small)
    render_matches_oracle(gpu_renderer, oracle_scene("cornell"), small)


def test_allocation_failures_during_scene_upload_leave_the_renderer_usable(gpu_renderer, scene_factory, oracle_scene):
    L = pathtracer.lib("det")
    s = scene_factory("cornell-all")
    o = oracle_scene("cornell-all")
    gpu_renderer.upload_scene(s)
    failures = 0
    try:
        for k in range(1, 64):
            L.gpt_inject_allocation_failure(k)
            try:
                gpu_renderer.upload_scene(s)
            except pathtracer.GptError as e:
                assert e.code == OUT_OF_MEMORY
                failures += 1
                # the previous scene stays in place and renders
                render_matches_oracle(gpu_renderer, o, s)
                continue
            break
    finally:
        L.gpt_inject_allocation_failure(0)
    assert failures >= 10  # every device allocation of the upload was made to fail once
    gpu_renderer.upload_scene(s)
    render_matches_oracle(gpu_renderer, o, s)


def test_allocation_failures_of_frame_buffers_and_server(gpu_renderer, scene_factory, oracle_scene):
    L = pathtracer.lib("det")
    s = scene_factory("cornell")
    o = oracle_scene("cornell")
    gpu_renderer.upload_scene(s)
    cam = scenes.scene_camera(s, 200, 120)
    try:
        # a larger frame than any before (24.6M samples): its per-sample buffer is allocated anew and fails
        L.gpt_inject_allocation_failure(1)
        with pytest.raises(pathtracer.GptError) as e:
            gpu_renderer.render_frame(cam, 200, 120, 1024, 8, True)
        assert e.value.code == OUT_OF_MEMORY
        L.gpt_inject_allocation_failure(1)
        with pytest.raises(pathtracer.GptError) as e:
            gpu_renderer.init_rendering_buffers(1024, 1024)
        assert e.value.code == OUT_OF_MEMORY
    finally:
        L.gpt_inject_allocation_failure(0)
    render_matches_oracle(gpu_renderer, o, s)
    # job server: creation and scene registration fail cleanly, then work
    for k in (1, 3, 7):
        L.gpt_inject_allocation_failure(k)
        try:
            with pytest.raises(pathtracer.GptError) as e:
                pathtracer.Server(0, pool_size=1 << 16, hbm_budget_bytes=1 << 28, variant="det")
            assert e.value.code == OUT_OF_MEMORY
        finally:
            L.gpt_inject_allocation_failure(0)
    srv = pathtracer.Server(0, pool_size=1 << 16, hbm_budget_bytes=1 << 28, variant="det")
    try:
        L.gpt_inject_allocation_failure(1)
        try:
            with pytest.raises(pathtracer.GptError) as e:
                srv.add_scene(s)
            assert e.value.code == OUT_OF_MEMORY
        finally:
            L.gpt_inject_allocation_failure(0)
        sid = srv.add_scene(s)
        cam2 = scenes.scene_camera(s, 32, 32)
        jid = srv.submit(sid, cam2, 32, 32, 4, 8, True)
        st = srv.wait(jid, 60.0)
        assert st["state"] == "done"
        img, _ = srv.result(jid)
        gpu_renderer.render_frame(cam2, 32, 32, 4, 8, True)
        assert np.array_equal(img, gpu_renderer.framebuffer())
        srv.release(jid)
    finally:
        srv.close()
