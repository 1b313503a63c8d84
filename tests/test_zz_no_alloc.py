"""The allocation-free alias-table entry point against the scene-upload path.

gpt_build_alias_table_noalloc serves callers that cannot allocate device memory when they
build a light sampler; its working memory is a fixed array inside the library. This file is
collected last on purpose, so a run that stops at the first failure has already run every
other test. It must pass both alone in a fresh process and after the rest of the suite.
"""
import numpy as np
import pytest

import pathtracer
import scenes

pytestmark = pytest.mark.gpu


def light_weights(scene):
    """Area of every emissive triangle in input order, with the device's float operations
    (0.5 * length(cross(e1, e2)), LightSampler.cpp:16-19)."""
    models = scene.materials["model"][scene.material_ids]
    p = scene.positions[models == scenes.MODEL_EMISSIVE].astype(np.float32)
    e1 = p[:, 1] - p[:, 0]
    e2 = p[:, 2] - p[:, 0]
    cx = e1[:, 1] * e2[:, 2] - e1[:, 2] * e2[:, 1]
    cy = e1[:, 2] * e2[:, 0] - e1[:, 0] * e2[:, 2]
    cz = e1[:, 0] * e2[:, 1] - e1[:, 1] * e2[:, 0]
    d = (cx * cx + cy * cy) + cz * cz
    return (np.float32(0.5) * np.sqrt(d)).astype(np.float32)


def many_lights_scene(n, seed=5):
    """n small emissive triangles of varied size over a ground quad."""
    rng = np.random.default_rng(seed)
    base = scenes.cornell_box(1)
    c = rng.uniform(0.0, 10.0, (n, 3)).astype(np.float32)
    s = rng.uniform(0.01, 0.3, (n, 1)).astype(np.float32)
    p = np.stack([c, c + s * np.array([1, 0, 0], np.float32), c + s * np.array([0, 0, 1], np.float32)], 1)
    tris = np.concatenate([base.positions[:2], p]).astype(np.float32)
    nrm = np.zeros_like(tris)
    nrm[..., 1] = 1.0
    tan = np.zeros((tris.shape[0], 3, 4), np.float32)
    tan[..., 0] = 1.0
    tan[..., 3] = 1.0
    uv = np.zeros((tris.shape[0], 3, 2), np.float32)
    mats = np.concatenate([scenes.material(scenes.MODEL_DIFFUSE), scenes.material(scenes.MODEL_EMISSIVE, emission=(1, 1, 1))])
    mid = np.concatenate([np.zeros(2, np.uint32), np.ones(n, np.uint32)])
    return scenes.Scene(tris, nrm, tan, uv, mid, mats).contiguous()


def reference_table(scene):
    r = pathtracer.Renderer(0)
    try:
        r.upload_scene(scene)
        return r.alias_table()
    finally:
        r.close()


def build_noalloc(weights):
    import torch
    w = torch.from_numpy(weights).cuda()
    bins = torch.full((weights.size, 4), -1, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    rc = pathtracer.build_alias_table_noalloc(w, bins)
    assert rc == 0, pathtracer.lib().gpt_status_string(rc)
    torch.cuda.synchronize()
    return bins.cpu().numpy().view(np.uint32)


def test_noalloc_alias_table_matches_scene_upload_two_calls_in_a_row():
    a = scenes.config_scene("spheres-small")      # 8 lights
    b = many_lights_scene(20000)                   # 20,000 lights
    ref_a, ref_b = reference_table(a), reference_table(b)
    wa, wb = light_weights(a), light_weights(b)
    assert ref_a.shape == (wa.size, 4) and ref_b.shape == (wb.size, 4)
    got_b = build_noalloc(wb)        # first call: the larger table
    assert np.array_equal(got_b, ref_b)
    got_a = build_noalloc(wa)        # second call, right after: a smaller table over the same scratch
    assert np.array_equal(got_a, ref_a)


def test_noalloc_on_a_non_default_stream_and_with_no_lights():
    """The build is ordered on the caller's stream (here a side stream, not the default one), and a
    call with no lights succeeds without touching the output."""
    import ctypes

    import torch
    b = many_lights_scene(3000, seed=9)
    ref = reference_table(b)
    w = torch.from_numpy(light_weights(b)).cuda()
    bins = torch.full((w.shape[0], 4), -1, dtype=torch.int32, device="cuda")
    side = torch.cuda.Stream()
    torch.cuda.synchronize()
    with torch.cuda.stream(side):
        rc = pathtracer.build_alias_table_noalloc(w, bins)   # binds torch's current stream: the side stream
        done = bins.cpu()                                   # ordered after the build on the same stream
    assert rc == 0
    assert np.array_equal(done.numpy().view(np.uint32), ref)
    before = bins.clone()
    rc = pathtracer.lib().gpt_build_alias_table_noalloc(ctypes.c_void_p(w.data_ptr()), 0, ctypes.c_void_p(bins.data_ptr()),
                                                        ctypes.c_void_p(side.cuda_stream))
    torch.cuda.synchronize()
    assert rc == 0
    assert torch.equal(bins, before)


def test_noalloc_rejects_tables_above_its_limit():
    import torch
    n = 65537  # GPT_NOALLOC_MAX_LIGHTS + 1
    w = torch.ones(n, dtype=torch.float32, device="cuda")
    bins = torch.zeros((n, 4), dtype=torch.int32, device="cuda")
    assert pathtracer.build_alias_table_noalloc(w, bins) == 6  # GPT_ERR_CAPACITY
