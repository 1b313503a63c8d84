"""The product against the reference itself: the reference's own kernel sources (Intersect.cu,
PathGeneration.cu, MaterialEval.cu, Iteration.cu, HostBvh.cpp) compiled for sm_100a into
oracle/_ref/ and driven through their launchers (oracle/ref_harness), GPU against GPU.

* The product build (libgpt_b200.so) computes as the reference's build does (multiply-add
  contraction, CUDA's sinf/cosf/powf/rsqrtf), so against the reference built with its own flags:
  hit triangle ids and (u, v, t) bit-exact on 2^20 rays except at exact ties (two triangles at the
  bit-identical t: the reference keeps the first its DFS visits, the product the smaller input
  index; such rays are counted), per-iteration queue counts bit-exact, and every path's radiance
  within 1e-4 relative at spp = 1, with constant and with image-textured materials.
* The oracle's pin: against the reference built with -fmad=false (the oracle's operator-by-operator
  rounding) the oracle's hits are bit-exact except exact ties; its deterministic transcendentals
  differ from CUDA's in the last bits, so its frames agree with the reference's statistically, with
  the bounds stated below.
The materials handed to the product and the oracle are the texel values the reference's own sRGB
textures return on the device (hardware decode), read back from the reference harness.
"""
import numpy as np
import pytest

import oracle
import scenes

ref_harness = pytest.importorskip("ref_harness")
pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not ref_harness.available(), reason="oracle/_ref not built (needs the reference sources)")]

INVALID = 0xFFFFFFFF


def with_materials(s, mats):
    return scenes.Scene(s.positions, s.normals, s.tangents, s.uvs, s.material_ids, mats, s.name, s.camera).contiguous()


_cache = {}


class _LazyOracle:
    """The oracle's scene of a decoded scene, built on first use (its host BVH build is the slow
    part at millions of triangles, and the product-against-reference tests do not need it)."""

    def __init__(self, scene):
        self.scene, self.o = scene, None

    def __getattr__(self, attr):
        if self.o is None:
            self.o = oracle.OracleScene(self.scene)
        return getattr(self.o, attr)


def pair(name, fma):
    key = (name, fma)
    if key not in _cache:
        s = scenes.config_scene(name)
        R = ref_harness.RefScene(s, fma=fma)
        decoded = with_materials(s, R.decoded_materials())
        _cache[key] = (s, R, decoded, _LazyOracle(decoded))
    return _cache[key]


def hits_against_reference(tg, ug, tr, ur):
    """Counts of (id mismatches at an exact tie, other mismatches, (u, v, t) bit mismatches on equal ids)."""
    diff = tg != tr
    tie = diff & (tg != INVALID) & (tr != INVALID) & (ug[:, 2].view(np.uint32) == ur[:, 2].view(np.uint32))
    same_hit = ~diff & (tr != INVALID)
    uvt = same_hit & np.any(ug.view(np.uint32) != ur.view(np.uint32), axis=1)
    return int(tie.sum()), int((diff & ~tie).sum()), int(uvt.sum())


@pytest.mark.parametrize("name", ["cornell", "cornell-all", "spheres-small", "spheres-200k", "spheres-1m", "spheres-8m"])
def test_product_hits_bit_exact_against_reference_build(gpu_renderer_product, name):
    s, R, decoded, _ = pair(name, True)
    gpu_renderer_product.upload_scene(decoded)
    rays = scenes.hit_ray_set(s, 1 << 20, seed=11)
    tr, ur = R.trace_closest(rays)
    tg, ug = gpu_renderer_product.trace_closest_np(rays)
    ties, other, uvt = hits_against_reference(tg, ug, tr, ur)
    assert other == 0 and uvt == 0, (ties, other, uvt)
    assert ties <= 1e-3 * rays.shape[0]


@pytest.mark.parametrize("name,w,h", [("cornell-all", 256, 256), ("spheres-small", 192, 128), ("spheres-1m", 240, 135),
                                      ("spheres-8m", 256, 144)])
@pytest.mark.parametrize("nee", [False, True])
def test_product_frames_against_reference_build(gpu_renderer_product, name, w, h, nee):
    """spp = 1 (one path per pixel, so the reference's float-atomic pixel sum is that path's
    radiance): identical per-iteration queue counts and every path within 1e-4 relative."""
    s, R, decoded, _ = pair(name, True)
    r = gpu_renderer_product
    r.upload_scene(decoded)
    cam = scenes.scene_camera(s, w, h)
    rr = R.render(cam, w, h, 1, 10, nee)
    st = r.render_frame(cam, w, h, 1, 10, nee, pool_size=1 << 20)
    assert st["iterations"] == rr["iterations"]
    assert np.array_equal(r.queue_log(), rr["queue_log"][:len(r.queue_log())])
    a = r.sample_radiance().astype(np.float64)
    b = rr["accumulation"][:, :3].astype(np.float64)
    rel = np.abs(a - b) / np.maximum(np.abs(b), 1e-6)
    assert np.all(rel <= 1e-4), (int(np.sum(np.any(rel > 1e-4, axis=1))), float(rel.max()))


def test_reference_texture_decode_is_close_to_the_srgb_formula():
    s, R, decoded, _ = pair("cornell-all", True)
    for field in ("color", "specular", "shininess", "rma", "emission", "normal"):
        diff = np.abs(decoded.materials[field].astype(np.float64) - s.materials[field].astype(np.float64))
        assert diff.max() <= 2.5e-3, field


@pytest.mark.parametrize("name", ["cornell", "spheres-200k"])
def test_hits_bit_exact_against_reference_kernels_without_fma(name):
    s, R, _, O = pair(name, False)
    rays = scenes.hit_ray_set(s, 1 << 20, seed=11)
    tr, ur = R.trace_closest(rays)
    to, uo = O.trace_closest(rays)
    same = tr == to
    # where the ids differ, both found a hit at the bit-identical distance (an exact tie)
    diff = ~same
    assert np.all(tr[diff] != INVALID) and np.all(to[diff] != INVALID)
    assert np.array_equal(ur[diff, 2].view(np.uint32), uo[diff, 2].view(np.uint32))
    assert diff.mean() < 1e-3
    hit = same & (to != INVALID)
    assert np.array_equal(ur[hit].view(np.uint32), uo[hit].view(np.uint32))


@pytest.mark.parametrize("name", ["cornell", "spheres-200k"])
def test_hits_against_reference_build(name):
    s, R, _, O = pair(name, True)
    rays = scenes.hit_ray_set(s, 1 << 20, seed=11)
    tr, ur = R.trace_closest(rays)
    to, uo = O.trace_closest(rays)
    assert np.array_equal(tr != INVALID, to != INVALID)
    hit = to != INVALID
    rel = np.abs(ur[hit, 2] - uo[hit, 2]) / np.maximum(uo[hit, 2], 1e-3)
    # FMA contraction moves the Moller-Trumbore t by a few ulps; grazing rays (cancellation in
    # the dot products) move more, so the bound is on the distribution
    assert np.mean(rel <= 4e-6) >= 0.999
    assert np.median(rel) == 0.0
    # ids differ only at near-ties (coplanar or abutting triangles)
    assert (tr != to).mean() < 5e-3


@pytest.mark.parametrize("fma", [False, True])
@pytest.mark.parametrize("nee", [False, True])
def test_per_path_radiance_against_reference_kernels(fma, nee):
    s, R, decoded, O = pair("cornell-all", fma)
    W = H = 256
    cam = scenes.scene_camera(s, W, H)
    rr = R.render(cam, W, H, 1, 10, nee)
    oo = O.render(cam, W, H, 1, 10, nee, accumulation=0)
    a, b = rr["accumulation"][:, :3].astype(np.float64), oo["sample_radiance"].astype(np.float64)
    rel = np.abs(a - b) / np.maximum(np.abs(b), 1e-6)
    within = np.all(rel <= 1e-4, axis=1).mean()
    # spp = 1: the reference's pixel accumulation is one path's radiance
    assert within >= (0.9999 if not nee else 0.998)
    assert np.all(np.abs(a.mean(0) - b.mean(0)) <= 1e-5 * np.abs(b.mean(0)) + 1e-7)
    n = min(len(rr["queue_log"]), len(oo["queue_log"]))
    assert rr["iterations"] == oo["iterations"]
    assert np.max(np.abs(rr["queue_log"][:n].astype(np.int64) - oo["queue_log"][:n].astype(np.int64))) <= 4


def test_converged_image_against_reference_kernels():
    s, R, decoded, O = pair("cornell", True)
    W = H = 64
    cam = scenes.scene_camera(s, W, H)
    rr = R.render(cam, W, H, 256, 8, True)
    oo = O.render(cam, W, H, 256, 8, True, accumulation=2)
    a = rr["accumulation"][:, :3].astype(np.float64) / 256
    b = oo["accumulation"][:, :3].astype(np.float64) / 256
    rmse = float(np.sqrt(np.mean((a - b) ** 2)))
    assert rmse <= 1e-3 * float(np.sqrt(np.mean(b ** 2)))


@pytest.mark.parametrize("nee", [False, True])
def test_textured_materials_against_reference_kernels(gpu_renderer, nee):
    """Image textures in every slot (albedo, normal, shininess, RMA, specular, emission maps): the
    product and the reference's own kernels sample them through the same texture hardware with the
    same descriptors, so they are compared GPU against GPU (reference built with -fmad=false)."""
    s = scenes.config_scene("cornell-textured")
    R = ref_harness.RefScene(s, fma=False)
    decoded = with_materials(s, R.decoded_materials())
    decoded.textures, decoded.material_textures = s.textures, s.material_textures
    gpu_renderer.upload_scene(decoded)
    W = H = 192
    cam = scenes.scene_camera(s, W, H)
    gpu_renderer.render_frame(cam, W, H, 1, 10, nee)
    a = gpu_renderer.sample_radiance().astype(np.float64)
    rr = R.render(cam, W, H, 1, 10, nee)
    R.close()
    b = rr["accumulation"][:, :3].astype(np.float64)
    rel = np.abs(a - b) / np.maximum(np.abs(b), 1e-6)
    within = np.all(rel <= 1e-4, axis=1).mean()
    assert within >= (0.999 if not nee else 0.995)
    assert np.all(np.abs(a.mean(0) - b.mean(0)) <= 1e-4 * np.abs(b.mean(0)) + 1e-6)
    assert np.all(np.isfinite(a)) and a.mean() > 0


@pytest.mark.parametrize("nee", [False, True])
def test_product_textured_frames_against_reference_build(gpu_renderer_product, nee):
    """Image textures in every slot, the product build against the reference built with its own
    flags: identical per-iteration queue counts and every path within 1e-4 relative at spp = 1."""
    s = scenes.config_scene("cornell-textured")
    R = ref_harness.RefScene(s, fma=True)
    decoded = with_materials(s, R.decoded_materials())
    decoded.textures, decoded.material_textures = s.textures, s.material_textures
    r = gpu_renderer_product
    r.upload_scene(decoded)
    W = H = 192
    cam = scenes.scene_camera(s, W, H)
    st = r.render_frame(cam, W, H, 1, 10, nee, pool_size=1 << 20)
    rr = R.render(cam, W, H, 1, 10, nee)
    R.close()
    assert st["iterations"] == rr["iterations"]
    assert np.array_equal(r.queue_log(), rr["queue_log"][:len(r.queue_log())])
    a = r.sample_radiance().astype(np.float64)
    b = rr["accumulation"][:, :3].astype(np.float64)
    rel = np.abs(a - b) / np.maximum(np.abs(b), 1e-6)
    assert np.all(rel <= 1e-4), (int(np.sum(np.any(rel > 1e-4, axis=1))), float(rel.max()))
    assert a.mean() > 0
