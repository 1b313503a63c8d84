"""The two production modes the reference does not have: the PCG32 RNG policy and power-weighted
light selection with its parallel alias-table build.

CPU: the oracle's PCG32 reproduces the generator's published sequence, its jump-ahead continues the
stream, and the power-weighted table encodes the target distribution (a size-independent property).
GPU: the deterministic build against the oracle, bit for bit (tables, queue counts, per-path
radiance); the product build's job server against its frame renderer; and power sampling lowering
the error of a frame at equal paths on a scene whose lights span three decades of power.
"""
import numpy as np
import pytest

import oracle
import scenes

INVALID = 0xFFFFFFFF


# ---------------------------------------------------------------------------- CPU

def test_pcg32_reproduces_the_published_sequence():
    # pcg32_srandom_r(42, 54) followed by six draws, the generator's demonstration output
    # (O'Neill, pcg-c-basic); the oracle's seeding and output function are those of the paper
    got = oracle.pcg_seeded_words(42, 54, 6)
    assert [int(x) for x in got] == [0xA15C02B7, 0x7B47F409, 0xBA1D3330, 0x83D2F293, 0xBFA4784B, 0xCBED606E]


def test_pcg32_jump_ahead_continues_the_stream():
    for key in (0, 1, 12345, 2**40 + 3):
        words, uni = oracle.pcg_words(key, 0, 96)
        for pos in (1, 4, 5, 17, 63, 90):
            w2, u2 = oracle.pcg_words(key, pos, 96 - pos)
            assert np.array_equal(words[pos:], w2), (key, pos)
            assert np.array_equal(uni[pos:].view(np.uint32), u2.view(np.uint32))
        assert np.all(uni > 0.0) and np.all(uni <= 1.0)
    # distinct keys give distinct streams
    a, _ = oracle.pcg_words(7, 0, 16)
    b, _ = oracle.pcg_words(8, 0, 16)
    assert not np.array_equal(a, b)


@pytest.mark.parametrize("n", [1, 2, 3, 7, 64, 1023, 1025, 40000])
def test_power_alias_table_encodes_the_target_distribution(n):
    rng = np.random.default_rng(n)
    area = rng.uniform(0.01, 1.0, n)
    power = area * 10.0 ** rng.uniform(0.0, 3.0, n)
    if n > 10:
        power[::7] = 0.0                      # black emitters: never picked
    bins = oracle.power_alias_build(power, area)
    target = power / power.sum()
    implied = oracle.alias_implied_pmf(bins)
    assert np.all((bins["q"] >= 0.0) & (bins["q"] <= 1.0))
    assert np.array_equal(bins["value"], np.arange(n, dtype=np.uint32))
    valid = bins["alias"] != INVALID
    assert np.all(bins["alias"][valid] < n)
    # every outcome's probability is the target's to float precision
    assert np.all(np.abs(implied - target) <= 2e-7 * target + 1e-12)
    assert np.all(np.abs(bins["p"].astype(np.float64) - target) <= 1e-7 * target + 1e-30)
    assert np.all(implied[power == 0.0] <= 1e-12)


def test_power_alias_table_falls_back_to_area_weights_without_power():
    area = np.random.default_rng(3).uniform(0.1, 1.0, 300)
    bins = oracle.power_alias_build(np.zeros(300), area)
    assert np.all(np.abs(oracle.alias_implied_pmf(bins) - area / area.sum()) <= 2e-7 * area / area.sum())


def test_device_order_scan_is_an_exclusive_prefix_sum():
    x = np.random.default_rng(4).uniform(0.0, 1.0, 70000)
    got = oracle.device_order_scan(x)
    ref = np.concatenate([[0.0], np.cumsum(x)[:-1]])
    assert got[0] == 0.0
    assert np.all(np.abs(got - ref) <= 1e-12 * np.maximum(ref, 1.0))


# ---------------------------------------------------------------------------- GPU

def many_lights_scene(n, seed=5):
    """n emissive triangles of varied size and power over a ground quad."""
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
    k = 16
    emit = [scenes.material(scenes.MODEL_EMISSIVE, emission=tuple(float(10.0 ** e) * np.array([1.0, 0.8, 0.6])))
            for e in np.linspace(-1.0, 2.0, k)]
    mats = np.concatenate([scenes.material(scenes.MODEL_DIFFUSE)] + emit)
    mid = np.concatenate([np.zeros(2, np.uint32), 1 + (np.arange(n) % k).astype(np.uint32)])
    return scenes.Scene(tris, nrm, tan, uv, mid, mats).contiguous()


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["spheres-small", "spheres-200k", "many-20000"])
def test_power_alias_table_bit_exact_with_oracle(gpu_renderer, scene_factory, name):
    s = many_lights_scene(20000) if name == "many-20000" else scene_factory(name)
    o = oracle.OracleScene(s)
    gpu_renderer.upload_scene(s)
    got = gpu_renderer.alias_table(power=True)
    ref = o.alias_table(power=True).view(np.uint32).reshape(-1, 4)
    assert got.shape == ref.shape and got.shape[0] > 1
    assert np.array_equal(got, ref)
    # and the area table is untouched by the power build
    assert np.array_equal(gpu_renderer.alias_table(), o.alias_table().view(np.uint32).reshape(-1, 4))
    implied = oracle.alias_implied_pmf(got.view(oracle.BIN_DTYPE).reshape(-1))
    p = got[:, 1].view(np.float32).astype(np.float64)
    assert np.all(np.abs(implied - p) <= 2e-7 * p + 1e-12)


def assert_mode_parity(r, o, cam, w, h, spp, depth, nee, pool, rng_policy, light_sampling):
    st = r.render_frame(cam, w, h, spp, depth, nee, pool_size=pool, rng_policy=rng_policy, light_sampling=light_sampling)
    ref = o.render(cam, w, h, spp, depth, nee, pool_size=pool, rng_policy=rng_policy, light_sampling=light_sampling)
    assert st["iterations"] == ref["iterations"]
    assert np.array_equal(r.queue_log(), ref["queue_log"])
    assert np.array_equal(r.sample_radiance().view(np.uint32), ref["sample_radiance"].view(np.uint32))
    return r.sample_radiance()


@pytest.mark.gpu
@pytest.mark.parametrize("rng_policy,light_sampling", [(1, 0), (0, 1), (1, 1)])
def test_production_modes_bit_exact_with_oracle(gpu_renderer, scene_factory, oracle_scene, rng_policy, light_sampling):
    s = scene_factory("spheres-small")
    o = oracle_scene("spheres-small")
    gpu_renderer.upload_scene(s)
    cam = scenes.scene_camera(s, 96, 64)
    rad = assert_mode_parity(gpu_renderer, o, cam, 96, 64, 4, 12, True, 3000, rng_policy, light_sampling)
    assert np.all(np.isfinite(rad)) and rad.mean() > 0
    s2 = scene_factory("cornell-all")
    gpu_renderer.upload_scene(s2)
    cam2 = scenes.scene_camera(s2, 64, 64)
    assert_mode_parity(gpu_renderer, oracle_scene("cornell-all"), cam2, 64, 64, 16, 10, True, 1 << 20, rng_policy, light_sampling)


@pytest.mark.gpu
def test_pcg32_streams_differ_from_philox_but_agree_in_the_mean(gpu_renderer_product, scene_factory):
    s = scene_factory("cornell")
    r = gpu_renderer_product
    r.upload_scene(s)
    cam = scenes.scene_camera(s, 64, 64)
    r.render_frame(cam, 64, 64, 64, 8, True, rng_policy=0)
    a = r.accumulation()[:, :3].astype(np.float64) / 64
    r.render_frame(cam, 64, 64, 64, 8, True, rng_policy=1)
    b = r.accumulation()[:, :3].astype(np.float64) / 64
    assert not np.array_equal(a, b)
    assert abs(a.mean() - b.mean()) <= 0.02 * a.mean()


@pytest.mark.gpu
def test_unknown_modes_are_rejected(gpu_renderer_product, scene_factory):
    import pathtracer
    s = scene_factory("cornell")
    gpu_renderer_product.upload_scene(s)
    cam = scenes.scene_camera(s, 8, 8)
    for kw in (dict(rng_policy=2), dict(light_sampling=2)):
        with pytest.raises(pathtracer.GptError) as e:
            gpu_renderer_product.render_frame(cam, 8, 8, 1, 2, True, **kw)
        assert e.value.code == 1


@pytest.mark.gpu
def test_power_sampling_lowers_the_error_at_equal_paths(gpu_renderer_product, scene_factory):
    """spheres-small has emitters whose power spans three decades: picking them by power puts the
    shadow rays where the light is, so at equal spp the image is closer to a converged one. Each mode
    is compared with its own 1,024-spp image (the shadow clamp of Intersect.cu:178 makes the two
    converged images differ slightly)."""
    r = gpu_renderer_product
    s = scene_factory("spheres-small")
    r.upload_scene(s)
    W, H = 96, 64
    cam = scenes.scene_camera(s, W, H)
    rmse = {}
    for mode in (0, 1):
        r.render_frame(cam, W, H, 1024, 8, True, light_sampling=mode, rng_offset=1 << 40)
        ref = r.accumulation_fp64() / 1024
        errs = []
        for k in range(4):
            r.render_frame(cam, W, H, 16, 8, True, light_sampling=mode, rng_offset=k * W * H * 16)
            img = r.accumulation()[:, :3].astype(np.float64) / 16
            errs.append(np.sqrt(np.mean((img - ref) ** 2)))
        rmse[mode] = float(np.mean(errs))
    assert rmse[1] < rmse[0], rmse
