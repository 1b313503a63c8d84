"""The oracle (CPU restatement of the reference renderer) on its own: determinism,
invariants of the wavefront schedule, the alias table, the deterministic math and
the golden vectors captured from the device (tests/golden/)."""
import json
import math
import os

import numpy as np
import pytest

import oracle
import scenes

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def test_deterministic_math_accuracy():
    x = np.linspace(0.0, 2 * math.pi, 100001, dtype=np.float32)
    s, c = oracle.sincos(x)
    ref_s = np.sin(x.astype(np.float64))
    ref_c = np.cos(x.astype(np.float64))
    ulp = np.spacing(np.abs(np.float32(1.0)))
    assert np.max(np.abs(s - ref_s)) <= ulp
    assert np.max(np.abs(c - ref_c)) <= ulp
    xs = np.random.default_rng(0).random(20000, dtype=np.float32)
    ys = np.random.default_rng(1).uniform(0.0, 1000.0, 20000).astype(np.float32)
    p = oracle.powf(xs, ys)
    ref = np.power(xs.astype(np.float64), ys.astype(np.float64))
    rel = np.abs(p - ref) / np.maximum(ref, 1e-30)
    assert np.max(rel[ref > 1e-30]) < 2e-7
    assert oracle.powf(np.array([0.0, 1.0], np.float32), np.array([2.0, 7.0], np.float32)).tolist() == [0.0, 1.0]


def test_philox_stream_positions_are_consistent():
    words, uni = oracle.philox_words(17, 0, 64)
    w2, _ = oracle.philox_words(17, 13, 20)
    assert np.array_equal(words[13:33], w2)
    assert np.all(uni > 0.0) and np.all(uni <= 1.0)
    other, _ = oracle.philox_words(18, 0, 64)
    assert not np.array_equal(words, other)


def test_philox_matches_device_golden():
    path = os.path.join(GOLDEN, "philox_curand.json")
    if not os.path.exists(path):
        pytest.skip("device-captured Philox golden vectors not generated yet")
    g = json.load(open(path))
    for rec in g["records"]:
        words, uni = oracle.philox_words(rec["subsequence"], 0, 8)
        assert words.tolist() == rec["words"]
        _, u = oracle.philox_words(rec["subsequence"], 0, 17)
        sched = [float(v) for v in rec["schedule"]]
        # draw schedule uniform4, uniform4, uniform, uniform4, uniform = stream positions 0..13
        assert np.array_equal(np.array(sched, np.float32), u[:14])


def test_alias_table_reference_semantics():
    w = np.array([1.0, 2.0, 3.0, 4.0], dtype=np.float32)
    bins = oracle.alias_build(w)
    # outcome probability of each index from the table
    n = len(w)
    prob = np.zeros(n)
    for i, b in enumerate(bins):
        prob[i] += b["q"] / n
        if b["alias"] != 0xFFFFFFFF:
            prob[b["alias"]] += (1 - b["q"]) / n
    assert np.allclose(prob, w / w.sum(), atol=1e-6)
    u = np.random.default_rng(0).random(200000, dtype=np.float32)
    idx, pmf = oracle.alias_sample(bins, u)
    freq = np.bincount(idx, minlength=n) / len(u)
    assert np.allclose(freq, w / w.sum(), atol=5e-3)
    assert np.allclose(pmf, (w / w.sum())[idx], atol=1e-6)


def test_reference_bvh_structure():
    s = scenes.cornell_box(1)
    o = oracle.OracleScene(s)
    nodes, order, depth = o.bvh()
    assert sorted(order.tolist()) == list(range(36))
    leaves = nodes[(nodes["left"] == 0xFFFFFFFF)]
    assert leaves["count"].sum() == 36
    assert depth <= 11  # ceil(2 log2 36)


def test_closest_hit_against_brute_force():
    s = scenes.cornell_all_models(1)
    o = oracle.OracleScene(s)
    rays = scenes.hit_ray_set(s, 2000, seed=5)
    tri, uvt = o.trace_closest(rays, threads=1)
    # brute-force Moller-Trumbore in float64 for the hit distance
    p = s.positions.astype(np.float64)
    v0, e1, e2 = p[:, 0], p[:, 1] - p[:, 0], p[:, 2] - p[:, 0]
    for i in range(0, 2000, 37):
        o_, d_ = rays[i, :3].astype(np.float64), rays[i, 3:6].astype(np.float64)
        pv = np.cross(d_, e2)
        det = (e1 * pv).sum(1)
        ok = np.abs(det) > 1e-7
        inv = np.where(ok, 1.0 / np.where(ok, det, 1.0), 0.0)
        sv = o_ - v0
        u = (sv * pv).sum(1) * inv
        q = np.cross(sv, e1)
        v = (d_ * q).sum(1) * inv
        t = (e2 * q).sum(1) * inv
        valid = ok & (u >= 0) & (u <= 1) & (v >= 0) & (u + v <= 1) & (t >= 1e-4)
        if valid.any():
            best = np.min(t[valid])
            assert tri[i] != 0xFFFFFFFF
            assert abs(uvt[i, 2] - best) <= 1e-5 * max(1.0, best)
        else:
            assert tri[i] == 0xFFFFFFFF


def test_render_is_thread_count_independent():
    s = scenes.cornell_all_models(1)
    o = oracle.OracleScene(s)
    cam = scenes.scene_camera(s, 32, 32)
    a = o.render(cam, 32, 32, 4, 8, True, pool_size=1000, threads=1)
    b = o.render(cam, 32, 32, 4, 8, True, pool_size=1000, threads=8)
    assert np.array_equal(a["sample_radiance"], b["sample_radiance"])
    assert np.array_equal(a["queue_log"], b["queue_log"])
    assert np.array_equal(a["framebuffer"], b["framebuffer"])


def test_wavefront_schedule_invariants():
    s = scenes.cornell_box(1)
    o = oracle.OracleScene(s)
    cam = scenes.scene_camera(s, 32, 32)
    pool = 1500
    r = o.render(cam, 32, 32, 9, 8, True, pool_size=pool)
    log = r["queue_log"].astype(np.int64)
    total = 9 * 32 * 32
    assert log[0, 0] == min(total, pool)
    launched = log[0, 0]
    for k in range(len(log)):
        rays, mats, shadow, regen = log[k, 0], log[k, 1:7], log[k, 7], log[k, 8]
        assert mats.sum() <= rays and regen >= rays - mats.sum() and shadow <= mats.sum()
        regenerate = min(regen, total - launched)
        if k + 1 < len(log):
            assert log[k + 1, 0] == rays - regen + regenerate
        launched += regenerate
    assert launched == total
    assert r["iterations"] == len(log)


def test_fp64_and_kahan_accumulation_agree():
    s = scenes.cornell_box(1)
    o = oracle.OracleScene(s)
    cam = scenes.scene_camera(s, 16, 16)
    a = o.render(cam, 16, 16, 64, 8, True, accumulation=1)
    b = o.render(cam, 16, 16, 64, 8, True, accumulation=2)
    assert np.array_equal(a["sample_radiance"], b["sample_radiance"])
    rel = np.abs(a["accumulation"] - b["accumulation"]) / np.maximum(np.abs(b["accumulation"]), 1e-6)
    assert rel.max() < 1e-6


def test_render_emissive_only_sees_light():
    s = scenes.cornell_box(1)
    o = oracle.OracleScene(s)
    cam = scenes.scene_camera(s, 24, 24)
    r = o.render(cam, 24, 24, 1, 1, False)  # depth 1, no NEE: only camera-ray emitter hits count
    rad = r["sample_radiance"]
    lit = np.any(rad > 0, axis=1)
    assert lit.sum() > 0
    assert np.allclose(rad[lit], [17.0, 12.0, 4.0])
