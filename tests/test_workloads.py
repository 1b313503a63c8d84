"""Seeded job mixes of the batched and served workloads (host only)."""
import math

import numpy as np

import workloads


def test_batched_mix_is_seeded_and_in_range():
    a, b = workloads.batched_jobs(), workloads.batched_jobs()
    assert len(a) == 64
    assert [(j.scene, j.width, j.height, j.spp, j.depth) for j in a] == [(j.scene, j.width, j.height, j.spp, j.depth) for j in b]
    assert all(np.array_equal(x.camera, y.camera) for x, y in zip(a, b))
    for j in a:
        assert j.scene in workloads.BATCH_SCENES
        assert 256 <= j.width <= 1920 and 256 <= j.height <= 1080
        assert j.spp in (1, 4, 16, 64) and 8 <= j.depth <= 12
        assert j.paths == j.width * j.height * j.spp
        assert j.camera.shape == (12,) and np.all(np.isfinite(j.camera))
    assert len({j.scene for j in a}) == len(workloads.BATCH_SCENES)
    assert len({j.spp for j in a}) == 4


def test_orbit_camera_looks_at_the_field_centre():
    rng = np.random.default_rng(5)
    for _ in range(20):
        cam = workloads.orbit_camera(rng, 320, 200)
        origin, llc, hor, ver = cam[0:3], cam[3:6], cam[6:9], cam[9:12]
        centre_dir = llc + 0.5 * hor + 0.5 * ver - origin
        to_centre = np.array([10.0, 5.0, 10.0]) - origin
        cosang = centre_dir @ to_centre / np.linalg.norm(centre_dir) / np.linalg.norm(to_centre)
        assert cosang > 0.9999
        assert abs(np.linalg.norm(to_centre) - 18.0) < 1e-3
        assert origin[1] > 5.0


def test_served_arrivals_are_poisson_and_seeded():
    for rate in (20.0, 50.0, 100.0):
        jobs = workloads.served_jobs(rate, 400)
        t = np.array([j.arrival_s for j in jobs])
        assert np.all(np.diff(t) > 0)
        gaps = np.diff(np.concatenate([[0.0], t]))
        assert abs(gaps.mean() * rate - 1.0) < 0.15  # mean gap 1/rate
        assert [j.arrival_s for j in workloads.served_jobs(rate, 400)] == list(t)
        for j in jobs:
            assert j.scene in workloads.SERVE_SCENES and j.spp in (4, 16, 64, 256)
            assert 128 <= j.width <= 2048 and 128 <= j.height <= 2048 and j.width == j.height
    # every rate serves the same jobs; only the arrival times scale with 1/rate
    a, b = workloads.served_jobs(20.0, 48), workloads.served_jobs(100.0, 48)
    assert [(j.scene, j.width, j.height, j.spp, j.depth) for j in a] == [(j.scene, j.width, j.height, j.spp, j.depth) for j in b]
    assert all(np.array_equal(x.camera, y.camera) for x, y in zip(a, b))
    assert np.allclose([j.arrival_s * 20.0 for j in a], [j.arrival_s * 100.0 for j in b], rtol=1e-12)


def test_percentile_is_nearest_rank():
    v = list(range(1, 101))
    assert workloads.percentile(v, 50) == 50
    assert workloads.percentile(v, 99) == 99
    assert workloads.percentile([3.0], 99) == 3.0
    assert math.isnan(workloads.percentile([], 50))
