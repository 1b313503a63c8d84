"""Synthetic workload generators: sizes and encodings of the named scenes."""
import numpy as np
import pytest

import scenes


def test_cornell_box_shape():
    s = scenes.cornell_box(1)
    assert s.triangle_count == 36
    assert s.positions.shape == (36, 3, 3) and s.tangents.shape == (36, 3, 4) and s.uvs.shape == (36, 3, 2)
    models = s.materials["model"][s.material_ids]
    assert (models == scenes.MODEL_EMISSIVE).sum() == 2
    assert (models == scenes.MODEL_DIFFUSE).sum() == 34
    lo = s.positions.reshape(-1, 3).min(0)
    hi = s.positions.reshape(-1, 3).max(0)
    assert np.allclose(lo, 0.0) and np.allclose(hi, 1.0)


def test_cornell_seeded_and_deterministic():
    a, b, c = scenes.cornell_box(1), scenes.cornell_box(1), scenes.cornell_box(2)
    assert np.array_equal(a.positions, b.positions)
    assert not np.array_equal(a.positions, c.positions)


def test_icosphere_counts():
    for level, faces in [(0, 20), (1, 80), (3, 1280), (5, 20480)]:
        v, f = scenes.icosphere(level)
        assert f.shape[0] == faces
        assert np.allclose(np.linalg.norm(v, axis=1), 1.0)


def test_sphere_field_small_materials():
    s = scenes.config_scene("spheres-small")
    assert s.triangle_count == 4 * 1280 + 2 + 8
    models = set(s.materials["model"].tolist())
    assert scenes.MODEL_EMISSIVE in models and scenes.MODEL_DIFFUSE in models
    n = s.normals.reshape(-1, 3)
    assert np.allclose(np.linalg.norm(n, axis=1), 1.0, atol=1e-5)


@pytest.mark.parametrize("value,expected_u8", [(0.0, 0), (1.0, 255), (0.73, 222), (0.5, 188)])
def test_srgb_encoding_matches_reference_rounding(value, expected_u8):
    # LinearNormalizedFloatToSrgbU8 (Manager.cpp:65-79) with lround
    assert scenes._srgb_encode_u8(value) == expected_u8


def test_material_record_layout():
    m = scenes.material(scenes.MODEL_GGX, color=(0.5, 0.5, 0.5), rma=(0.3, 1.0, 1.0), ior=1.5)
    assert m.dtype.itemsize == 80
    assert m["model"][0] == scenes.MODEL_GGX
    assert abs(float(m["rma"][0][0]) - 77 / 255) < 1e-7  # lround(76.5) = 77 (NormalizedFloatToU8)
    assert np.allclose(m["normal"][0], [128 / 255, 128 / 255, 1.0])


def test_hit_ray_set_is_normalized_and_seeded():
    s = scenes.cornell_box(1)
    r1 = scenes.hit_ray_set(s, 4096, seed=3)
    r2 = scenes.hit_ray_set(s, 4096, seed=3)
    assert np.array_equal(r1, r2)
    d = r1[:, 3:6]
    assert np.allclose(np.linalg.norm(d, axis=1), 1.0, atol=1e-5)
