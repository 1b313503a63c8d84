"""Headless OBJ/MTL ingest (host code of the library, no GPU): a scene written as OBJ + MTL comes
back as the same world-space triangles and the reference's constant-material texel encoding."""
import math
import os

import numpy as np
import pytest

import pathtracer
import scenes

MODEL_NAMES = {scenes.MODEL_NORMAL: "normal", scenes.MODEL_DIFFUSE: "diffuse", scenes.MODEL_MIRROR: "mirror",
               scenes.MODEL_PHONG: "phong", scenes.MODEL_GGX: "ggx", scenes.MODEL_EMISSIVE: "emissive"}


def write_obj(scene, directory, with_default=False):
    obj = os.path.join(directory, "scene.obj")
    mtl = os.path.join(directory, "scene.mtl")
    with open(mtl, "w") as f:
        for i, m in enumerate(scene.materials):
            f.write(f"newmtl m{i}\n")
            f.write("Kd %.9g %.9g %.9g\n" % tuple(m["color"]))
            f.write("Ks %.9g %.9g %.9g\n" % tuple(m["specular"]))
            f.write("Ke %.9g %.9g %.9g\n" % tuple(m["emission"]))
            f.write("Ns %.9g\n" % (float(m["shininess"]) * 999.0 + 1.0))
            f.write("Ni %.9g\n" % float(m["ior"]))
            f.write(f"surface {MODEL_NAMES[int(m['model'])]}\n")
    with open(obj, "w") as f:
        f.write("mtllib scene.mtl\n")
        n = scene.triangle_count
        for t in range(n):
            for k in range(3):
                f.write("v %.9g %.9g %.9g\n" % tuple(scene.positions[t, k]))
                f.write("vn %.9g %.9g %.9g\n" % tuple(scene.normals[t, k]))
                f.write("vt %.9g %.9g\n" % tuple(scene.uvs[t, k]))
        # one shape per material keeps the file's triangle order per material
        for mat in range(len(scene.materials)):
            tris = np.nonzero(scene.material_ids == mat)[0]
            if tris.size == 0:
                continue
            f.write(f"o part{mat}\nusemtl m{mat}\n")
            for t in tris:
                c = [3 * t + k + 1 for k in range(3)]
                f.write("f " + " ".join(f"{i}/{i}/{i}" for i in c) + "\n")
        if with_default:
            f.write("o nomat\nusemtl\n")
    return obj


def test_obj_roundtrip_cornell(tmp_path):
    s = scenes.cornell_all_models(1)
    path = write_obj(s, str(tmp_path))
    got = pathtracer.load_obj(path)
    order = np.concatenate([np.nonzero(s.material_ids == m)[0] for m in range(len(s.materials))])
    assert got.triangle_count == s.triangle_count
    assert np.allclose(got.positions, s.positions[order], atol=1e-6)
    assert np.allclose(got.normals, s.normals[order], atol=1e-6)
    assert np.allclose(got.uvs, s.uvs[order], atol=1e-7)
    assert np.array_equal(got.material_ids, s.material_ids[order])
    assert got.material_names == [f"m{i}" for i in range(len(s.materials))]
    assert np.array_equal(got.materials["model"], s.materials["model"])
    assert np.allclose(got.materials["color"], s.materials["color"], atol=2.5e-3)
    assert np.allclose(got.materials["emission"], s.materials["emission"])
    assert np.allclose(got.materials["normal"], s.materials["normal"])
    # the reference's import keeps the default RMA texel for constant materials (Manager.cpp:369-372)
    assert np.allclose(got.materials["rma"], [1.0, 0.0, 1.0])
    t = got.tangents[..., :3].reshape(-1, 3)
    n = got.normals.reshape(-1, 3)
    assert np.allclose(np.linalg.norm(t, axis=1), 1.0, atol=1e-5)
    assert np.max(np.abs((t * n).sum(1))) < 1e-5
    assert set(np.unique(got.tangents[..., 3]).tolist()) <= {-1.0, 1.0}
    assert pathtracer.bvh8_check(got)["violations"] == 0


def test_obj_transform_and_errors(tmp_path):
    s = scenes.cornell_box(1)
    path = write_obj(s, str(tmp_path))
    a = math.radians(30.0)
    m = np.array([[math.cos(a), 0, math.sin(a), 1.0], [0, 2.0, 0, 0.5], [-math.sin(a), 0, math.cos(a), -2.0], [0, 0, 0, 1]],
                 dtype=np.float32)
    got = pathtracer.load_obj(path, transform=m)
    base = pathtracer.load_obj(path)
    p = np.concatenate([base.positions.reshape(-1, 3), np.ones((base.triangle_count * 3, 1), np.float32)], 1)
    assert np.allclose(got.positions.reshape(-1, 3), (p @ m.T)[:, :3], atol=1e-5)
    nrm = got.normals.reshape(-1, 3)
    assert np.allclose(np.linalg.norm(nrm, axis=1), 1.0, atol=1e-5)
    with pytest.raises(pathtracer.GptError):
        pathtracer.load_obj(str(tmp_path / "missing.obj"))
    bad = tmp_path / "nonormals.obj"
    bad.write_text("v 0 0 0\nv 1 0 0\nv 0 1 0\nvt 0 0\nf 1/1 2/1 3/1\n")
    with pytest.raises(pathtracer.GptError):  # the reference requires vertex normals
        pathtracer.load_obj(str(bad))


def test_obj_polygon_fan_and_default_material(tmp_path):
    p = tmp_path / "quad.obj"
    p.write_text("v 0 0 0\nv 1 0 0\nv 1 1 0\nv 0 1 0\nvt 0 0\nvt 1 0\nvt 1 1\nvt 0 1\nvn 0 0 1\n"
                 "f 1/1/1 2/2/1 3/3/1 4/4/1\nf -4/-4/-1 -3/-3/-1 -2/-2/-1\n")
    got = pathtracer.load_obj(str(p))
    assert got.triangle_count == 3
    assert got.material_names == ["default"]
    assert got.materials["model"][0] == scenes.MODEL_DIFFUSE
    assert np.allclose(got.materials["color"][0], 1.0)
