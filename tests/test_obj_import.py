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


def write_png(path, pixels, colour_type, bit_depth=8, filters=(0, 1, 2, 3, 4), palette=None):
    """A PNG written independently of the library (Python zlib): [H, W, C] samples, the given
    colour type, each row with one of `filters` in turn."""
    import struct
    import zlib
    h, w = pixels.shape[:2]
    c = pixels.shape[2] if pixels.ndim == 3 else 1
    samples = pixels.reshape(h, w * c).astype(np.int64)
    if bit_depth == 16:
        rows = [np.stack([samples[y] >> 8, samples[y] & 255], 1).reshape(-1) for y in range(h)]
        bpp = 2 * c
    else:
        rows = [samples[y] for y in range(h)]
        bpp = c
    raw = b""
    prev = np.zeros_like(rows[0])
    for y, row in enumerate(rows):
        f = filters[y % len(filters)]
        out = np.zeros_like(row)
        for i in range(len(row)):
            a = row[i - bpp] if i >= bpp else 0
            b = prev[i]
            cc = prev[i - bpp] if i >= bpp else 0
            pred = [0, a, b, (a + b) // 2, 0][f]
            if f == 4:
                p = a + b - cc
                pa, pb, pc = abs(p - a), abs(p - b), abs(p - cc)
                pred = a if pa <= pb and pa <= pc else (b if pb <= pc else cc)
            out[i] = (row[i] - pred) & 255
        raw += bytes([f]) + bytes(out.astype(np.uint8))
        prev = row

    def chunk(t, body):
        return struct.pack(">I", len(body)) + t + body + struct.pack(">I", zlib.crc32(t + body) & 0xFFFFFFFF)
    data = b"\x89PNG\r\n\x1a\n" + chunk(b"IHDR", struct.pack(">IIBBBBB", w, h, bit_depth, colour_type, 0, 0, 0))
    if palette is not None:
        data += chunk(b"PLTE", bytes(palette.astype(np.uint8).reshape(-1)))
    data += chunk(b"IDAT", zlib.compress(raw)) + chunk(b"IEND", b"")
    path.write_bytes(data)


def test_obj_texture_maps_are_loaded(tmp_path):
    rng = np.random.default_rng(3)
    albedo = rng.integers(0, 256, (5, 7, 3))
    rma = rng.integers(0, 256, (4, 6, 4))
    shin = rng.integers(0, 65536, (3, 5, 1))
    pal = rng.integers(0, 256, (4, 3))
    idx = rng.integers(0, 4, (6, 6, 1))
    write_png(tmp_path / "albedo.png", albedo, 2)
    write_png(tmp_path / "rma.png", rma, 6)
    write_png(tmp_path / "shin.png", shin, 0, bit_depth=16)
    write_png(tmp_path / "nrm.png", idx, 3, palette=pal)
    emit = rng.integers(0, 256, (2, 3, 3)).astype(np.uint8)
    (tmp_path / "emit.ppm").write_bytes(b"P6\n# emission\n3 2\n255\n" + emit.tobytes())
    (tmp_path / "t.mtl").write_text(
        "newmtl a\nKd 0.5 0.5 0.5\nmap_Kd albedo.png\nmap_RMA rma.png\nmap_Ns shin.png\nmap_Bump -bm 1.0 nrm.png\nsurface ggx\n"
        "newmtl b\nKe 1 1 1\nmap_Ke emit.ppm\nmap_Kd albedo.png\nflip_textures true\nsurface emissive\n")
    (tmp_path / "t.obj").write_text("mtllib t.mtl\nv 0 0 0\nv 1 0 0\nv 0 1 0\nvt 0 0\nvt 1 0\nvt 0 1\nvn 0 0 1\n"
                                    "usemtl a\nf 1/1/1 2/2/1 3/3/1\nusemtl b\nf 1/1/1 3/3/1 2/2/1\n")
    s = pathtracer.load_obj(str(tmp_path / "t.obj"))
    slots = s.material_textures
    assert slots.shape == (2, 6)
    tex = s.textures

    def get(m, k):
        return tex[slots[m, k]]
    assert get(0, 0)["format"] == 0 and np.array_equal(get(0, 0)["data"], albedo)
    assert get(0, 3)["format"] == 1 and np.array_equal(get(0, 3)["data"], rma)
    assert get(0, 2)["data"].shape == (3, 5, 1) and np.array_equal(get(0, 2)["data"], shin >> 8)
    assert np.array_equal(get(0, 5)["data"], pal[idx[..., 0]])
    assert slots[0, 1] == -1 and slots[0, 4] == -1
    # flip_textures: the same albedo file again, rows reversed, as its own texture
    assert slots[1, 0] != slots[0, 0] and np.array_equal(get(1, 0)["data"], albedo[::-1])
    assert np.array_equal(get(1, 4)["data"], emit[::-1]) and get(1, 4)["format"] == 1
    assert pathtracer.bvh8_check(s)["violations"] == 0


def test_obj_texture_errors(tmp_path):
    (tmp_path / "x.jpg").write_bytes(b"\xff\xd8\xff\xe0not decoded here")
    (tmp_path / "t.mtl").write_text("newmtl a\nmap_Kd x.jpg\n")
    (tmp_path / "t.obj").write_text("mtllib t.mtl\nv 0 0 0\nv 1 0 0\nv 0 1 0\nvt 0 0\nvn 0 0 1\nusemtl a\nf 1/1/1 2/1/1 3/1/1\n")
    with pytest.raises(pathtracer.GptError):
        pathtracer.load_obj(str(tmp_path / "t.obj"))
    bad = np.zeros((2, 2, 3), np.int64)
    write_png(tmp_path / "x.png", bad, 2)
    data = bytearray((tmp_path / "x.png").read_bytes())
    data[40] ^= 0xFF  # inside IDAT: the chunk CRC no longer matches
    (tmp_path / "x.png").write_bytes(bytes(data))
    (tmp_path / "t.mtl").write_text("newmtl a\nmap_Kd x.png\n")
    with pytest.raises(pathtracer.GptError):
        pathtracer.load_obj(str(tmp_path / "t.obj"))
