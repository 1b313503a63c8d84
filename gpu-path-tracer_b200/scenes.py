"""Seeded synthetic scenes and ray sets for the wavefront path tracer.

The reference renders OBJ/MTL scenes whose assets are not part of its tree, so
every workload here is generated from a seed. Scenes are returned as flat,
world-space triangle arrays: exactly what the reference's
``BuildTriangles`` produces from its ECS registry
(Core/Source/Graphics/Cuda/PathTracing/Renderer.cpp:159-213) and what the C-ABI
``gpt_init_scene_buffers`` takes.

Material constants are encoded the way the reference's asset importer encodes
an MTL constant (Core/Source/Assets/Manager.cpp:56-88,321-380): colours become
sRGB u8 texels (``lround``) that the texture unit decodes back to linear;
shininess becomes a linear u8 of ``(s - 1) / 999``; RMA values are linear u8
texels; emission is stored as float32; the normal map is the default
``(128, 128, 255)`` texel.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

# GlobalShadingModel order (Core/Include/Core/Graphics/Cuda/PathTracing/Material.hpp:8-17)
MODEL_NORMAL, MODEL_DIFFUSE, MODEL_MIRROR, MODEL_PHONG, MODEL_GGX, MODEL_EMISSIVE = range(6)

MATERIAL_DTYPE = np.dtype([
    ("model", "<u4"),
    ("color", "<f4", 3),
    ("specular", "<f4", 3),
    ("shininess", "<f4"),      # normalised texel in [0, 1]; shininess = t * 999 + 1
    ("rma", "<f4", 3),
    ("emission", "<f4", 3),
    ("normal", "<f4", 3),      # tangent-space normal-map texel in [0, 1]
    ("ior", "<f4"),
    ("transmission", "<f4"),
    ("pad", "<f4"),
])
assert MATERIAL_DTYPE.itemsize == 80


def _srgb_encode_u8(x: float) -> int:
    """LinearNormalizedFloatToSrgbU8 (Manager.cpp:65-79)."""
    x = np.float32(x)
    if not np.isfinite(x):
        x = np.float32(0.0)
    x = np.float32(min(max(float(x), 0.0), 1.0))
    if x <= np.float32(0.0031308):
        s = np.float32(12.92) * x
    else:
        s = np.float32(1.055) * np.float32(math.pow(float(x), 1.0 / 2.4)) - np.float32(0.055)
    v = float(np.float32(s) * np.float32(255.0))
    return int(math.floor(v + 0.5)) if v >= 0 else int(math.ceil(v - 0.5))


def _srgb_decode(u8: int) -> float:
    """sRGB texel -> linear, as the texture unit decodes an sRGB texture."""
    c = u8 / 255.0
    lin = c / 12.92 if c <= 0.04045 else ((c + 0.055) / 1.055) ** 2.4
    return float(np.float32(lin))


def _linear_u8(x: float) -> int:
    """NormalizedFloatToU8 (Manager.cpp:48-54)."""
    x = min(max(float(np.float32(x)), 0.0), 1.0)
    return int(math.floor(float(np.float32(x) * np.float32(255.0)) + 0.5))


def srgb_texel(rgb) -> list[float]:
    return [_srgb_decode(_srgb_encode_u8(c)) for c in rgb]


def linear_texel(values) -> list[float]:
    return [float(np.float32(_linear_u8(v) / 255.0)) for v in values]


DEFAULT_NORMAL_TEXEL = [float(np.float32(128 / 255.0)), float(np.float32(128 / 255.0)), 1.0]


def material(model: int, color=(1.0, 1.0, 1.0), specular=(0.0, 0.0, 0.0), shininess=1.0,
             rma=(1.0, 0.0, 1.0), emission=(0.0, 0.0, 0.0), ior=1.0, transmission=0.0) -> np.ndarray:
    """One material record from MTL-style constants, texel-encoded as the reference does."""
    rec = np.zeros(1, dtype=MATERIAL_DTYPE)
    rec["model"] = model
    rec["color"] = srgb_texel(color)
    rec["specular"] = srgb_texel(specular)
    s = min(max(float(shininess), 1.0), 1000.0)
    rec["shininess"] = linear_texel([(s - 1.0) / 999.0])[0]
    rec["rma"] = linear_texel(rma)
    rec["emission"] = np.asarray(emission, dtype=np.float32)
    rec["normal"] = DEFAULT_NORMAL_TEXEL
    rec["ior"] = ior
    rec["transmission"] = transmission
    return rec


@dataclass
class Scene:
    """World-space triangle soup plus its material table."""
    positions: np.ndarray      # [T, 3, 3] float32
    normals: np.ndarray        # [T, 3, 3] float32
    tangents: np.ndarray       # [T, 3, 4] float32 (xyz + handedness sign)
    uvs: np.ndarray            # [T, 3, 2] float32
    material_ids: np.ndarray   # [T] uint32
    materials: np.ndarray      # [M] MATERIAL_DTYPE
    name: str = "scene"
    camera: dict = field(default_factory=dict)
    textures: list = field(default_factory=list)      # [{"data": [H, W, C] u8/f32 array, "format": 0/1/2}]
    material_textures: np.ndarray | None = None       # [M, 6] int32 texture index per slot, -1 = constant

    @property
    def triangle_count(self) -> int:
        return int(self.positions.shape[0])

    def contiguous(self) -> "Scene":
        self.positions = np.ascontiguousarray(self.positions, dtype=np.float32)
        self.normals = np.ascontiguousarray(self.normals, dtype=np.float32)
        self.tangents = np.ascontiguousarray(self.tangents, dtype=np.float32)
        self.uvs = np.ascontiguousarray(self.uvs, dtype=np.float32)
        self.material_ids = np.ascontiguousarray(self.material_ids, dtype=np.uint32)
        self.materials = np.ascontiguousarray(self.materials)
        return self


def make_camera(position, look_at, fov_y_degrees: float, aspect: float, up=(0.0, 1.0, 0.0)) -> np.ndarray:
    """Pinhole camera as (origin, lowerLeftCorner, horizontal, vertical), 12 float32.

    Same construction as MakeDeviceCamera (Renderer.cpp:237-257) with the frame
    (right, up, forward) given by a look-at instead of a quaternion.
    """
    f32 = np.float32
    pos = np.asarray(position, dtype=np.float32)
    fwd = np.asarray(look_at, dtype=np.float32) - pos
    fwd = (fwd / np.float32(np.sqrt(np.dot(fwd, fwd)))).astype(np.float32)
    right = np.cross(fwd, np.asarray(up, dtype=np.float32)).astype(np.float32)
    right = (right / np.float32(np.sqrt(np.dot(right, right)))).astype(np.float32)
    upv = np.cross(right, fwd).astype(np.float32)
    half_h = f32(math.tan(math.radians(fov_y_degrees) * 0.5))
    half_w = f32(half_h * f32(aspect))
    horizontal = (f32(2.0) * half_w) * right
    vertical = (f32(2.0) * half_h) * upv
    llc = pos + fwd - half_w * right - half_h * upv
    return np.concatenate([pos, llc, horizontal, vertical]).astype(np.float32)


# ----------------------------------------------------------------------------
# Triangle helpers
# ----------------------------------------------------------------------------

def _quad(p0, p1, p2, p3, normal):
    """Two triangles (p0,p1,p2), (p0,p2,p3) with flat normal, u along p0->p1."""
    tris = np.array([[p0, p1, p2], [p0, p2, p3]], dtype=np.float32)
    uv = np.array([[[0, 0], [1, 0], [1, 1]], [[0, 0], [1, 1], [0, 1]]], dtype=np.float32)
    nv = np.asarray(normal, dtype=np.float64)
    nv = (nv / np.linalg.norm(nv)).astype(np.float32)
    n = np.broadcast_to(nv, (2, 3, 3)).copy()
    t = np.asarray(p1, dtype=np.float32) - np.asarray(p0, dtype=np.float32)
    t = t / np.linalg.norm(t)
    tan = np.zeros((2, 3, 4), dtype=np.float32)
    tan[..., :3] = t
    tan[..., 3] = 1.0
    return tris, n, tan, uv


def _box(center_xz, size, height, yaw):
    """Axis box of footprint size x size and given height, rotated by yaw about +Y; 12 triangles, outward normals."""
    c, s = math.cos(yaw), math.sin(yaw)
    hx = size * 0.5

    def xf(lx, y, lz):
        return [center_xz[0] + c * lx + s * lz, y, center_xz[1] - s * lx + c * lz]

    def rot(nx, ny, nz):
        return [c * nx + s * nz, ny, -s * nx + c * nz]

    quads = [
        # top (+y)
        (xf(-hx, height, hx), xf(hx, height, hx), xf(hx, height, -hx), xf(-hx, height, -hx), rot(0, 1, 0)),
        # bottom (-y)
        (xf(-hx, 0, -hx), xf(hx, 0, -hx), xf(hx, 0, hx), xf(-hx, 0, hx), rot(0, -1, 0)),
        # +z
        (xf(-hx, 0, hx), xf(hx, 0, hx), xf(hx, height, hx), xf(-hx, height, hx), rot(0, 0, 1)),
        # -z
        (xf(hx, 0, -hx), xf(-hx, 0, -hx), xf(-hx, height, -hx), xf(hx, height, -hx), rot(0, 0, -1)),
        # +x
        (xf(hx, 0, hx), xf(hx, 0, -hx), xf(hx, height, -hx), xf(hx, height, hx), rot(1, 0, 0)),
        # -x
        (xf(-hx, 0, -hx), xf(-hx, 0, hx), xf(-hx, height, hx), xf(-hx, height, -hx), rot(-1, 0, 0)),
    ]
    parts = [_quad(*q) for q in quads]
    return [np.concatenate([p[i] for p in parts]) for i in range(4)]


def _assemble(parts, materials, name, camera=None) -> Scene:
    pos = np.concatenate([p[0] for p in parts]).astype(np.float32)
    nrm = np.concatenate([p[1] for p in parts]).astype(np.float32)
    tan = np.concatenate([p[2] for p in parts]).astype(np.float32)
    uv = np.concatenate([p[3] for p in parts]).astype(np.float32)
    mid = np.concatenate([np.full(p[0].shape[0], p[4], dtype=np.uint32) for p in parts])
    mats = np.concatenate(materials)
    return Scene(pos, nrm, tan, uv, mid, mats, name=name, camera=camera or {}).contiguous()


# ----------------------------------------------------------------------------
# C1: procedural Cornell box (36 triangles)
# ----------------------------------------------------------------------------

def cornell_box(seed: int = 1) -> Scene:
    """5 wall quads in the 0..1 m cube, two boxes (heights 0.3 and 0.6, seeded yaw
    in [0, pi/2)), one ceiling emitter quad with radiance (17, 12, 4); Lambert
    albedo 0.73 white, 0.65 red and green walls."""
    rng = np.random.default_rng(seed)
    white = material(MODEL_DIFFUSE, color=(0.73, 0.73, 0.73))
    red = material(MODEL_DIFFUSE, color=(0.65, 0.05, 0.05))
    green = material(MODEL_DIFFUSE, color=(0.12, 0.65, 0.15))
    light = material(MODEL_EMISSIVE, emission=(17.0, 12.0, 4.0))
    mats = [white, red, green, light]
    parts = []

    def add(q, mid):
        parts.append((*q, mid))

    add(_quad([0, 0, 1], [1, 0, 1], [1, 0, 0], [0, 0, 0], [0, 1, 0]), 0)      # floor
    add(_quad([0, 1, 0], [1, 1, 0], [1, 1, 1], [0, 1, 1], [0, -1, 0]), 0)     # ceiling
    add(_quad([0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], [0, 0, 1]), 0)      # back wall
    add(_quad([0, 0, 1], [0, 0, 0], [0, 1, 0], [0, 1, 1], [1, 0, 0]), 1)      # left wall (red)
    add(_quad([1, 0, 0], [1, 0, 1], [1, 1, 1], [1, 1, 0], [-1, 0, 0]), 2)     # right wall (green)
    yaw = rng.uniform(0.0, math.pi / 2, size=2)
    add(_box((0.33, 0.62), 0.28, 0.3, float(yaw[0])), 0)
    add(_box((0.66, 0.32), 0.28, 0.6, float(yaw[1])), 0)
    add(_quad([0.38, 0.999, 0.38], [0.62, 0.999, 0.38], [0.62, 0.999, 0.62], [0.38, 0.999, 0.62], [0, -1, 0]), 3)
    cam = dict(position=(0.5, 0.5, 2.0), look_at=(0.5, 0.5, 0.0), fov_y=40.0)
    return _assemble(parts, mats, "cornell-box", cam)


def cornell_all_models(seed: int = 1) -> Scene:
    """The Cornell box with every shading model of the reference on some surface: Lambert
    floor and left wall, Phong ceiling and tall box, GGX back wall (metal) and right wall
    (dielectric), mirror short box, a Normal-model panel and the emitter."""
    rng = np.random.default_rng(seed)
    mats = [
        material(MODEL_DIFFUSE, color=(0.73, 0.73, 0.73)),                                           # 0 floor
        material(MODEL_PHONG, color=(0.5, 0.5, 0.5), specular=(0.3, 0.3, 0.3), shininess=50.0),       # 1 ceiling
        material(MODEL_GGX, color=(0.9, 0.7, 0.5), rma=(0.3, 1.0, 1.0), ior=1.5),                     # 2 back wall
        material(MODEL_DIFFUSE, color=(0.65, 0.05, 0.05)),                                            # 3 left
        material(MODEL_GGX, color=(0.12, 0.65, 0.15), rma=(0.5, 0.0, 1.0), ior=1.5),                 # 4 right
        material(MODEL_MIRROR, specular=(0.9, 0.9, 0.9)),                                             # 5 short box
        material(MODEL_PHONG, color=(0.4, 0.4, 0.6), specular=(0.5, 0.5, 0.5), shininess=200.0),     # 6 tall box
        material(MODEL_NORMAL),                                                                       # 7 panel
        material(MODEL_EMISSIVE, emission=(17.0, 12.0, 4.0)),                                         # 8 light
    ]
    parts = []

    def add(q, mid):
        parts.append((*q, mid))

    add(_quad([0, 0, 1], [1, 0, 1], [1, 0, 0], [0, 0, 0], [0, 1, 0]), 0)
    add(_quad([0, 1, 0], [1, 1, 0], [1, 1, 1], [0, 1, 1], [0, -1, 0]), 1)
    add(_quad([0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], [0, 0, 1]), 2)
    add(_quad([0, 0, 1], [0, 0, 0], [0, 1, 0], [0, 1, 1], [1, 0, 0]), 3)
    add(_quad([1, 0, 0], [1, 0, 1], [1, 1, 1], [1, 1, 0], [-1, 0, 0]), 4)
    yaw = rng.uniform(0.0, math.pi / 2, size=2)
    add(_box((0.33, 0.62), 0.28, 0.3, float(yaw[0])), 5)
    add(_box((0.66, 0.32), 0.28, 0.6, float(yaw[1])), 6)
    add(_quad([0.08, 0.7, 0.25], [0.25, 0.7, 0.25], [0.25, 0.87, 0.25], [0.08, 0.87, 0.25], [0.3, 0.2, 0.93]), 7)
    add(_quad([0.38, 0.999, 0.38], [0.62, 0.999, 0.38], [0.62, 0.999, 0.62], [0.38, 0.999, 0.62], [0, -1, 0]), 8)
    cam = dict(position=(0.5, 0.5, 2.0), look_at=(0.5, 0.5, 0.0), fov_y=40.0)
    return _assemble(parts, mats, "cornell-all-models", cam)


TEXEL_U8_SRGB, TEXEL_U8_LINEAR, TEXEL_F32 = 0, 1, 2
SLOT_COLOR, SLOT_SPECULAR, SLOT_SHININESS, SLOT_RMA, SLOT_EMISSION, SLOT_NORMAL = range(6)


def cornell_textured(seed: int = 1) -> Scene:
    """The all-models Cornell box with image textures in every material slot somewhere: a checker
    albedo (sRGB) on the floor and back wall, a bump normal map on the floor, a shininess map on
    the Phong ceiling, an RMA map on the GGX walls, a specular map on the mirror box and an HDR
    emission map on the light."""
    rng = np.random.default_rng(seed)
    s = cornell_all_models(seed)
    yy, xx = np.mgrid[0:64, 0:64]
    checker = ((xx // 8 + yy // 8) % 2).astype(np.float64)
    albedo = np.stack([60 + 150 * checker, 80 + 120 * (1 - checker), np.full_like(checker, 140)], -1).astype(np.uint8)
    hx = np.sin(xx / 64 * 2 * np.pi * 4) * 0.35
    hy = np.cos(yy / 64 * 2 * np.pi * 3) * 0.35
    nrm = np.stack([hx, hy, np.ones_like(hx)], -1)
    nrm /= np.linalg.norm(nrm, axis=-1, keepdims=True)
    normal = np.round((nrm * 0.5 + 0.5) * 255).astype(np.uint8)
    shin = rng.integers(20, 200, (16, 16, 1)).astype(np.uint8)
    rma = np.stack([rng.integers(30, 230, (16, 16)), rng.integers(0, 256, (16, 16)), np.full((16, 16), 255)], -1).astype(np.uint8)
    spec = rng.integers(150, 256, (16, 16, 3)).astype(np.uint8)
    emis = (rng.random((8, 8, 3)) * np.array([17.0, 12.0, 4.0]) * 1.5).astype(np.float32)
    s.textures = [dict(data=albedo, format=TEXEL_U8_SRGB), dict(data=normal, format=TEXEL_U8_LINEAR),
                  dict(data=shin, format=TEXEL_U8_LINEAR), dict(data=rma, format=TEXEL_U8_LINEAR),
                  dict(data=spec, format=TEXEL_U8_SRGB), dict(data=emis, format=TEXEL_F32)]
    slots = np.full((len(s.materials), 6), -1, dtype=np.int32)
    slots[0, SLOT_COLOR] = 0      # floor: albedo + normal map
    slots[0, SLOT_NORMAL] = 1
    slots[1, SLOT_SHININESS] = 2  # phong ceiling
    slots[2, SLOT_COLOR] = 0      # GGX back wall: albedo + rma
    slots[2, SLOT_RMA] = 3
    slots[4, SLOT_RMA] = 3        # GGX right wall
    slots[5, SLOT_SPECULAR] = 4   # mirror box
    slots[8, SLOT_EMISSION] = 5   # light
    s.material_textures = slots
    s.name = "cornell-textured"
    return s


# ----------------------------------------------------------------------------
# Displaced icospheres (C2-C5)
# ----------------------------------------------------------------------------

def icosphere(level: int):
    """Unit icosphere: returns (vertices [V,3] float64, faces [F,3] int64), F = 20 * 4^level."""
    t = (1.0 + math.sqrt(5.0)) / 2.0
    verts = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
             (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
             (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5),
             (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    v = np.array(verts, dtype=np.float64)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    f = np.array(faces, dtype=np.int64)
    for _ in range(level):
        e = np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]])
        e.sort(axis=1)
        uniq, inv = np.unique(e, axis=0, return_inverse=True)
        inv = inv.reshape(-1)
        mids = v[uniq[:, 0]] + v[uniq[:, 1]]
        mids /= np.linalg.norm(mids, axis=1, keepdims=True)
        base = v.shape[0]
        v = np.concatenate([v, mids])
        n = f.shape[0]
        a = inv[:n] + base
        b = inv[n:2 * n] + base
        c = inv[2 * n:] + base
        f = np.concatenate([
            np.stack([f[:, 0], a, c], 1), np.stack([f[:, 1], b, a], 1),
            np.stack([f[:, 2], c, b], 1), np.stack([a, b, c], 1)])
    return v, f


def _perlin_perm(rng):
    p = rng.permutation(256)
    return np.concatenate([p, p]).astype(np.int64)


def perlin3(p: np.ndarray, perm: np.ndarray) -> np.ndarray:
    """Gradient noise in [-1, 1] (Perlin, "Improving Noise", SIGGRAPH 2002)."""
    pi = np.floor(p).astype(np.int64)
    f = p - pi
    pi &= 255
    u = f * f * f * (f * (f * 6 - 15) + 10)

    def grad(h, x, y, z):
        h = h & 15
        a = np.where(h < 8, x, y)
        b = np.where(h < 4, y, np.where((h == 12) | (h == 14), x, z))
        return np.where(h & 1, -a, a) + np.where(h & 2, -b, b)

    X, Y, Z = pi[:, 0], pi[:, 1], pi[:, 2]
    x, y, z = f[:, 0], f[:, 1], f[:, 2]
    A = perm[X] + Y
    AA = perm[A] + Z
    AB = perm[A + 1] + Z
    B = perm[X + 1] + Y
    BA = perm[B] + Z
    BB = perm[B + 1] + Z

    def lerp(t, a, b):
        return a + t * (b - a)

    return lerp(u[:, 2],
                lerp(u[:, 1], lerp(u[:, 0], grad(perm[AA], x, y, z), grad(perm[BA], x - 1, y, z)),
                     lerp(u[:, 0], grad(perm[AB], x, y - 1, z), grad(perm[BB], x - 1, y - 1, z))),
                lerp(u[:, 1], lerp(u[:, 0], grad(perm[AA + 1], x, y, z - 1), grad(perm[BA + 1], x - 1, y, z - 1)),
                     lerp(u[:, 0], grad(perm[AB + 1], x, y - 1, z - 1), grad(perm[BB + 1], x - 1, y - 1, z - 1))))


_ICO_CACHE: dict = {}


def displaced_sphere(center, radius, level, perm, amplitude=0.05, frequency=3.0):
    """Icosphere displaced along its normal by amplitude * r * noise; per-vertex
    smooth normals, tangents along +phi, spherical uvs. Returns per-triangle arrays."""
    if level not in _ICO_CACHE:
        _ICO_CACHE[level] = icosphere(level)
    v, f = _ICO_CACHE[level]
    disp = perlin3(v * frequency + np.asarray(center) * 0.173, perm)
    pos = np.asarray(center, dtype=np.float64) + v * (radius * (1.0 + amplitude * disp))[:, None]
    tri = pos[f]
    fn = np.cross(tri[:, 1] - tri[:, 0], tri[:, 2] - tri[:, 0])
    vn = np.zeros_like(pos)
    for k in range(3):
        np.add.at(vn, f[:, k], fn)
    vn /= np.linalg.norm(vn, axis=1, keepdims=True)
    up = np.array([0.0, 1.0, 0.0])
    tn = np.cross(up, vn)
    bad = np.linalg.norm(tn, axis=1) < 1e-6
    tn[bad] = np.array([1.0, 0.0, 0.0])
    tn /= np.linalg.norm(tn, axis=1, keepdims=True)
    uvv = np.stack([0.5 + np.arctan2(v[:, 2], v[:, 0]) / (2 * math.pi), 0.5 - np.arcsin(np.clip(v[:, 1], -1, 1)) / math.pi], 1)
    tans = np.concatenate([tn, np.ones((tn.shape[0], 1))], 1)
    return (tri.astype(np.float32), vn[f].astype(np.float32), tans[f].astype(np.float32), uvv[f].astype(np.float32))


def sphere_field(n_spheres: int = 64, level: int = 5, n_lights: int = 256, seed: int = 2, box: float = 20.0,
                 name: str | None = None) -> Scene:
    """Displaced icospheres (20,480 tris each at level 5) placed uniformly in a
    box over a 2-triangle ground plane, with emissive triangles above them.
    Materials per mesh: 40% Lambert (albedo U[0.1,0.9]^3), 40% GGX (roughness
    U[0.05,0.8]; half dielectric F0 = 0.04 i.e. ior 1.5, half metal with
    F0 = base colour U[0.5,1]^3), 20% mirror. Light emission is log-uniform over
    3 decades."""
    rng = np.random.default_rng(seed)
    perm = _perlin_perm(rng)
    parts = []
    mats = []
    kinds = np.array([0] * int(round(0.4 * n_spheres)) + [1] * int(round(0.4 * n_spheres)), dtype=np.int64)
    kinds = np.concatenate([kinds, np.full(max(0, n_spheres - kinds.size), 2, dtype=np.int64)])[:n_spheres]
    rng.shuffle(kinds)
    for i in range(n_spheres):
        r = float(rng.uniform(0.5, 1.5))
        c = [float(rng.uniform(r, box - r)), float(rng.uniform(r, box * 0.5)), float(rng.uniform(r, box - r))]
        k = int(kinds[i])
        if k == 0:
            m = material(MODEL_DIFFUSE, color=tuple(rng.uniform(0.1, 0.9, 3)))
        elif k == 1:
            rough = float(rng.uniform(0.05, 0.8))
            if rng.uniform() < 0.5:
                m = material(MODEL_GGX, color=tuple(rng.uniform(0.1, 0.9, 3)), rma=(rough, 0.0, 1.0), ior=1.5)
            else:
                m = material(MODEL_GGX, color=tuple(rng.uniform(0.5, 1.0, 3)), rma=(rough, 1.0, 1.0), ior=1.5)
        else:
            m = material(MODEL_MIRROR, specular=(0.9, 0.9, 0.9))
        mats.append(m)
        parts.append((*displaced_sphere(c, r, level, perm), len(mats) - 1))
    # ground plane (2 triangles)
    mats.append(material(MODEL_DIFFUSE, color=(0.5, 0.5, 0.5)))
    g = 2.0 * box
    parts.append((*_quad([-box * 0.5, 0, box * 1.5], [box * 1.5, 0, box * 1.5], [box * 1.5, 0, -box * 0.5],
                         [-box * 0.5, 0, -box * 0.5], [0, 1, 0]), len(mats) - 1))
    del g
    # emissive triangles above the spheres, facing down
    for _ in range(n_lights):
        cx, cz = rng.uniform(0.0, box, 2)
        cy = float(rng.uniform(0.7 * box, 0.95 * box))
        s = float(rng.uniform(0.3, 0.8))
        a = float(rng.uniform(0, 2 * math.pi))
        p = [[cx + s * math.cos(a + k * 2.0944), cy, cz + s * math.sin(a + k * 2.0944)] for k in range(3)]
        tri = np.array([[p[0], p[2], p[1]]], dtype=np.float32)
        n = np.broadcast_to(np.array([0, -1, 0], dtype=np.float32), (1, 3, 3)).copy()
        tan = np.zeros((1, 3, 4), dtype=np.float32)
        tan[..., 0] = 1.0
        tan[..., 3] = 1.0
        uv = np.array([[[0, 0], [1, 0], [0, 1]]], dtype=np.float32)
        power = 10.0 ** float(rng.uniform(0.0, 3.0))
        col = rng.uniform(0.5, 1.0, 3)
        mats.append(material(MODEL_EMISSIVE, emission=tuple(col * power * 0.05)))
        parts.append((tri, n, tan, uv, len(mats) - 1))
    cam = dict(position=(box * 0.5, box * 0.45, -box * 0.7), look_at=(box * 0.5, box * 0.15, box * 0.5), fov_y=45.0)
    return _assemble(parts, mats, name or f"spheres-{n_spheres}x{level}", cam)


# name: (spheres, subdivision level, emissive triangles, seed). Level-5 spheres have 20,480
# triangles, level-4 ones 5,120; every field adds a 2-triangle ground plane.
SPHERE_FIELDS = {
    "spheres-1m": (64, 5, 256, 2),
    "spheres-10k": (2, 4, 16, 3),
    "spheres-200k": (10, 5, 64, 4),
    "spheres-2m": (100, 5, 256, 5),
    "spheres-8m": (400, 5, 4096, 6),
    "spheres-small": (4, 3, 8, 7),
    # resident scenes of the served workload (50k-4M triangles)
    "spheres-50k": (10, 4, 32, 8),
    "spheres-100k": (5, 5, 32, 9),
    "spheres-250k": (12, 5, 64, 10),
    "spheres-500k": (25, 5, 128, 11),
    "spheres-3m": (150, 5, 256, 12),
    "spheres-4m": (200, 5, 256, 13),
}


def config_scene(name: str) -> Scene:
    """Named workloads: 'cornell' (36 tris), 'spheres-1m' (64 spheres, 1.31 M tris),
    'spheres-10k', 'spheres-200k', 'spheres-2m', 'spheres-8m'."""
    if name == "cornell":
        return cornell_box(1)
    if name == "cornell-all":
        return cornell_all_models(1)
    if name == "cornell-textured":
        return cornell_textured(1)
    n, lvl, nl, seed = SPHERE_FIELDS[name]
    return sphere_field(n, lvl, nl, seed, name=name)


def scene_camera(scene: Scene, width: int, height: int) -> np.ndarray:
    c = scene.camera
    return make_camera(c["position"], c["look_at"], c["fov_y"], width / height)


def hit_ray_set(scene: Scene, n: int, seed: int = 11, width: int = 512, height: int = 512) -> np.ndarray:
    """A fixed ray set [n, 8] (origin3, dir3, tMin, tMax): half jittered camera
    rays, half rays from points uniform in the scene bounds with directions
    uniform on the sphere."""
    rng = np.random.default_rng(seed)
    cam = scene_camera(scene, width, height)
    n_cam = n // 2
    u = rng.random(n_cam, dtype=np.float32)
    v = rng.random(n_cam, dtype=np.float32)
    o = cam[0:3]
    llc, hor, ver = cam[3:6], cam[6:9], cam[9:12]
    d = llc[None, :] + u[:, None] * hor[None, :] + v[:, None] * ver[None, :] - o[None, :]
    d = d / np.sqrt((d * d).sum(1, keepdims=True))
    lo = scene.positions.reshape(-1, 3).min(0)
    hi = scene.positions.reshape(-1, 3).max(0)
    n_rand = n - n_cam
    ro = lo[None, :] + rng.random((n_rand, 3), dtype=np.float32) * (hi - lo)[None, :]
    rd = rng.normal(size=(n_rand, 3)).astype(np.float32)
    rd = rd / np.sqrt((rd * rd).sum(1, keepdims=True))
    rays = np.zeros((n, 8), dtype=np.float32)
    rays[:n_cam, 0:3] = o
    rays[:n_cam, 3:6] = d
    rays[n_cam:, 0:3] = ro
    rays[n_cam:, 3:6] = rd
    rays[:, 6] = np.float32(1e-4)
    rays[:, 7] = np.float32(1e34)
    return rays
