"""ORACLE — test infrastructure only: ctypes binding of oracle/_ref/libref_harness.so.

The library holds the reference's own kernels (built from the reference sources by
oracle/ref_harness/Makefile) behind a small driver. tests/ use it to pin the oracle
against the reference; bench.py uses it to time the reference's build on the same GPU.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_ref", "libref_harness.so")
LIB_PATH_NOFMA = os.path.join(_HERE, "_ref", "libref_harness_nofma.so")
_libs = {}

REF_MATERIAL_DTYPE = np.dtype([("model", "<u4"), ("color", "<u4"), ("specular", "<u4"), ("shininess", "<u4"),
                               ("rma", "<u4"), ("normal", "<u4"), ("emission", "<f4", 3), ("ior", "<f4"),
                               ("transmission", "<f4"), ("pad", "<u4")])
assert REF_MATERIAL_DTYPE.itemsize == 48
IMAGE_DTYPE = np.dtype([("width", "<u4"), ("height", "<u4"), ("channels", "<u4"), ("format", "<u4"), ("data", "<u8")])


LIB_PATH_MIKK = os.path.join(_HERE, "_ref", "libmikk_ref.so")


def mikk_available() -> bool:
    return os.path.exists(LIB_PATH_MIKK)


def mikk_tangents(positions, normals, uvs, indices) -> np.ndarray:
    """Per-vertex tangents [V, 4] from the reference's own MikkTSpace build (oracle/_ref/libmikk_ref.so)."""
    if "mikk" not in _libs:
        L = ctypes.CDLL(LIB_PATH_MIKK)
        L.mikk_ref_tangents.restype = ctypes.c_int
        L.mikk_ref_tangents.argtypes = [ctypes.c_void_p] * 4 + [ctypes.c_int, ctypes.c_void_p]
        _libs["mikk"] = L
    p = np.ascontiguousarray(positions, dtype=np.float32).reshape(-1, 3)
    n = np.ascontiguousarray(normals, dtype=np.float32).reshape(-1, 3)
    t = np.ascontiguousarray(uvs, dtype=np.float32).reshape(-1, 2)
    i = np.ascontiguousarray(indices, dtype=np.uint32).reshape(-1, 3)
    out = np.zeros((p.shape[0], 4), dtype=np.float32)
    out[:, 0] = 1.0
    out[:, 3] = -1.0
    rc = _libs["mikk"].mikk_ref_tangents(_p(p), _p(n), _p(t), _p(i), i.shape[0], _p(out))
    if rc:
        raise RuntimeError("genTangSpaceDefault failed")
    return out


def available() -> bool:
    return os.path.exists(LIB_PATH) and os.path.exists(LIB_PATH_NOFMA)


def lib(fma: bool = True):
    """fma=True: the reference's own build flags; fma=False: the same sources with -fmad=false."""
    if fma not in _libs:
        L = ctypes.CDLL(LIB_PATH if fma else LIB_PATH_NOFMA)
        vp, u32 = ctypes.c_void_p, ctypes.c_uint32
        L.ref_scene_create.restype = vp
        L.ref_scene_create.argtypes = [u32, vp, vp, vp, vp, vp, u32, vp, ctypes.POINTER(ctypes.c_int), u32, vp, vp]
        L.ref_scene_destroy.argtypes = [vp]
        L.ref_scene_info.argtypes = [vp, vp, vp, vp]
        L.ref_scene_decoded_materials.argtypes = [vp, vp]
        L.ref_trace_closest.argtypes = [vp, vp, u32, vp, vp]
        L.ref_render.argtypes = [vp, vp, u32, u32, u32, u32, u32, u32, vp, vp, vp, u32, vp, vp]
        _libs[fma] = L
    return _libs[fma]


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _srgb_code(v: float) -> int:
    """u8 sRGB code whose decoded value is v (materials are generated from such codes)."""
    codes = np.arange(256) / 255.0
    lin = np.where(codes <= 0.04045, codes / 12.92, ((codes + 0.055) / 1.055) ** 2.4).astype(np.float32)
    k = int(np.argmin(np.abs(lin - np.float32(v))))
    return k


def _pack(codes) -> int:
    return int(codes[0]) | (int(codes[1]) << 8) | (int(codes[2]) << 16)


def reference_materials(materials: np.ndarray) -> np.ndarray:
    """The material table as the reference's texel codes (Manager.cpp:321-380)."""
    out = np.zeros(len(materials), dtype=REF_MATERIAL_DTYPE)
    for i, m in enumerate(materials):
        out[i]["model"] = m["model"]
        out[i]["color"] = _pack([_srgb_code(c) for c in m["color"]])
        out[i]["specular"] = _pack([_srgb_code(c) for c in m["specular"]])
        out[i]["shininess"] = int(round(float(m["shininess"]) * 255.0))
        out[i]["rma"] = _pack([int(round(float(c) * 255.0)) for c in m["rma"]])
        out[i]["normal"] = _pack([int(round(float(c) * 255.0)) for c in m["normal"]])
        out[i]["emission"] = m["emission"]
        out[i]["ior"] = m["ior"]
        out[i]["transmission"] = m["transmission"]
    return out


class RefScene:
    def __init__(self, scene, fma: bool = True):
        self.L = lib(fma)
        s = scene.contiguous()
        self.scene = s
        self.refmats = reference_materials(s.materials)
        status = ctypes.c_int(1)
        images = None
        slots = None
        self._keep = []
        textures = getattr(s, "textures", None) or []
        if textures:
            images = np.zeros(len(textures), dtype=IMAGE_DTYPE)
            for i, t in enumerate(textures):
                data = np.asarray(t["data"])
                if data.shape[2] == 3:  # Import::ConvertRgbToRgba
                    alpha = np.full(data.shape[:2] + (1,), 255 if data.dtype == np.uint8 else 1.0, dtype=data.dtype)
                    data = np.concatenate([data, alpha], -1)
                data = np.ascontiguousarray(data)
                self._keep.append(data)
                images[i] = (data.shape[1], data.shape[0], data.shape[2], int(t["format"]), data.ctypes.data)
            slots = np.ascontiguousarray(s.material_textures, dtype=np.int32)
            self._keep += [images, slots]
        self.h = self.L.ref_scene_create(s.triangle_count, _p(s.positions), _p(s.normals), _p(s.tangents), _p(s.uvs),
                                        _p(s.material_ids), len(s.materials), _p(self.refmats), ctypes.byref(status),
                                        len(textures), _p(images) if images is not None else None,
                                        _p(slots) if slots is not None else None)
        if not self.h or status.value != 0:
            raise RuntimeError("ref_scene_create failed")

    def close(self):
        if self.h:
            self.L.ref_scene_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def info(self):
        n, d, l = np.zeros(1, np.uint32), np.zeros(1, np.uint32), np.zeros(1, np.uint32)
        self.L.ref_scene_info(self.h, _p(n), _p(d), _p(l))
        return dict(nodes=int(n[0]), depth=int(d[0]), lights=int(l[0]))

    def decoded_materials(self) -> np.ndarray:
        """Material records holding the texel values the reference kernels read from their textures."""
        import scenes
        raw = np.zeros((len(self.scene.materials), 20), dtype=np.float32)
        rc = self.L.ref_scene_decoded_materials(self.h, _p(raw))
        if rc:
            raise RuntimeError("ref_scene_decoded_materials failed")
        out = raw.view(scenes.MATERIAL_DTYPE).reshape(-1).copy()
        out["model"] = self.scene.materials["model"]
        out["pad"] = 0.0
        return out

    def trace_closest(self, rays: np.ndarray):
        rays = np.ascontiguousarray(rays, dtype=np.float32)
        tri = np.zeros(rays.shape[0], dtype=np.uint32)
        uvt = np.zeros((rays.shape[0], 3), dtype=np.float32)
        rc = self.L.ref_trace_closest(self.h, _p(rays), rays.shape[0], _p(tri), _p(uvt))
        if rc:
            raise RuntimeError(f"ref_trace_closest failed ({rc})")
        return tri, uvt

    def render(self, camera, width, height, spp, depth, nee=True, pool_size=1 << 20, log_capacity=1 << 16):
        cam = np.ascontiguousarray(camera, dtype=np.float32)
        acc = np.zeros((width * height, 4), dtype=np.float32)
        fb = np.zeros(width * height, dtype=np.uint32)
        log = np.zeros((log_capacity, 9), dtype=np.uint32)
        it = np.zeros(1, np.uint32)
        ms = np.zeros(1, np.float32)
        rc = self.L.ref_render(self.h, _p(cam), width, height, spp, depth, 1 if nee else 0, pool_size, _p(acc), _p(fb),
                              _p(log), log_capacity, _p(it), _p(ms))
        if rc:
            raise RuntimeError(f"ref_render failed ({rc})")
        n = int(it[0])
        return dict(accumulation=acc, framebuffer=fb, queue_log=log[:min(n, log_capacity)], iterations=n,
                    frame_ms=float(ms[0]))
