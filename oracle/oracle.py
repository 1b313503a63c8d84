"""ORACLE — test infrastructure only (ctypes binding of oracle/liboracle.so).

The CPU restatement of the reference path tracer (oracle/oracle.cpp). Only
tests/, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg use it,
always as the checker or the timed CPU reference, never as the product.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "liboracle.so")
_lib = None

NODE_DTYPE = np.dtype([("bmin", "<f4", 3), ("bmax", "<f4", 3), ("left", "<u4"), ("right", "<u4"),
                       ("first", "<u4"), ("count", "<u4")])
BIN_DTYPE = np.dtype([("q", "<f4"), ("p", "<f4"), ("alias", "<u4"), ("value", "<u4")])


def build() -> str:
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB):
            build()
        L = ctypes.CDLL(_LIB)
        vp, u32, i32, u64, f32 = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_int, ctypes.c_uint64, ctypes.c_float
        L.oracle_scene_create.restype = vp
        L.oracle_scene_create.argtypes = [u32, vp, vp, vp, vp, vp, u32, vp]
        L.oracle_scene_destroy.argtypes = [vp]
        L.oracle_scene_bvh_node_count.restype = u32
        L.oracle_scene_bvh_node_count.argtypes = [vp]
        L.oracle_scene_bvh_depth.restype = u32
        L.oracle_scene_bvh_depth.argtypes = [vp]
        L.oracle_scene_bvh_export.argtypes = [vp, vp, vp]
        L.oracle_scene_light_count.restype = u32
        L.oracle_scene_light_count.argtypes = [vp]
        L.oracle_scene_alias_export.argtypes = [vp, vp]
        L.oracle_trace_closest.argtypes = [vp, vp, u32, vp, vp, i32]
        L.oracle_trace_any.argtypes = [vp, vp, u32, vp, i32]
        L.oracle_alias_build.argtypes = [vp, u32, vp]
        L.oracle_alias_sample.argtypes = [vp, u32, vp, u32, vp, vp]
        L.oracle_philox_words.argtypes = [u64, u64, u32, vp, vp]
        L.oracle_sincos.argtypes = [vp, u32, vp, vp]
        L.oracle_pow.argtypes = [vp, vp, u32, vp]
        L.oracle_render.restype = i32
        L.oracle_render.argtypes = [vp, vp, u32, u32, u32, u32, u32, u32, u64, i32, i32, vp, vp, vp, vp, u32, vp, u64, u32, u32]
        L.oracle_scene_alias_power_export.argtypes = [vp, vp]
        L.oracle_power_alias_build.argtypes = [vp, vp, u32, vp]
        L.oracle_device_order_scan.argtypes = [vp, u32, vp]
        L.oracle_pcg_words.argtypes = [u64, u64, u32, vp, vp]
        L.oracle_pcg_seeded_words.argtypes = [u64, u64, u32, vp]
        L.oracle_make_camera.argtypes = [f32, f32, vp, vp, vp]
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def default_threads() -> int:
    return max(1, len(os.sched_getaffinity(0)))


class OracleScene:
    """Scene prepared the reference way: triangle records, area-weighted light
    alias table, median-split BVH (Renderer.cpp:292-306)."""

    def __init__(self, scene):
        self.scene = scene
        self._keep = (scene.positions, scene.normals, scene.tangents, scene.uvs, scene.material_ids, scene.materials)
        self.handle = lib().oracle_scene_create(scene.triangle_count, _p(scene.positions), _p(scene.normals),
                                                _p(scene.tangents), _p(scene.uvs), _p(scene.material_ids),
                                                len(scene.materials), _p(scene.materials))

    def close(self):
        if self.handle:
            lib().oracle_scene_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def bvh(self):
        n = lib().oracle_scene_bvh_node_count(self.handle)
        nodes = np.zeros(n, dtype=NODE_DTYPE)
        order = np.zeros(self.scene.triangle_count, dtype=np.uint32)
        lib().oracle_scene_bvh_export(self.handle, _p(nodes), _p(order))
        return nodes, order, lib().oracle_scene_bvh_depth(self.handle)

    def alias_table(self, power: bool = False):
        """The light alias table: area weights (the reference's), or the product's power weights."""
        n = lib().oracle_scene_light_count(self.handle)
        bins = np.zeros(n, dtype=BIN_DTYPE)
        if n:
            (lib().oracle_scene_alias_power_export if power else lib().oracle_scene_alias_export)(self.handle, _p(bins))
        return bins

    def trace_closest(self, rays: np.ndarray, threads: int | None = None):
        rays = np.ascontiguousarray(rays, dtype=np.float32)
        n = rays.shape[0]
        tri = np.zeros(n, dtype=np.uint32)
        uvt = np.zeros((n, 3), dtype=np.float32)
        lib().oracle_trace_closest(self.handle, _p(rays), n, _p(tri), _p(uvt), threads or default_threads())
        return tri, uvt

    def trace_any(self, rays: np.ndarray, threads: int | None = None):
        rays = np.ascontiguousarray(rays, dtype=np.float32)
        occ = np.zeros(rays.shape[0], dtype=np.uint8)
        lib().oracle_trace_any(self.handle, _p(rays), rays.shape[0], _p(occ), threads or default_threads())
        return occ

    def render(self, camera: np.ndarray, width: int, height: int, spp: int, depth: int, nee: bool = True,
               pool_size: int = 1 << 20, max_samples: int = 0, threads: int | None = None, accumulation: int = 1,
               log_capacity: int = 1 << 16, rng_offset: int = 0, rng_policy: int = 0, light_sampling: int = 0):
        """Replay of Renderer::RenderFrame on the CPU. accumulation: 0 = FP32 in
        sample order, 1 = FP32 Kahan in sample order, 2 = FP64. rng_policy: 0 = Philox
        (the reference's), 1 = PCG32; light_sampling: 0 = area (the reference's), 1 = power."""
        spa = int(np.sqrt(spp))
        spp_eff = spa * spa
        total = spp_eff * width * height
        if max_samples:
            total = min(total, max_samples)
        camera = np.ascontiguousarray(camera, dtype=np.float32)
        radiance = np.zeros((max(total, 1), 3), dtype=np.float32)
        accum = np.zeros((width * height, 4), dtype=np.float32)
        fb = np.zeros(width * height, dtype=np.uint32)
        qlog = np.zeros((log_capacity, 9), dtype=np.uint32)
        iters = ctypes.c_uint32(0)
        rc = lib().oracle_render(self.handle, _p(camera), width, height, spp, depth, 1 if nee else 0, pool_size,
                                 max_samples, threads or default_threads(), accumulation, _p(radiance), _p(accum),
                                 _p(fb), _p(qlog), log_capacity, ctypes.byref(iters), rng_offset, rng_policy,
                                 light_sampling)
        if rc != 0:
            raise RuntimeError(f"oracle_render failed: {rc}")
        it = iters.value
        return dict(sample_radiance=radiance[:total], accumulation=accum, framebuffer=fb,
                    queue_log=qlog[:min(it, log_capacity)], iterations=it, total_samples=total)


def alias_build(weights: np.ndarray) -> np.ndarray:
    weights = np.ascontiguousarray(weights, dtype=np.float32)
    bins = np.zeros(weights.size, dtype=BIN_DTYPE)
    lib().oracle_alias_build(_p(weights), weights.size, _p(bins))
    return bins


def alias_sample(bins: np.ndarray, u: np.ndarray):
    u = np.ascontiguousarray(u, dtype=np.float32)
    idx = np.zeros(u.size, dtype=np.uint32)
    pmf = np.zeros(u.size, dtype=np.float32)
    lib().oracle_alias_sample(_p(np.ascontiguousarray(bins)), bins.size, _p(u), u.size, _p(idx), _p(pmf))
    return idx, pmf


def philox_words(subsequence: int, position: int, count: int):
    words = np.zeros(count, dtype=np.uint32)
    uni = np.zeros(count, dtype=np.float32)
    lib().oracle_philox_words(subsequence, position, count, _p(words), _p(uni))
    return words, uni


def power_alias_build(power: np.ndarray, area: np.ndarray) -> np.ndarray:
    """The product's power-weighted alias table (parallel sweep, device-order FP64 prefix sums)."""
    power = np.ascontiguousarray(power, dtype=np.float64)
    area = np.ascontiguousarray(area, dtype=np.float64)
    bins = np.zeros(power.size, dtype=BIN_DTYPE)
    lib().oracle_power_alias_build(_p(power), _p(area), power.size, _p(bins))
    return bins


def device_order_scan(x: np.ndarray) -> np.ndarray:
    x = np.ascontiguousarray(x, dtype=np.float64)
    out = np.zeros_like(x)
    lib().oracle_device_order_scan(_p(x), x.size, _p(out))
    return out


def pcg_words(key: int, position: int, count: int):
    words = np.zeros(count, dtype=np.uint32)
    uni = np.zeros(count, dtype=np.float32)
    lib().oracle_pcg_words(key, position, count, _p(words), _p(uni))
    return words, uni


def pcg_seeded_words(initstate: int, initseq: int, count: int) -> np.ndarray:
    words = np.zeros(count, dtype=np.uint32)
    lib().oracle_pcg_seeded_words(initstate, initseq, count, _p(words))
    return words


def alias_implied_pmf(bins: np.ndarray) -> np.ndarray:
    """Probability of every outcome that an alias table encodes: (q_k + sum over bins aliasing k of
    (1 - q)) / n, in FP64. Equals the target pmf for a correct table."""
    n = bins.size
    q = bins["q"].astype(np.float64)
    out = q.copy()
    alias = bins["alias"]
    valid = alias != 0xFFFFFFFF
    np.add.at(out, alias[valid].astype(np.int64), 1.0 - q[valid])
    out[~valid] += 1.0 - q[~valid]  # leftovers keep their own outcome (q is 1 there)
    return out / n


def sincos(x: np.ndarray):
    x = np.ascontiguousarray(x, dtype=np.float32)
    s = np.zeros_like(x)
    c = np.zeros_like(x)
    lib().oracle_sincos(_p(x), x.size, _p(s), _p(c))
    return s, c


def powf(x: np.ndarray, y: np.ndarray):
    x = np.ascontiguousarray(x, dtype=np.float32)
    y = np.ascontiguousarray(y, dtype=np.float32)
    out = np.zeros_like(x)
    lib().oracle_pow(_p(x), _p(y), x.size, _p(out))
    return out


def make_camera_from_motion(fov_y: float, aspect: float, position, quat_wxyz) -> np.ndarray:
    pos = np.ascontiguousarray(position, dtype=np.float32)
    q = np.ascontiguousarray(quat_wxyz, dtype=np.float32)
    out = np.zeros(12, dtype=np.float32)
    lib().oracle_make_camera(ctypes.c_float(fov_y), ctypes.c_float(aspect), _p(pos), _p(q), _p(out))
    return out


def resample_motion(samples, interval: float):
    """Capture::ResampleMotion (Core/Source/Capture/Resampling.cpp:17-55), in float32 arithmetic:
    samples (position3, quaternion wxyz, time) at increasing times -> one state per interval from the
    first time; position by glm::mix (a (1 - t) + b t), rotation by SlerpShortest
    (Utils/Math/Interpolation.hpp: b negated onto a's hemisphere, slerp with a linear fallback when
    cos(theta) > 1 - FLT_EPSILON, then normalised)."""
    f = np.float32
    samples = [(np.asarray(p, f), np.asarray(q, f), f(t)) for p, q, t in samples]
    if not samples:
        return []
    if len(samples) == 1:
        return [(samples[0][0], samples[0][1])]

    def slerp_shortest(a, b, t):
        if f(np.dot(a, b)) < f(0):
            b = -b
        cos_theta = f(a[0] * b[0] + a[1] * b[1] + a[2] * b[2] + a[3] * b[3])
        if cos_theta > f(1) - np.finfo(f).eps:
            q = a * (f(1) - t) + b * t
        else:
            theta = np.arccos(cos_theta, dtype=f)
            q = (a * np.sin((f(1) - t) * theta, dtype=f) + b * np.sin(t * theta, dtype=f)) * (f(1) / np.sin(theta, dtype=f))
        n = np.sqrt(f(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]), dtype=f)
        return q * (f(1) / n) if n > 0 else np.array([1, 0, 0, 0], f)

    first = samples[0][2]
    out = [(samples[0][0], samples[0][1])]
    for i in range(1, len(samples)):
        (p0, q0, t0), (p1, q1, t1) = samples[i - 1], samples[i]
        while True:
            target = f(first + f(len(out)) * f(interval))
            if target > t1:
                break
            t = f((target - t0) / (t1 - t0))
            out.append((p0 * (f(1) - t) + p1 * t, slerp_shortest(q0, q1, t)))
    return out
