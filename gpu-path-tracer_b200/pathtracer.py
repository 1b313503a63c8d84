"""ctypes binding of libgpt_b200.so (include/gpt_b200.h) for tests, benchmarks and scripting.

The product is the C ABI; this module only marshals numpy arrays and torch
device tensors into it. There is no fallback: if the shared library is missing
or no CUDA device is present, the calls raise.

Two builds export the same ABI (gpu-path-tracer_b200/Makefile):
  "product"  libgpt_b200.so: the reference build's arithmetic (multiply-add contraction, CUDA's
             sinf/cosf/powf/rsqrtf); what bench.py measures.
  "det"      libgpt_b200_det.so: no contraction and IEEE definitions of the transcendentals, so
             results are reproducible bit for bit by the CPU oracle.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgpt_b200.so")
LIB_PATHS = {"product": LIB_PATH, "det": os.path.join(HERE, "libgpt_b200_det.so")}
QUEUE_LOG_COLUMNS = 9
INVALID = 0xFFFFFFFF

_libs = {}


class GptError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"{message} (status {code})")
        self.code = code


class gpt_material(ctypes.Structure):
    _fields_ = [("model", ctypes.c_uint32), ("color", ctypes.c_float * 3), ("specular", ctypes.c_float * 3),
                ("shininess", ctypes.c_float), ("rma", ctypes.c_float * 3), ("emission", ctypes.c_float * 3),
                ("normal", ctypes.c_float * 3), ("ior", ctypes.c_float), ("transmission", ctypes.c_float),
                ("reserved", ctypes.c_float)]


class gpt_texture_desc(ctypes.Structure):
    _fields_ = [("width", ctypes.c_uint32), ("height", ctypes.c_uint32), ("channels", ctypes.c_uint32),
                ("format", ctypes.c_uint32), ("data", ctypes.c_void_p)]


class gpt_scene_desc(ctypes.Structure):
    _fields_ = [("triangle_count", ctypes.c_uint32), ("positions", ctypes.c_void_p), ("normals", ctypes.c_void_p),
                ("tangents", ctypes.c_void_p), ("uvs", ctypes.c_void_p), ("material_ids", ctypes.c_void_p),
                ("material_count", ctypes.c_uint32), ("materials", ctypes.c_void_p), ("texture_count", ctypes.c_uint32),
                ("textures", ctypes.c_void_p), ("material_textures", ctypes.c_void_p)]


TEXEL_U8_SRGB, TEXEL_U8_LINEAR, TEXEL_F32 = 0, 1, 2


class gpt_device_camera(ctypes.Structure):
    _fields_ = [("origin", ctypes.c_float * 3), ("lower_left", ctypes.c_float * 3),
                ("horizontal", ctypes.c_float * 3), ("vertical", ctypes.c_float * 3)]


class gpt_motion_state(ctypes.Structure):
    _fields_ = [("position", ctypes.c_float * 3), ("rotation", ctypes.c_float * 4)]


class gpt_motion_sample(ctypes.Structure):
    _fields_ = [("state", gpt_motion_state), ("time", ctypes.c_float)]


class gpt_render_settings(ctypes.Structure):
    _fields_ = [("width", ctypes.c_uint32), ("height", ctypes.c_uint32), ("samples_per_pixel", ctypes.c_uint32),
                ("path_depth", ctypes.c_uint32), ("use_nee", ctypes.c_uint32), ("pool_size", ctypes.c_uint32),
                ("max_samples", ctypes.c_uint64), ("trace_block", ctypes.c_uint32), ("trace_refill", ctypes.c_uint32),
                ("rng_offset", ctypes.c_uint64), ("loop_mode", ctypes.c_uint32), ("trace_occupancy", ctypes.c_uint32),
                ("bvh_format", ctypes.c_uint32), ("wavefront_layout", ctypes.c_uint32), ("rng_policy", ctypes.c_uint32),
                ("light_sampling", ctypes.c_uint32), ("max_iterations", ctypes.c_uint32), ("trace_stack", ctypes.c_uint32)]

LOOP_GRAPH, LOOP_HOST = 0, 1
RNG_PHILOX, RNG_PCG32 = 0, 1
LIGHTS_AREA, LIGHTS_POWER = 0, 1
BVH8_Q8, BVH2_FP32 = 0, 1
BVH_BUILD_HOST, BVH_BUILD_DEVICE = 0, 1
WAVEFRONT_B200, WAVEFRONT_QUEUES = 0, 1
SCHEDULE_SHORTEST_FIRST, SCHEDULE_OLDEST_FIRST, SCHEDULE_DEADLINE, SCHEDULE_TWO_CLASS = 1, 2, 3, 4
NODE_BYTES = {BVH8_Q8: 64 + 4, BVH2_FP32: 64}  # bytes a node visit reads: BVH8 header + its child reference; the whole binary node


class gpt_frame_stats(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_uint32), ("kernel_launches", ctypes.c_uint32), ("samples", ctypes.c_uint64),
                ("rays", ctypes.c_uint64), ("shadow_rays", ctypes.c_uint64), ("node_visits", ctypes.c_uint64 * 2),
                ("triangle_tests", ctypes.c_uint64 * 2), ("device_ms", ctypes.c_float), ("phase_ms", ctypes.c_float * 4),
                ("trace_event_ms", ctypes.c_float)]

PHASES = ("trace", "shade", "shadow", "regen")


class gpt_server_config(ctypes.Structure):
    _fields_ = [("pool_size", ctypes.c_uint32), ("max_jobs", ctypes.c_uint32), ("max_active_jobs", ctypes.c_uint32),
                ("ring_passes", ctypes.c_uint32), ("hbm_budget_bytes", ctypes.c_uint64), ("trace_block", ctypes.c_uint32),
                ("trace_refill", ctypes.c_uint32), ("trace_occupancy", ctypes.c_uint32),
                ("max_slice_iterations", ctypes.c_uint32), ("schedule", ctypes.c_uint32), ("deadline_slowdown", ctypes.c_float),
                ("short_job_seconds", ctypes.c_float), ("bvh_build", ctypes.c_uint32)]


class gpt_job_desc(ctypes.Structure):
    _fields_ = [("scene", ctypes.c_uint32), ("width", ctypes.c_uint32), ("height", ctypes.c_uint32),
                ("samples_per_pixel", ctypes.c_uint32), ("path_depth", ctypes.c_uint32), ("use_nee", ctypes.c_uint32),
                ("rng_offset", ctypes.c_uint64), ("camera", gpt_device_camera), ("keep_accumulation", ctypes.c_uint32),
                ("rng_policy", ctypes.c_uint32), ("light_sampling", ctypes.c_uint32), ("reserved", ctypes.c_uint32)]


class gpt_job_status(ctypes.Structure):
    _fields_ = [("state", ctypes.c_uint32), ("passes_done", ctypes.c_uint32), ("passes_total", ctypes.c_uint32),
                ("reserved", ctypes.c_uint32), ("samples_total", ctypes.c_uint64), ("admitted_bytes", ctypes.c_uint64),
                ("submit_s", ctypes.c_double), ("admit_s", ctypes.c_double), ("done_s", ctypes.c_double)]


class gpt_server_stats(ctypes.Structure):
    _fields_ = [("slices", ctypes.c_uint64), ("iterations", ctypes.c_uint64), ("samples", ctypes.c_uint64),
                ("rays", ctypes.c_uint64), ("shadow_rays", ctypes.c_uint64), ("admitted_bytes", ctypes.c_uint64),
                ("admitted_high_water", ctypes.c_uint64), ("budget_bytes", ctypes.c_uint64),
                ("active_jobs", ctypes.c_uint32), ("queued_jobs", ctypes.c_uint32), ("completed_jobs", ctypes.c_uint32),
                ("scenes", ctypes.c_uint32), ("device_ms", ctypes.c_double), ("phase_ms", ctypes.c_float * 4)]


JOB_QUEUED, JOB_RUNNING, JOB_DONE, JOB_CANCELLED, JOB_FAILED = 0, 1, 2, 3, 4
JOB_STATES = ("queued", "running", "done", "cancelled", "failed")


# (name, restype, argtypes) of every C entry point in include/gpt_b200.h
_SIGNATURES = [
    ("gpt_status_string", ctypes.c_char_p, [ctypes.c_int]),
    ("gpt_create", ctypes.c_int, [ctypes.POINTER(ctypes.c_void_p), ctypes.c_int]),
    ("gpt_destroy", None, [ctypes.c_void_p]),
    ("gpt_init_rendering_buffers", ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32]),
    ("gpt_init_scene_buffers", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(gpt_scene_desc)]),
    ("gpt_clear", ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint8, ctypes.c_uint8, ctypes.c_uint8, ctypes.c_uint8]),
    ("gpt_start_simulation", ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_float,
                                            ctypes.POINTER(gpt_motion_state), ctypes.c_uint32, ctypes.c_uint32,
                                            ctypes.c_uint32, ctypes.c_char_p, ctypes.c_int]),
    ("gpt_resume_simulation", ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint32]),
    ("gpt_stop_rendering", ctypes.c_int, [ctypes.c_void_p]),
    ("gpt_is_rendering", ctypes.c_int, [ctypes.c_void_p]),
    ("gpt_get_done_frames", ctypes.c_uint32, [ctypes.c_void_p]),
    ("gpt_get_total_frames", ctypes.c_uint32, [ctypes.c_void_p]),
    ("gpt_get_done_samples", ctypes.c_uint64, [ctypes.c_void_p]),
    ("gpt_get_total_samples", ctypes.c_uint64, [ctypes.c_void_p]),
    ("gpt_get_width", ctypes.c_uint32, [ctypes.c_void_p]),
    ("gpt_get_height", ctypes.c_uint32, [ctypes.c_void_p]),
    ("gpt_lock_frame", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_size_t),
                                      ctypes.POINTER(ctypes.c_size_t)]),
    ("gpt_unlock_frame", ctypes.c_int, [ctypes.c_void_p]),
    ("gpt_peek_last_error", ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_size_t]),
    ("gpt_consume_last_error", ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_size_t]),
    ("gpt_render_frame", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(gpt_device_camera),
                                        ctypes.POINTER(gpt_render_settings), ctypes.POINTER(gpt_frame_stats)]),
    ("gpt_autotune", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(gpt_device_camera), ctypes.POINTER(gpt_render_settings),
                                    ctypes.POINTER(gpt_render_settings), ctypes.POINTER(ctypes.c_float),
                                    ctypes.POINTER(ctypes.c_uint32)]),
    ("gpt_read_framebuffer", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t]),
    ("gpt_read_accumulation", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t]),
    ("gpt_read_sample_radiance", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64]),
    ("gpt_copy_accumulation_device", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p]),
    ("gpt_read_accumulation_fp64", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t]),
    ("gpt_read_queue_log", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32,
                                          ctypes.POINTER(ctypes.c_uint32)]),
    ("gpt_intersect_closest", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p,
                                             ctypes.c_void_p, ctypes.c_void_p]),
    ("gpt_intersect_any", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p,
                                         ctypes.c_void_p]),
    ("gpt_intersect_closest_binary", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p,
                                                    ctypes.c_void_p, ctypes.c_void_p]),
    ("gpt_intersect_any_binary", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p,
                                                ctypes.c_void_p]),
    ("gpt_scene_info", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(ctypes.c_uint32),
                                      ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(ctypes.c_uint32)]),
    ("gpt_scene_info_binary", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint32),
                                             ctypes.POINTER(ctypes.c_uint32)]),
    ("gpt_scene_upload_times", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double),
                                              ctypes.POINTER(ctypes.c_double)]),
    ("gpt_set_bvh_build", ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint32]),
    ("gpt_check_bvh", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32, ctypes.POINTER(ctypes.c_uint64),
                                     ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64)]),
    ("gpt_read_alias_table", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32]),
    ("gpt_read_alias_table_power", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32]),
    ("gpt_inject_allocation_failure", ctypes.c_int, [ctypes.c_uint32]),
    ("gpt_bvh8_check", ctypes.c_int, [ctypes.POINTER(gpt_scene_desc), ctypes.POINTER(ctypes.c_uint32),
                                      ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(ctypes.c_uint64),
                                      ctypes.POINTER(ctypes.c_uint64)]),
    ("gpt_build_alias_table_noalloc", ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p]),
    ("gpt_generate_tangents", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32,
                                             ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p]),
    ("gpt_obj_load", ctypes.c_int, [ctypes.c_char_p, ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)]),
    ("gpt_obj_scene_desc", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(gpt_scene_desc)]),
    ("gpt_obj_material_name", ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_char_p, ctypes.c_size_t]),
    ("gpt_obj_free", None, [ctypes.c_void_p]),
    ("gpt_abi_struct_sizes", ctypes.c_int, [ctypes.POINTER(ctypes.c_uint32), ctypes.c_uint32]),
    ("gpt_make_device_camera", ctypes.c_int, [ctypes.c_float, ctypes.c_float, ctypes.POINTER(gpt_motion_state),
                                              ctypes.POINTER(gpt_device_camera)]),
    ("gpt_resample_motion", ctypes.c_int, [ctypes.POINTER(gpt_motion_sample), ctypes.c_uint32, ctypes.c_float,
                                           ctypes.POINTER(gpt_motion_state), ctypes.c_uint32, ctypes.POINTER(ctypes.c_uint32)]),
    ("gpt_server_create", ctypes.c_int, [ctypes.POINTER(ctypes.c_void_p), ctypes.c_int, ctypes.POINTER(gpt_server_config)]),
    ("gpt_server_destroy", ctypes.c_int, [ctypes.c_void_p]),
    ("gpt_server_add_scene", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(gpt_scene_desc), ctypes.POINTER(ctypes.c_uint32)]),
    ("gpt_server_submit", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(gpt_job_desc), ctypes.POINTER(ctypes.c_uint64)]),
    ("gpt_server_poll", ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, ctypes.POINTER(gpt_job_status)]),
    ("gpt_server_wait", ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_double]),
    ("gpt_server_read", ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p, ctypes.c_void_p]),
    ("gpt_server_release", ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64]),
    ("gpt_server_cancel", ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64]),
    ("gpt_server_set_loop_mode", ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint32]),
    ("gpt_server_get_stats", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(gpt_server_stats)]),
    ("gpt_server_peek_last_error", ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_size_t]),
]


def build(verbose: bool = False) -> str:
    """Compile both library builds for sm_100a (nvcc cross-compiles without a GPU)."""
    subprocess.run(["make", "-C", HERE] + ([] if verbose else ["-s"]), check=True)
    return LIB_PATH


def lib(variant: str = "product"):
    """The loaded library of one build: "product" (libgpt_b200.so) or "det" (libgpt_b200_det.so)."""
    if variant not in LIB_PATHS:
        raise ValueError(f"unknown library build {variant!r}; expected one of {sorted(LIB_PATHS)}")
    if variant not in _libs:
        path = LIB_PATHS[variant]
        if not os.path.exists(path):
            raise GptError(-1, f"{path} is missing: run `make -C {HERE}` (or __graft_entry__.build())")
        L = ctypes.CDLL(path)
        for name, res, args in _SIGNATURES:
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _libs[variant] = L
    return _libs[variant]


def declared_symbols() -> list[str]:
    return [s[0] for s in _SIGNATURES]


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def camera_struct(camera12) -> gpt_device_camera:
    c = np.asarray(camera12, dtype=np.float32).reshape(12)
    cam = gpt_device_camera()
    for k in range(3):
        cam.origin[k] = c[k]
        cam.lower_left[k] = c[3 + k]
        cam.horizontal[k] = c[6 + k]
        cam.vertical[k] = c[9 + k]
    return cam


class Renderer:
    """Handle on one gpt_renderer (one device, one render stream)."""

    def __init__(self, device: int = 0, variant: str = "product"):
        self.L = lib(variant)
        self.variant = variant
        h = ctypes.c_void_p()
        rc = self.L.gpt_create(ctypes.byref(h), device)
        if rc != 0:
            raise GptError(rc, f"gpt_create(device={device}) failed: {self.L.gpt_status_string(rc).decode()}")
        self.h = h
        self._scene_keep = None

    def close(self):
        if getattr(self, "h", None):
            self.L.gpt_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc: int, what: str):
        if rc != 0:
            buf = ctypes.create_string_buffer(1024)
            self.L.gpt_consume_last_error(self.h, buf, 1024)
            raise GptError(rc, f"{what}: {buf.value.decode() or self.L.gpt_status_string(rc).decode()}")

    def last_error(self, consume: bool = False) -> str | None:
        buf = ctypes.create_string_buffer(1024)
        fn = self.L.gpt_consume_last_error if consume else self.L.gpt_peek_last_error
        return buf.value.decode() if fn(self.h, buf, 1024) else None

    def init_rendering_buffers(self, width: int, height: int):
        self._check(self.L.gpt_init_rendering_buffers(self.h, width, height), "gpt_init_rendering_buffers")

    def upload_scene(self, scene):
        desc, keep = scene_desc_with_textures(scene)
        self._scene_keep = keep
        self._check(self.L.gpt_init_scene_buffers(self.h, ctypes.byref(desc)), "gpt_init_scene_buffers")

    def scene_info(self) -> dict:
        n, d, l, t = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint32()
        self._check(self.L.gpt_scene_info(self.h, ctypes.byref(n), ctypes.byref(d), ctypes.byref(l), ctypes.byref(t)),
                    "gpt_scene_info")
        n2, d2 = ctypes.c_uint32(), ctypes.c_uint32()
        self._check(self.L.gpt_scene_info_binary(self.h, ctypes.byref(n2), ctypes.byref(d2)), "gpt_scene_info_binary")
        return dict(nodes=n.value, depth=d.value, lights=l.value, triangles=t.value, binary_nodes=n2.value,
                    binary_depth=d2.value)

    def upload_times(self) -> dict:
        """Seconds of the last upload: the BVH build (host or device), and the whole upload."""
        b, u = ctypes.c_double(), ctypes.c_double()
        self._check(self.L.gpt_scene_upload_times(self.h, ctypes.byref(b), ctypes.byref(u)), "gpt_scene_upload_times")
        return dict(bvh_build_s=b.value, upload_s=u.value)

    def set_bvh_build(self, build: int):
        """Where the next upload_scene builds the BVH8: BVH_BUILD_HOST (default) or BVH_BUILD_DEVICE."""
        self._check(self.L.gpt_set_bvh_build(self.h, build), "gpt_set_bvh_build")

    def check_bvh(self, scene) -> dict:
        """Host check of the uploaded BVH8 against the scene's positions (gpt_check_bvh)."""
        pos = np.ascontiguousarray(scene.positions, dtype=np.float32)
        a, b, c = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
        self._check(self.L.gpt_check_bvh(self.h, _ptr(pos), pos.shape[0], ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)),
                    "gpt_check_bvh")
        return dict(containment_violations=a.value, triangles_not_exactly_once=b.value, leaf_triangles=c.value)

    def alias_table(self, power: bool = False) -> np.ndarray:
        """[lights, 4] words (q, p, alias, value): the area-weighted table, or with power=True the
        power-weighted one."""
        lights = self.scene_info()["lights"]
        out = np.zeros((lights, 4), dtype=np.uint32)
        if lights:
            fn = self.L.gpt_read_alias_table_power if power else self.L.gpt_read_alias_table
            self._check(fn(self.h, _ptr(out), lights), "gpt_read_alias_table")
        return out

    def render_frame(self, camera12, width: int, height: int, spp: int, depth: int, nee: bool = True,
                     pool_size: int = 0, max_samples: int = 0, trace_block: int = 0, trace_refill: int = 0,
                     rng_offset: int = 0, loop_mode: int = LOOP_GRAPH, trace_occupancy: int = 0,
                     bvh_format: int = BVH8_Q8, wavefront_layout: int = WAVEFRONT_B200, rng_policy: int = RNG_PHILOX,
                     light_sampling: int = LIGHTS_AREA, max_iterations: int = 0, trace_stack: int = 0) -> dict:
        cam = camera_struct(camera12)
        st = gpt_render_settings(width, height, spp, depth, 1 if nee else 0, pool_size, max_samples, trace_block,
                                 trace_refill, rng_offset, loop_mode, trace_occupancy, bvh_format, wavefront_layout,
                                 rng_policy, light_sampling, max_iterations, trace_stack)
        stats = gpt_frame_stats()
        self._check(self.L.gpt_render_frame(self.h, ctypes.byref(cam), ctypes.byref(st), ctypes.byref(stats)),
                    "gpt_render_frame")
        self.width, self.height = width, height
        spa = int(np.sqrt(spp))
        total = spa * spa * width * height
        self.total_samples = min(total, max_samples) if max_samples else total
        return dict(iterations=stats.iterations, kernel_launches=stats.kernel_launches, samples=stats.samples,
                    rays=stats.rays, shadow_rays=stats.shadow_rays, node_visits=list(stats.node_visits),
                    triangle_tests=list(stats.triangle_tests), device_ms=stats.device_ms,
                    phase_ms={k: stats.phase_ms[i] for i, k in enumerate(PHASES)}, trace_event_ms=stats.trace_event_ms)

    def autotune(self, camera12, width: int, height: int, spp: int, depth: int, nee: bool = True) -> dict:
        """Measured tuning knobs for this workload: pool_size, trace_occupancy, trace_refill, trace_block."""
        cam = camera_struct(camera12)
        base = gpt_render_settings(width, height, spp, depth, 1 if nee else 0, 0, 0, 0, 0, 0, LOOP_GRAPH, 0, BVH8_Q8, 0)
        best = gpt_render_settings()
        ms = ctypes.c_float()
        n = ctypes.c_uint32()
        self._check(self.L.gpt_autotune(self.h, ctypes.byref(cam), ctypes.byref(base), ctypes.byref(best), ctypes.byref(ms),
                                        ctypes.byref(n)), "gpt_autotune")
        return dict(pool_size=best.pool_size, trace_occupancy=best.trace_occupancy, trace_refill=best.trace_refill,
                    trace_block=best.trace_block, trial_ms=ms.value, candidates=n.value)

    def framebuffer(self) -> np.ndarray:
        out = np.zeros(self.width * self.height, dtype=np.uint32)
        self._check(self.L.gpt_read_framebuffer(self.h, _ptr(out), out.size), "gpt_read_framebuffer")
        return out

    def accumulation(self) -> np.ndarray:
        out = np.zeros((self.width * self.height, 4), dtype=np.float32)
        self._check(self.L.gpt_read_accumulation(self.h, _ptr(out), self.width * self.height), "gpt_read_accumulation")
        return out

    def accumulation_fp64(self) -> np.ndarray:
        """[pixels, 3] float64: the last frame's samples summed per pixel in FP64 on the device."""
        out = np.zeros((self.width * self.height, 3), dtype=np.float64)
        self._check(self.L.gpt_read_accumulation_fp64(self.h, _ptr(out), self.width * self.height), "gpt_read_accumulation_fp64")
        return out

    def copy_accumulation_to(self, dst_dev, stream=None):
        """The last frame's [pixels, 4] float32 accumulation into a device tensor of the same GPU."""
        self._check(self.L.gpt_copy_accumulation_device(self.h, ctypes.c_void_p(dst_dev.data_ptr()), self.width * self.height,
                                                        ctypes.c_void_p(stream)), "gpt_copy_accumulation_device")

    def sample_radiance(self) -> np.ndarray:
        out = np.zeros((self.total_samples, 3), dtype=np.float32)
        self._check(self.L.gpt_read_sample_radiance(self.h, _ptr(out), self.total_samples), "gpt_read_sample_radiance")
        return out

    def queue_log(self, max_rows: int = 1 << 16) -> np.ndarray:
        out = np.zeros((max_rows, QUEUE_LOG_COLUMNS), dtype=np.uint32)
        n = ctypes.c_uint32()
        self._check(self.L.gpt_read_queue_log(self.h, _ptr(out), max_rows, ctypes.byref(n)), "gpt_read_queue_log")
        return out[:n.value]

    def clear(self, r: int, g: int, b: int, a: int):
        self._check(self.L.gpt_clear(self.h, r, g, b, a), "gpt_clear")

    def lock_frame(self) -> np.ndarray:
        """Copy of the host frame taken under the frame lock (GetFrameView().Lock())."""
        data = ctypes.c_void_p()
        size = ctypes.c_size_t()
        elem = ctypes.c_size_t()
        self._check(self.L.gpt_lock_frame(self.h, ctypes.byref(data), ctypes.byref(size), ctypes.byref(elem)),
                    "gpt_lock_frame")
        try:
            buf = (ctypes.c_uint32 * size.value).from_address(data.value) if size.value else []
            return np.array(buf, dtype=np.uint32)
        finally:
            self.L.gpt_unlock_frame(self.h)

    # -- ray batches on device memory (torch tensors as plumbing) --
    def intersect_closest(self, rays_dev, tri_dev, uvt_dev, stream=None, bvh_format: int = BVH8_Q8):
        n = rays_dev.shape[0]
        name = "gpt_intersect_closest_binary" if bvh_format == BVH2_FP32 else "gpt_intersect_closest"
        self._check(getattr(self.L, name)(self.h, ctypes.c_void_p(rays_dev.data_ptr()), n,
                                          ctypes.c_void_p(tri_dev.data_ptr()), ctypes.c_void_p(uvt_dev.data_ptr()),
                                          ctypes.c_void_p(stream)), name)

    def intersect_any(self, rays_dev, occ_dev, stream=None, bvh_format: int = BVH8_Q8):
        n = rays_dev.shape[0]
        name = "gpt_intersect_any_binary" if bvh_format == BVH2_FP32 else "gpt_intersect_any"
        self._check(getattr(self.L, name)(self.h, ctypes.c_void_p(rays_dev.data_ptr()), n,
                                          ctypes.c_void_p(occ_dev.data_ptr()), ctypes.c_void_p(stream)), name)

    def trace_closest_np(self, rays: np.ndarray, bvh_format: int = BVH8_Q8):
        """Closest hits of a host ray batch [n, 8]: returns (tri [n] uint32, uvt [n, 3] float32)."""
        import torch
        r = torch.from_numpy(np.ascontiguousarray(rays, dtype=np.float32)).cuda()
        tri = torch.empty(rays.shape[0], dtype=torch.int32, device="cuda")
        uvt = torch.empty((rays.shape[0], 3), dtype=torch.float32, device="cuda")
        torch.cuda.synchronize()
        self.intersect_closest(r, tri, uvt, bvh_format=bvh_format)
        return tri.cpu().numpy().view(np.uint32), uvt.cpu().numpy()

    def trace_any_np(self, rays: np.ndarray, bvh_format: int = BVH8_Q8):
        import torch
        r = torch.from_numpy(np.ascontiguousarray(rays, dtype=np.float32)).cuda()
        occ = torch.empty(rays.shape[0], dtype=torch.uint8, device="cuda")
        torch.cuda.synchronize()
        self.intersect_any(r, occ, bvh_format=bvh_format)
        return occ.cpu().numpy()

    # -- asynchronous simulation (StartSimulation / StopRendering / ResumeSimulation) --
    def start_simulation(self, width, height, fov_y, motion_states, spp, depth, output_folder=None, nee=True):
        arr = (gpt_motion_state * len(motion_states))()
        for i, (pos, quat) in enumerate(motion_states):
            for k in range(3):
                arr[i].position[k] = pos[k]
            for k in range(4):
                arr[i].rotation[k] = quat[k]
        self._motion_keep = arr
        folder = output_folder.encode() if output_folder else None
        self._check(self.L.gpt_start_simulation(self.h, width, height, fov_y, arr, len(motion_states), spp, depth, folder,
                                                1 if nee else 0), "gpt_start_simulation")
        self.width, self.height = width, height

    def resume_simulation(self, start_frame: int):
        self._check(self.L.gpt_resume_simulation(self.h, start_frame), "gpt_resume_simulation")

    def stop_rendering(self):
        self._check(self.L.gpt_stop_rendering(self.h), "gpt_stop_rendering")

    def is_rendering(self) -> bool:
        return bool(self.L.gpt_is_rendering(self.h))

    def progress(self) -> dict:
        return dict(done_frames=self.L.gpt_get_done_frames(self.h), total_frames=self.L.gpt_get_total_frames(self.h),
                    done_samples=self.L.gpt_get_done_samples(self.h), total_samples=self.L.gpt_get_total_samples(self.h))


def scene_desc_with_textures(scene):
    """gpt_scene_desc of a scenes.Scene plus the objects that must stay alive while it is used."""
    s = scene.contiguous()
    keep = [s]
    desc = gpt_scene_desc(s.triangle_count, _ptr(s.positions).value, _ptr(s.normals).value, _ptr(s.tangents).value,
                          _ptr(s.uvs).value, _ptr(s.material_ids).value, len(s.materials), _ptr(s.materials).value,
                          0, None, None)
    textures = getattr(s, "textures", None) or []
    if textures:
        arr = (gpt_texture_desc * len(textures))()
        for i, t in enumerate(textures):
            data = np.ascontiguousarray(t["data"])
            keep.append(data)
            h, w, c = data.shape
            arr[i] = gpt_texture_desc(w, h, c, int(t["format"]), _ptr(data).value)
        slots = np.ascontiguousarray(s.material_textures, dtype=np.int32)
        keep += [arr, slots]
        desc.texture_count = len(textures)
        desc.textures = ctypes.cast(arr, ctypes.c_void_p)
        desc.material_textures = _ptr(slots).value
    return desc, keep


def scene_desc(scene) -> gpt_scene_desc:
    return scene_desc_with_textures(scene)[0]


def abi_struct_sizes() -> dict:
    """sizeof() of the public structs as compiled into the library."""
    names = ["gpt_material", "gpt_scene_desc", "gpt_device_camera", "gpt_motion_state", "gpt_render_settings",
             "gpt_frame_stats", "gpt_texture_desc", "gpt_server_config", "gpt_job_desc", "gpt_job_status",
             "gpt_server_stats", "gpt_motion_sample"]
    out = (ctypes.c_uint32 * len(names))()
    lib().gpt_abi_struct_sizes(out, len(names))
    return {n: out[i] for i, n in enumerate(names)}


def resample_motion(samples, interval: float):
    """Recorded camera path -> one (position, quaternion wxyz) state per frame (gpt_resample_motion).
    samples: iterable of (position3, quaternion4 wxyz, time)."""
    samples = list(samples)
    arr = (gpt_motion_sample * max(1, len(samples)))()
    for i, (pos, quat, t) in enumerate(samples):
        for k in range(3):
            arr[i].state.position[k] = pos[k]
        for k in range(4):
            arr[i].state.rotation[k] = quat[k]
        arr[i].time = t
    n = ctypes.c_uint32()
    rc = lib().gpt_resample_motion(arr, len(samples), ctypes.c_float(interval), None, 0, ctypes.byref(n))
    if rc not in (0, 6):
        raise GptError(rc, "gpt_resample_motion")
    out = (gpt_motion_state * max(1, n.value))()
    rc = lib().gpt_resample_motion(arr, len(samples), ctypes.c_float(interval), out, n.value, ctypes.byref(n))
    if rc != 0:
        raise GptError(rc, "gpt_resample_motion")
    return [(tuple(out[i].position), tuple(out[i].rotation)) for i in range(n.value)]


def bvh8_check(scene) -> dict:
    """Host-only structural validation of the BVH8 builder (no GPU needed)."""
    desc = scene_desc(scene)
    n, d = ctypes.c_uint32(), ctypes.c_uint32()
    v, m = ctypes.c_uint64(), ctypes.c_uint64()
    rc = lib().gpt_bvh8_check(ctypes.byref(desc), ctypes.byref(n), ctypes.byref(d), ctypes.byref(v), ctypes.byref(m))
    if rc != 0:
        raise GptError(rc, "gpt_bvh8_check")
    return dict(nodes=n.value, depth=d.value, violations=v.value, misplaced=m.value)


def build_alias_table_noalloc(weights_dev, bins_dev, stream=None, variant: str = "product") -> int:
    """Allocation-free alias-table build on device tensors: float32 weights [n] in, 4-byte bins [n, 4] out.

    Both tensors must be contiguous CUDA tensors on the same device, with bins 16-byte aligned (the
    kernel stores whole 16-byte bins). The build is ordered on `stream` (a cudaStream_t handle as an
    int), by default torch's current stream on the tensors' device. Returns the C status code.
    """
    import torch
    if weights_dev.dtype != torch.float32 or weights_dev.dim() != 1:
        raise ValueError("weights must be a 1-D float32 tensor")
    n = int(weights_dev.shape[0])
    if bins_dev.dtype not in (torch.int32, torch.uint32) or tuple(bins_dev.shape) != (n, 4):
        raise ValueError(f"bins must be an int32/uint32 tensor of shape ({n}, 4)")
    if not (weights_dev.is_cuda and bins_dev.is_cuda) or weights_dev.device != bins_dev.device:
        raise ValueError("weights and bins must be CUDA tensors on the same device")
    if not (weights_dev.is_contiguous() and bins_dev.is_contiguous()):
        raise ValueError("weights and bins must be contiguous")
    if bins_dev.data_ptr() % 16 != 0:
        raise ValueError("bins must be 16-byte aligned")
    if stream is None:
        stream = torch.cuda.current_stream(weights_dev.device).cuda_stream
    with torch.cuda.device(weights_dev.device):
        return lib(variant).gpt_build_alias_table_noalloc(ctypes.c_void_p(weights_dev.data_ptr()), n,
                                                          ctypes.c_void_p(bins_dev.data_ptr()), ctypes.c_void_p(stream))


def generate_tangents(positions, normals, uvs, indices) -> np.ndarray:
    """[V, 4] tangents (xyz, sign) of an indexed mesh by Mikkelsen's method (gpt_generate_tangents)."""
    p = np.ascontiguousarray(positions, dtype=np.float32).reshape(-1, 3)
    n = np.ascontiguousarray(normals, dtype=np.float32).reshape(-1, 3)
    t = np.ascontiguousarray(uvs, dtype=np.float32).reshape(-1, 2)
    i = np.ascontiguousarray(indices, dtype=np.uint32).reshape(-1, 3)
    out = np.zeros((p.shape[0], 4), dtype=np.float32)
    rc = lib().gpt_generate_tangents(_ptr(p), _ptr(n), _ptr(t), p.shape[0], _ptr(i), i.shape[0], _ptr(out))
    if rc != 0:
        raise GptError(rc, "gpt_generate_tangents")
    return out


def load_obj(path: str, transform=None):
    """OBJ/MTL file -> scenes.Scene (world-space triangles, materials encoded as texels, texture maps
    decoded into scene.textures / scene.material_textures)."""
    import scenes
    L = lib()
    h = ctypes.c_void_p()
    t = None
    if transform is not None:
        t = np.ascontiguousarray(np.asarray(transform, dtype=np.float32).reshape(4, 4).T)  # row-major in, column-major out
    rc = L.gpt_obj_load(path.encode(), _ptr(t) if t is not None else None, ctypes.byref(h))
    if rc != 0:
        raise GptError(rc, f"gpt_obj_load({path})")
    try:
        d = gpt_scene_desc()
        L.gpt_obj_scene_desc(h, ctypes.byref(d))
        n, m = d.triangle_count, d.material_count

        def arr(ptr, count, dtype):
            return np.ctypeslib.as_array(ctypes.cast(ptr, ctypes.POINTER(dtype)), shape=(count,)).copy()
        pos = arr(d.positions, n * 9, ctypes.c_float).reshape(n, 3, 3)
        nrm = arr(d.normals, n * 9, ctypes.c_float).reshape(n, 3, 3)
        tan = arr(d.tangents, n * 12, ctypes.c_float).reshape(n, 3, 4)
        uv = arr(d.uvs, n * 6, ctypes.c_float).reshape(n, 3, 2)
        mid = arr(d.material_ids, n, ctypes.c_uint32)
        raw = np.ctypeslib.as_array(ctypes.cast(d.materials, ctypes.POINTER(ctypes.c_uint8)), shape=(m * 80,)).copy()
        mats = raw.view(scenes.MATERIAL_DTYPE).copy()
        names = []
        for i in range(m):
            buf = ctypes.create_string_buffer(256)
            L.gpt_obj_material_name(h, i, buf, 256)
            names.append(buf.value.decode())
        s = scenes.Scene(pos, nrm, tan, uv, mid, mats, name=os.path.basename(path)).contiguous()
        s.material_names = names
        if d.texture_count:
            descs = ctypes.cast(d.textures, ctypes.POINTER(gpt_texture_desc))
            for i in range(d.texture_count):
                t = descs[i]
                count = t.width * t.height * t.channels
                data = np.ctypeslib.as_array(ctypes.cast(t.data, ctypes.POINTER(ctypes.c_uint8)), shape=(count,)).copy()
                s.textures.append(dict(data=data.reshape(t.height, t.width, t.channels), format=int(t.format)))
            s.material_textures = arr(d.material_textures, m * 6, ctypes.c_int32).reshape(m, 6)
        return s
    finally:
        L.gpt_obj_free(h)


def make_device_camera(fov_y: float, aspect: float, position, quat_wxyz) -> np.ndarray:
    st = gpt_motion_state()
    for k in range(3):
        st.position[k] = position[k]
    for k in range(4):
        st.rotation[k] = quat_wxyz[k]
    cam = gpt_device_camera()
    rc = lib().gpt_make_device_camera(fov_y, aspect, ctypes.byref(st), ctypes.byref(cam))
    if rc != 0:
        raise GptError(rc, "gpt_make_device_camera")
    return np.array(list(cam.origin) + list(cam.lower_left) + list(cam.horizontal) + list(cam.vertical), dtype=np.float32)


class Server:
    """Handle on one gpt_server: resident scenes, submitted jobs rendered together on one device."""

    def __init__(self, device: int = 0, pool_size: int = 0, max_jobs: int = 0, max_active_jobs: int = 0,
                 ring_passes: int = 0, hbm_budget_bytes: int = 0, trace_block: int = 0, trace_refill: int = 0,
                 trace_occupancy: int = 0, max_slice_iterations: int = 0, schedule: int = 0, deadline_slowdown: float = 0.0,
                 short_job_seconds: float = 0.0, bvh_build: int = 0,
                 variant: str = "product"):
        self.L = lib(variant)
        cfg = gpt_server_config(pool_size, max_jobs, max_active_jobs, ring_passes, hbm_budget_bytes, trace_block,
                                trace_refill, trace_occupancy, max_slice_iterations, schedule, deadline_slowdown,
                                short_job_seconds, bvh_build)
        h = ctypes.c_void_p()
        rc = self.L.gpt_server_create(ctypes.byref(h), device, ctypes.byref(cfg))
        if rc != 0:
            raise GptError(rc, f"gpt_server_create(device={device}) failed: {self.L.gpt_status_string(rc).decode()}")
        self.h = h
        self._jobs = {}

    def close(self):
        if getattr(self, "h", None):
            self.L.gpt_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc: int, what: str):
        if rc != 0:
            buf = ctypes.create_string_buffer(1024)
            self.L.gpt_server_peek_last_error(self.h, buf, 1024)
            raise GptError(rc, f"{what}: {buf.value.decode() or self.L.gpt_status_string(rc).decode()}")

    def add_scene(self, scene) -> int:
        desc, keep = scene_desc_with_textures(scene)
        sid = ctypes.c_uint32()
        self._check(self.L.gpt_server_add_scene(self.h, ctypes.byref(desc), ctypes.byref(sid)), "gpt_server_add_scene")
        del keep
        return sid.value

    def submit(self, scene_id: int, camera12, width: int, height: int, spp: int, depth: int, nee: bool = True,
               rng_offset: int = 0, keep_accumulation: bool = False, rng_policy: int = RNG_PHILOX,
               light_sampling: int = LIGHTS_AREA) -> int:
        d = gpt_job_desc(scene_id, width, height, spp, depth, 1 if nee else 0, rng_offset, camera_struct(camera12),
                         1 if keep_accumulation else 0, rng_policy, light_sampling, 0)
        jid = ctypes.c_uint64()
        self._check(self.L.gpt_server_submit(self.h, ctypes.byref(d), ctypes.byref(jid)), "gpt_server_submit")
        self._jobs[jid.value] = (width, height)
        return jid.value

    def poll(self, job: int) -> dict:
        st = gpt_job_status()
        self._check(self.L.gpt_server_poll(self.h, job, ctypes.byref(st)), "gpt_server_poll")
        return dict(state=JOB_STATES[st.state], passes_done=st.passes_done, passes_total=st.passes_total,
                    samples_total=st.samples_total, admitted_bytes=st.admitted_bytes, submit_s=st.submit_s,
                    admit_s=st.admit_s, done_s=st.done_s)

    def wait(self, job: int, timeout_s: float = 600.0):
        self._check(self.L.gpt_server_wait(self.h, job, timeout_s), "gpt_server_wait")
        return self.poll(job)

    def result(self, job: int, accumulation: bool = False):
        """(framebuffer [h*w] uint32, accumulation [h*w, 4] float32 or None)."""
        w, h = self._jobs[job]
        fb = np.zeros(w * h, dtype=np.uint32)
        acc = np.zeros((w * h, 4), dtype=np.float32) if accumulation else None
        self._check(self.L.gpt_server_read(self.h, job, _ptr(fb), _ptr(acc) if acc is not None else None), "gpt_server_read")
        return fb, acc

    def release(self, job: int):
        self._check(self.L.gpt_server_release(self.h, job), "gpt_server_release")
        self._jobs.pop(job, None)

    def cancel(self, job: int):
        self._check(self.L.gpt_server_cancel(self.h, job), "gpt_server_cancel")

    def set_loop_mode(self, mode: int):
        """LOOP_GRAPH (default): a slice is one graph launch; LOOP_HOST: iterations launched by the host."""
        self._check(self.L.gpt_server_set_loop_mode(self.h, mode), "gpt_server_set_loop_mode")

    def stats(self) -> dict:
        st = gpt_server_stats()
        self._check(self.L.gpt_server_get_stats(self.h, ctypes.byref(st)), "gpt_server_get_stats")
        out = {name: getattr(st, name) for name, _ in gpt_server_stats._fields_ if name != "phase_ms"}
        out["phase_ms"] = dict(zip(PHASES, list(st.phase_ms)))
        return out

    def last_error(self) -> str | None:
        buf = ctypes.create_string_buffer(1024)
        return buf.value.decode() if self.L.gpt_server_peek_last_error(self.h, buf, 1024) else None
