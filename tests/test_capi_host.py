"""The C-ABI library without a GPU: it loads, exports every symbol include/gpt_b200.h
declares, and its host-only entry points (BVH8 builder validation, camera) behave."""
import ctypes
import math
import os
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

import oracle
import pathtracer
import scenes

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "gpt_b200.h")


def header_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(gpt_[a-z0-9_]+)\s*\(", text)))


@pytest.mark.parametrize("variant", ["product", "det"])
def test_library_loads_and_exports_every_declared_symbol(variant):
    lib = pathtracer.lib(variant)
    declared = header_functions()
    assert len(declared) >= 30
    out = subprocess.run(["nm", "-D", "--defined-only", pathtracer.LIB_PATHS[variant]], capture_output=True, text=True,
                         check=True).stdout
    exported = set(re.findall(r" T (gpt_[a-z0-9_]+)", out))
    missing = [f for f in declared if f not in exported]
    assert not missing, missing
    for f in declared:
        assert getattr(lib, f) is not None
    assert sorted(pathtracer.declared_symbols()) == declared


def test_library_is_built_for_sm100a():
    # the build recipe compiles every CUDA source for sm_100a and nothing else (the GPU tests run
    # its kernels, which a library without sm_100 code could not launch)
    makefile = (Path(pathtracer.LIB_PATH).parent / "Makefile").read_text()
    arch = re.findall(r"-gencode\s+arch=(\S+),code=(\S+)", makefile)
    assert arch == [("compute_100a", "sm_100a")]
    assert re.search(r"^ARCH\s*=", makefile, re.M)
    assert makefile.count("$(ARCH)") >= 2


def test_product_and_deterministic_builds_differ_only_in_the_wavefront_arithmetic():
    # the product compiles the wavefront kernels with contraction and CUDA's transcendentals; the
    # deterministic build without contraction and with the IEEE definitions; the scene-upload kernels
    # (host-code restatements) are shared and never contracted
    makefile = (Path(pathtracer.LIB_PATH).parent / "Makefile").read_text()
    flags = dict(re.findall(r"^(NVFLAGS_\w+)\s*=\s*(.*)$", makefile, re.M))
    assert "-fmad=false" in flags["NVFLAGS_DET"] and "-DPT_CUDA_MATH=0" in flags["NVFLAGS_DET"]
    assert "-fmad=false" not in flags["NVFLAGS_PROD"] and "-DPT_CUDA_MATH=1" in flags["NVFLAGS_PROD"]
    assert re.search(r"scene_kernels\.o: .*\n\t\$\(NVCC\) \$\(NVFLAGS_DET\)", makefile)
    assert re.search(r"kernels_prod\.o: .*\n\t\$\(NVCC\) \$\(NVFLAGS_PROD\)", makefile)


def test_noalloc_rejects_misaligned_or_missing_pointers_before_any_device_work():
    # argument checks run before the library touches the device, so fake addresses are safe here
    lib = pathtracer.lib()
    vp = ctypes.c_void_p
    assert lib.gpt_build_alias_table_noalloc(vp(0x10000), 4, vp(0x20008), None) == 1   # bins not 16-byte aligned
    assert lib.gpt_build_alias_table_noalloc(vp(0x10002), 4, vp(0x20000), None) == 1   # weights not 4-byte aligned
    assert lib.gpt_build_alias_table_noalloc(None, 4, vp(0x20000), None) == 1
    assert lib.gpt_build_alias_table_noalloc(vp(0x10000), 0, vp(0x20008), None) == 0   # no lights: nothing to do


def test_status_strings():
    lib = pathtracer.lib()
    assert lib.gpt_status_string(0) == b"ok"
    assert lib.gpt_status_string(5) == b"no scene uploaded"


@pytest.mark.parametrize("name", ["cornell", "cornell-all", "spheres-small", "spheres-200k"])
def test_bvh8_quantised_boxes_contain_their_subtrees(name):
    s = scenes.config_scene(name)
    r = pathtracer.bvh8_check(s)
    assert r["violations"] == 0
    assert r["misplaced"] == 0
    assert r["depth"] <= 64
    assert r["nodes"] >= 1


def test_bvh8_collapse_fills_wide_nodes():
    # the surface-area-optimal collapse spreads single-triangle leaves over the 8 slots: a sphere field
    # of 204,866 triangles needs about 40K wide nodes, 6 children each (greedily opening the largest
    # child left 4.1 children per node on the 1.3M-triangle field)
    s = scenes.config_scene("spheres-200k")
    r = pathtracer.bvh8_check(s)
    assert r["violations"] == 0 and r["misplaced"] == 0
    children_per_node = (s.triangle_count + r["nodes"] - 1) / r["nodes"]
    assert children_per_node > 5.5, children_per_node


def test_bvh8_degenerate_inputs():
    # all triangles identical (no SAH split possible) and a single triangle
    s = scenes.cornell_box(1)
    same = scenes.Scene(np.repeat(s.positions[:1], 64, 0), np.repeat(s.normals[:1], 64, 0), np.repeat(s.tangents[:1], 64, 0),
                        np.repeat(s.uvs[:1], 64, 0), np.zeros(64, np.uint32), s.materials[:1].copy())
    r = pathtracer.bvh8_check(same)
    assert r["violations"] == 0 and r["misplaced"] == 0
    one = scenes.Scene(s.positions[:1].copy(), s.normals[:1].copy(), s.tangents[:1].copy(), s.uvs[:1].copy(),
                       np.zeros(1, np.uint32), s.materials[:1].copy())
    r = pathtracer.bvh8_check(one)
    assert r["violations"] == 0 and r["misplaced"] == 0 and r["nodes"] == 1


def test_make_device_camera_matches_reference_restatement():
    pos = (0.3, 1.2, 4.0)
    q = np.array([0.9, 0.1, -0.3, 0.2], dtype=np.float64)
    q = q / np.linalg.norm(q)
    got = pathtracer.make_device_camera(math.radians(40.0), 16 / 9, pos, q)
    ref = oracle.make_camera_from_motion(math.radians(40.0), 16 / 9, pos, q)
    assert np.allclose(got, ref, rtol=0, atol=1e-6)


def test_scene_validation_rejects_bad_material_index():
    s = scenes.cornell_box(1)
    bad = scenes.Scene(s.positions.copy(), s.normals.copy(), s.tangents.copy(), s.uvs.copy(),
                       np.full(36, 99, np.uint32), s.materials.copy())
    with pytest.raises(pathtracer.GptError):
        pathtracer.bvh8_check(bad)


def test_python_binding_struct_layouts_match_the_library():
    sizes = pathtracer.abi_struct_sizes()
    for name, size in sizes.items():
        assert ctypes.sizeof(getattr(pathtracer, name)) == size, name
