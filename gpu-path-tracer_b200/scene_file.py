"""Headless loader for the reference's YAML scene files: entities, transforms, models, grids and the
camera -> one world-space `scenes.Scene` plus the camera's first motion state.

The reference builds an ECS registry from the file and the CUDA renderer reads triangles from it:

* file layout: `scripts` (optional; phase Awake/Update + name) and the `scene` sequence of entities,
  each with `components` and optional `children` (Import/SceneLoader.cpp:8-57, ECS/Scene.cpp:11-104);
* components: Transform (ECS/Transform.cpp:8-61), Camera (Graphics/Ecs/Camera.cpp:11-35), Model and
  Grid (Graphics/Ecs/Assets.cpp:66-162); Background, Light, MotionRecorder and the application's
  CameraController are registered builders that the path tracer does not read, so they are checked
  for their type only (ECS/BuilderRegistry.cpp:10-20, App/Source/Scripts/Layer.cpp:14);
* world matrices: parent x local, propagated from the root entities that have a Transform; an entity
  without one passes its parent's matrix on (ECS/Transform.cpp:64-96);
* triangles: every model part with its world matrix, normals by the inverse transpose
  (PathTracing/Renderer.cpp:159-213, done by `gpt_obj_load`'s transform); materials deduplicated
  by material handle, and one OBJ file imported twice shares its handles (Assets/Manager.cpp:127-142,
  PathTracing/Renderer.cpp:70-110);
* camera: Camera.fovY in radians and the first motion state of the camera entity, (translation,
  rotation with uniform scale removed) of its world matrix (Capture/MotionRecorder.cpp:20-60,
  Utils/Math/Transform.hpp:6-33), for MakeDeviceCamera (PathTracing/Renderer.cpp:237-257).

The reference's quaternions and matrices come from glm (a third-party header library that the
reference fetches at build time; it is not vendored): glm::quat(euler) is the product
qz * qy * qx of the three axis rotations, toMat4 is the standard rotation matrix of a unit
quaternion, and quat_cast is Shepperd's method (J. Guidance and Control 1(3), 1978), restated
here in float32.

Triangle order: the reference takes it from the registry's view iteration, which depends on the
ECS library's pool order. Here it is the file's order, depth first, parent before children, a
model's parts in their OBJ order. The order changes triangle ids and the light list, not what is
visible.
"""
from __future__ import annotations

import math
import os

import numpy as np
import yaml

import pathtracer
import scenes

_F = np.float32
_IGNORED_COMPONENTS = ("Background", "Light", "MotionRecorder", "CameraController")


class SceneFileError(ValueError):
    """A scene file the reference's loader would also reject."""


# ----------------------------------------------------------------------------
# glm's quaternion and matrix conventions, float32
# ----------------------------------------------------------------------------

def _qmul(a, b):
    aw, ax, ay, az = a
    bw, bx, by, bz = b
    return np.array([aw * bw - ax * bx - ay * by - az * bz,
                     aw * bx + ax * bw + ay * bz - az * by,
                     aw * by - ax * bz + ay * bw + az * bx,
                     aw * bz + ax * by - ay * bx + az * bw], dtype=_F)


def _normalize_q(q):
    q = np.asarray(q, dtype=_F)
    n = _F(np.sqrt(np.dot(q, q)))
    if n <= _F(0):
        return np.array([1, 0, 0, 0], dtype=_F)
    return (q / n).astype(_F)


def quat_from_euler(radians) -> np.ndarray:
    """(w, x, y, z) of the rotation about x, then y, then z: qz * qy * qx (glm::quat(vec3))."""
    hx, hy, hz = (_F(a) * _F(0.5) for a in radians)
    qx = np.array([np.cos(hx), np.sin(hx), 0, 0], dtype=_F)
    qy = np.array([np.cos(hy), 0, np.sin(hy), 0], dtype=_F)
    qz = np.array([np.cos(hz), 0, 0, np.sin(hz)], dtype=_F)
    return _qmul(qz, _qmul(qy, qx))


def quat_to_mat3(q) -> np.ndarray:
    """Rotation matrix of a unit quaternion (w, x, y, z); columns are the rotated axes."""
    w, x, y, z = (_F(c) for c in q)
    one, two = _F(1), _F(2)
    return np.array([[one - two * (y * y + z * z), two * (x * y - w * z), two * (x * z + w * y)],
                     [two * (x * y + w * z), one - two * (x * x + z * z), two * (y * z - w * x)],
                     [two * (x * z - w * y), two * (y * z + w * x), one - two * (x * x + y * y)]], dtype=_F)


def quat_from_mat3(m) -> np.ndarray:
    """Shepperd's method: the largest of 4w^2-1, 4x^2-1, 4y^2-1, 4z^2-1 picks the component that is
    taken by a square root; the others follow from sums and differences of off-diagonal terms."""
    m = np.asarray(m, dtype=_F)
    cand = [m[0, 0] + m[1, 1] + m[2, 2], m[0, 0] - m[1, 1] - m[2, 2],
            m[1, 1] - m[0, 0] - m[2, 2], m[2, 2] - m[0, 0] - m[1, 1]]
    k = int(np.argmax(np.array(cand, dtype=_F)))
    big = _F(np.sqrt(_F(cand[k]) + _F(1))) * _F(0.5)
    f = _F(0.25) / big
    if k == 0:
        q = [big, (m[2, 1] - m[1, 2]) * f, (m[0, 2] - m[2, 0]) * f, (m[1, 0] - m[0, 1]) * f]
    elif k == 1:
        q = [(m[2, 1] - m[1, 2]) * f, big, (m[1, 0] + m[0, 1]) * f, (m[0, 2] + m[2, 0]) * f]
    elif k == 2:
        q = [(m[0, 2] - m[2, 0]) * f, (m[1, 0] + m[0, 1]) * f, big, (m[2, 1] + m[1, 2]) * f]
    else:
        q = [(m[1, 0] - m[0, 1]) * f, (m[0, 2] + m[2, 0]) * f, (m[2, 1] + m[1, 2]) * f, big]
    return np.array(q, dtype=_F)


def _normalize_v(v):
    v = np.asarray(v, dtype=_F)
    return (v / _F(np.sqrt(np.dot(v, v)))).astype(_F)


def look_at_quat(position, target) -> np.ndarray:
    """Rotation of a Transform given by 'target': forward toward the target, world up (0, 1, 0)
    unless forward is within 0.999 of it, then (0, 0, 1); the frame (right, up, -forward)
    (ECS/Transform.cpp:41-58)."""
    forward = np.asarray(target, dtype=_F) - np.asarray(position, dtype=_F)
    if float(np.sqrt(np.dot(forward, forward))) <= 1e-6:
        raise SceneFileError("Transform 'target' must differ from 'position'")
    forward = _normalize_v(forward)
    up = np.array([0, 1, 0], dtype=_F)
    if abs(float(np.dot(forward, up))) > 0.999:
        up = np.array([0, 0, 1], dtype=_F)
    right = _normalize_v(np.cross(forward, up))
    up = _normalize_v(np.cross(right, forward))
    return _normalize_q(quat_from_mat3(np.stack([right, up, -forward], axis=1)))


def trs_matrix(translation, rotation_wxyz, scale) -> np.ndarray:
    """translate * rotate * scale as a row-major 4x4 float32 matrix (Transform::GetMatrix)."""
    m = np.eye(4, dtype=_F)
    m[:3, :3] = quat_to_mat3(rotation_wxyz) * np.asarray(scale, dtype=_F)[None, :]
    m[:3, 3] = np.asarray(translation, dtype=_F)
    return m


def motion_state(world) -> tuple[np.ndarray, np.ndarray]:
    """(position, rotation (w, x, y, z)) of a world matrix: its translation, and the rotation of its
    3x3 part divided by the length of the first column (ExtractRotationUniformScale)."""
    world = np.asarray(world, dtype=_F)
    lin = world[:3, :3]
    scale = _F(np.sqrt(np.dot(lin[:, 0], lin[:, 0])))
    if scale <= _F(1e-6):
        return world[:3, 3].copy(), np.array([1, 0, 0, 0], dtype=_F)
    return world[:3, 3].copy(), _normalize_q(quat_from_mat3(lin / scale))


# ----------------------------------------------------------------------------
# Components
# ----------------------------------------------------------------------------

def _get(node, key, kind, entity):
    if not isinstance(node, dict) or key not in node:
        raise SceneFileError(f"entity {entity}: missing '{key}'")
    v = node[key]
    try:
        if kind == "vec3" or kind == "vec4":
            n = 3 if kind == "vec3" else 4
            if not isinstance(v, (list, tuple)) or len(v) != n:
                raise TypeError
            return [float(c) for c in v]
        if kind == "float":
            return float(v)
        if kind == "uint":
            if isinstance(v, bool) or int(v) != v or v < 0:
                raise TypeError
            return int(v)
        if kind == "str":
            if not isinstance(v, str):
                raise TypeError
            return v
    except (TypeError, ValueError):
        pass
    raise SceneFileError(f"entity {entity}: '{key}' is not a {kind}")


def _transform(node, entity):
    translation = _get(node, "translation", "vec3", entity)
    scale = _get(node, "scale", "vec3", entity)
    has_q, has_t = "quaternion" in node, "target" in node
    has_euler = "euler-degrees" in node or "euler-radians" in node
    if int(has_q) + int(has_euler) + int(has_t) > 1:
        raise SceneFileError("Transform can only have one of 'quaternion', 'euler', or 'target' specified")
    if has_q:
        rotation = _normalize_q(_get(node, "quaternion", "vec4", entity))  # (w, x, y, z)
    elif "euler-degrees" in node:
        rotation = _normalize_q(quat_from_euler([math.radians(a) for a in _get(node, "euler-degrees", "vec3", entity)]))
    elif "euler-radians" in node:
        rotation = _normalize_q(quat_from_euler(_get(node, "euler-radians", "vec3", entity)))
    elif has_t:
        rotation = look_at_quat(translation, _get(node, "target", "vec3", entity))
    else:
        rotation = np.array([1, 0, 0, 0], dtype=_F)
    return trs_matrix(translation, rotation, scale)


def _camera(node, entity):
    fov = _get(node, "fov-y", "float", entity)
    near = _get(node, "near-plane", "float", entity)
    far = _get(node, "far-plane", "float", entity)
    if fov <= 0.0 or fov >= 180.0:
        raise SceneFileError("Camera 'fov-y' must be in range (0, 180) degrees")
    if near <= 0.0:
        raise SceneFileError("Camera 'near-plane' must be greater than 0")
    if far <= near:
        raise SceneFileError("Camera 'far-plane' must be greater than 'near-plane'")
    return dict(fov_y=float(_F(math.radians(fov))), near=near, far=far)


# ----------------------------------------------------------------------------
# Entities -> instances
# ----------------------------------------------------------------------------

class _Entity:
    def __init__(self, index, parent):
        self.index, self.parent = index, parent
        self.local = None      # 4x4 when the entity has a Transform
        self.world = np.eye(4, dtype=_F)
        self.models = []       # OBJ paths (a Model, or a Grid cell's Model)
        self.camera = None
        self.children = []


def _parse(root):
    if not isinstance(root, dict):
        raise SceneFileError("Failed to get scene root sequence")
    for script in root.get("scripts") or []:
        if not isinstance(script, dict) or "name" not in script:
            raise SceneFileError("Script is missing 'name' field")
        if "phase" not in script:
            raise SceneFileError("Script is missing 'phase' field")
        if script["phase"] not in ("Awake", "Update"):
            raise SceneFileError(f"Invalid script phase '{script['phase']}'")
    seq = root.get("scene")
    if not isinstance(seq, list):
        raise SceneFileError("Failed to get scene root sequence")
    entities = []

    def build(node, parent):
        e = _Entity(len(entities), parent)
        entities.append(e)
        comps = node.get("components") if isinstance(node, dict) else None
        if comps is not None:
            if not isinstance(comps, list):
                raise SceneFileError("Entity 'components' must be a sequence")
            seen = set()
            for c in comps:
                kind = _get(c, "type", "str", e.index)
                # The reference's registry holds one component of a type per entity, and Model and
                # Grid both give the entity its Children list: a second one is not a defined scene.
                slot = "Children" if kind in ("Model", "Grid") else kind
                if slot in ("Transform", "Camera", "Children"):
                    if slot in seen:
                        raise SceneFileError(f"entity {e.index}: more than one {'Model or Grid' if slot == 'Children' else kind} component")
                    seen.add(slot)
                if kind == "Transform":
                    e.local = _transform(c, e.index)
                elif kind == "Camera":
                    e.camera = _camera(c, e.index)
                elif kind == "Model":
                    e.models.append(_get(c, "path", "str", e.index))
                elif kind == "Grid":
                    rows, cols = _get(c, "rows", "uint", e.index), _get(c, "columns", "uint", e.index)
                    spacing, path = _get(c, "spacing", "float", e.index), _get(c, "path", "str", e.index)
                    for i in range(rows):
                        for j in range(cols):
                            cell = _Entity(len(entities), e)
                            entities.append(cell)
                            # integer halving as in the reference (int32 (columns) / 2), then float32
                            pos = [_F(j - int(cols / 2)) * _F(spacing), _F(i - int(rows / 2)) * _F(spacing), 0.0]
                            cell.local = trs_matrix(pos, [1, 0, 0, 0], [1, 1, 1])
                            cell.models.append(path)
                            e.children.append(cell)
                elif kind not in _IGNORED_COMPONENTS:
                    raise SceneFileError(f"no builder registered for component type '{kind}'")
        kids = node.get("children") if isinstance(node, dict) else None
        if kids is not None:
            if not isinstance(kids, list):
                raise SceneFileError("Entity 'children' must be a sequence")
            if e.models or e.children:
                raise SceneFileError(f"entity {e.index}: a Model or Grid entity cannot also list 'children' "
                                     "(both would be its Children list)")
            for k in kids:
                e.children.append(build(k, e))
        return e

    roots = [build(n, None) for n in seq]
    return roots, entities


def _propagate(e, parent_world):
    """e.world = the matrix its model parts get: parent x local, or the parent's own matrix when the
    entity has no Transform (its parts' identity transforms then sit directly under the parent)."""
    world = parent_world if e.local is None else (parent_world @ e.local).astype(_F)
    e.world = world
    for c in e.children:
        _propagate(c, world)


def load_scene(path: str, assets_root: str | None = None) -> scenes.Scene:
    """A reference YAML scene file -> world-space scenes.Scene.

    Model paths resolve against `assets_root` (default: the directory above the file's
    directory, as the reference's `Assets/Scenes/*.yaml` name `Models/...` under `Assets/`).
    `scene.camera` holds `fov_y` (radians), `near`, `far`, `position` and `rotation` (w, x, y, z):
    pass it to `device_camera`.
    """
    with open(path) as f:
        try:
            root = yaml.safe_load(f)
        except yaml.YAMLError as err:
            raise SceneFileError(f"Failed to load scene: {err}") from None
    roots, entities = _parse(root)
    for r in roots:
        if r.local is not None:  # only roots with a Transform propagate; the rest keep identity
            _propagate(r, np.eye(4, dtype=_F))
    cams = [e for e in entities if e.camera is not None]
    if len(cams) != 1:
        raise SceneFileError("Scene must contain exactly one camera!")
    if cams[0].local is None:
        raise SceneFileError("Camera entity must have a Transform component")
    if assets_root is None:
        assets_root = os.path.dirname(os.path.dirname(os.path.abspath(path)))

    parts, mats, textures, mat_tex = [], [], [], []
    first = {}  # resolved OBJ path -> (material offset, texture offset) of its first import
    for e in entities:
        for rel in e.models:
            resolved = os.path.normpath(os.path.join(assets_root, rel))
            if not os.path.isfile(resolved):
                raise SceneFileError(f"model file not found: {rel} (under {assets_root})")
            s = pathtracer.load_obj(resolved, transform=e.world)
            if resolved not in first:
                first[resolved] = (sum(len(m) for m in mats), len(textures))
                mats.append(s.materials)
                mt = s.material_textures if s.material_textures is not None else np.full((len(s.materials), 6), -1, np.int32)
                mat_tex.append(np.where(mt >= 0, mt + len(textures), -1).astype(np.int32))
                textures.extend(s.textures)
            moff = first[resolved][0]
            parts.append((s.positions, s.normals, s.tangents, s.uvs, (s.material_ids + np.uint32(moff)).astype(np.uint32)))
    if not parts:
        raise SceneFileError("scene has no model")
    out = scenes.Scene(np.concatenate([p[0] for p in parts]), np.concatenate([p[1] for p in parts]),
                       np.concatenate([p[2] for p in parts]), np.concatenate([p[3] for p in parts]),
                       np.concatenate([p[4] for p in parts]), np.concatenate(mats),
                       name=os.path.basename(path)).contiguous()
    if textures:
        out.textures = textures
        out.material_textures = np.concatenate(mat_tex)
    position, rotation = motion_state(cams[0].world)
    out.camera = dict(cams[0].camera, position=position, rotation=rotation)
    return out


def device_camera(scene: scenes.Scene, width: int, height: int) -> np.ndarray:
    """The 12-float DeviceCamera of a loaded scene file's camera for a width x height frame."""
    c = scene.camera
    return pathtracer.make_device_camera(c["fov_y"], float(_F(width) / _F(height)), c["position"], c["rotation"])
