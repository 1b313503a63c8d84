"""Headless YAML scene files (host code, no GPU): transforms in the reference's conventions, entity
hierarchy and grids, material sharing between imports of one OBJ, the camera's motion state, and the
reference loader's error cases."""
import math
import os

import numpy as np
import pytest

import pathtracer
import scene_file as sf
import scenes
from test_obj_import import write_obj


def axis_matrix(axis, a):
    c, s = math.cos(a), math.sin(a)
    if axis == 0:
        return np.array([[1, 0, 0], [0, c, -s], [0, s, c]])
    if axis == 1:
        return np.array([[c, 0, s], [0, 1, 0], [-s, 0, c]])
    return np.array([[c, -s, 0], [s, c, 0], [0, 0, 1]])


def same_rotation(q1, q2, tol=1e-6):
    return min(np.abs(q1 - q2).max(), np.abs(q1 + q2).max()) < tol


def test_euler_quaternion_is_x_then_y_then_z():
    rng = np.random.default_rng(5)
    for _ in range(50):
        e = rng.uniform(-math.pi, math.pi, 3)
        expect = axis_matrix(2, e[2]) @ axis_matrix(1, e[1]) @ axis_matrix(0, e[0])
        q = sf.quat_from_euler(e)
        assert abs(float(np.dot(q, q)) - 1.0) < 1e-6
        assert np.allclose(sf.quat_to_mat3(q), expect, atol=2e-6)


def test_matrix_quaternion_round_trip_covers_every_branch():
    rng = np.random.default_rng(6)
    qs = [np.array(q, np.float32) for q in ([1, 0, 0, 0], [0, 1, 0, 0], [0, 0, 1, 0], [0, 0, 0, 1])]
    qs += [sf._normalize_q(rng.normal(size=4)) for _ in range(200)]
    branches = set()
    for q in qs:
        m = sf.quat_to_mat3(q)
        branches.add(int(np.argmax([m[0, 0] + m[1, 1] + m[2, 2], m[0, 0] - m[1, 1] - m[2, 2],
                                    m[1, 1] - m[0, 0] - m[2, 2], m[2, 2] - m[0, 0] - m[1, 1]])))
        assert same_rotation(sf._normalize_q(sf.quat_from_mat3(m)), q, 2e-6)
    assert branches == {0, 1, 2, 3}


def test_look_at_points_forward_at_the_target():
    for pos, target in (([0, 10, 20], [0, 0, 0]), ([3, -2, 1], [-4, 5, 9]), ([0, 5, 0], [0, -5, 0])):
        q = sf.look_at_quat(pos, target)
        r = sf.quat_to_mat3(q)
        fwd = np.subtract(target, pos) / np.linalg.norm(np.subtract(target, pos))
        assert np.allclose(r @ [0, 0, -1], fwd, atol=1e-6)  # CoordinateSystem::Forward = -z
        assert abs(float((r @ [1, 0, 0])[1])) < 1e-6 or abs(fwd[1]) > 0.999  # right stays horizontal
    # straight down: world up is replaced by +z, so right = forward x +z = -x and the camera's up is +z
    r = sf.quat_to_mat3(sf.look_at_quat([0, 5, 0], [0, -5, 0]))
    assert np.allclose(r @ [0, 1, 0], [0, 0, 1], atol=1e-6) and np.allclose(r @ [1, 0, 0], [-1, 0, 0], atol=1e-6)


def test_motion_state_removes_uniform_scale():
    q = sf._normalize_q([0.9, 0.1, -0.3, 0.2])
    m = sf.trs_matrix([1, 2, 3], q, [2.5, 2.5, 2.5])
    pos, rot = sf.motion_state(m)
    assert np.array_equal(pos, np.float32([1, 2, 3]))
    assert same_rotation(rot, q, 2e-6)


@pytest.fixture
def assets(tmp_path):
    """Assets/Models/{Room,Ball} as OBJ + MTL, scene files go to Assets/Scenes."""
    root = tmp_path / "Assets"
    room, ball = root / "Models" / "Room", root / "Models" / "Ball"
    for d in (room, ball, root / "Scenes"):
        d.mkdir(parents=True)
    write_obj(scenes.cornell_box(1), str(room))
    sphere = scenes.sphere_field(1, 1, 2, 3, name="ball")
    write_obj(sphere, str(ball))
    return root


def write_scene(root, text, name="test.yaml"):
    p = root / "Scenes" / name
    p.write_text(text)
    return str(p)


SCENE = """
scripts:
    - phase: Awake
      name: AwakeCameraController
scene:
    - components:
        - type: Transform
          translation: [0.5, 0.5, 2.5]
          target: [0.5, 0.4, 0.0]
          scale: [1.0, 1.0, 1.0]
        - type: Camera
          fov-y: 40.0
          near-plane: 0.1
          far-plane: 100.0
        - type: CameraController
          speed: 10.0
          sensitivity: 0.01
    - components:
        - type: Transform
          translation: [0.0, 0.0, 0.0]
          euler-degrees: [0.0, 30.0, 0.0]
          scale: [1.0, 1.0, 1.0]
      children:
        - components:
            - type: Model
              path: Models/Room/scene.obj
        - components:
            - type: Transform
              translation: [0.25, 0.1, 0.5]
              quaternion: [1.0, 0.0, 0.0, 0.0]
              scale: [0.05, 0.05, 0.05]
            - type: Model
              path: Models/Ball/scene.obj
        - components:
            - type: Light
              color: [1.0, 1.0, 1.0]
              intensity: 1.0
    - components:
        - type: Transform
          translation: [0.5, 0.5, 0.5]
          euler-radians: [0.0, 0.0, 0.0]
          scale: [0.02, 0.02, 0.02]
        - type: Grid
          rows: 2
          columns: 3
          spacing: 10.0
          path: Models/Ball/scene.obj
"""


def test_scene_file_instances_materials_and_camera(assets):
    s = sf.load_scene(write_scene(assets, SCENE))
    room = pathtracer.load_obj(str(assets / "Models/Room/scene.obj"))
    ball = pathtracer.load_obj(str(assets / "Models/Ball/scene.obj"))
    nr, nb = room.triangle_count, ball.triangle_count
    assert s.triangle_count == nr + 7 * nb  # room, one child ball, a 2 x 3 grid of balls

    def placed(local, m):
        p = local.positions.reshape(-1, 3).astype(np.float64)
        return (p @ m[:3, :3].T.astype(np.float64) + m[:3, 3]).reshape(-1, 3, 3)

    rot_y = np.eye(4)
    rot_y[:3, :3] = axis_matrix(1, math.radians(30.0))
    assert np.allclose(s.positions[:nr], placed(room, rot_y), atol=1e-5)
    child = np.eye(4)
    child[:3, :3] = np.diag([0.05] * 3)
    child[:3, 3] = [0.25, 0.1, 0.5]
    assert np.allclose(s.positions[nr:nr + nb], placed(ball, rot_y @ child), atol=1e-5)
    grid = np.diag([0.02, 0.02, 0.02, 1.0])
    grid[:3, 3] = 0.5
    k = nr + nb
    for i in range(2):
        for j in range(3):
            cell = np.eye(4)
            cell[:3, 3] = [(j - 1) * 10.0, (i - 1) * 10.0, 0.0]
            assert np.allclose(s.positions[k:k + nb], placed(ball, grid @ cell), atol=1e-5)
            k += nb
    # one material table entry per material of each OBJ file, shared by all its imports
    assert len(s.materials) == len(room.materials) + len(ball.materials)
    assert np.array_equal(s.material_ids[:nr], room.material_ids)
    for k in range(nr, s.triangle_count, nb):
        assert np.array_equal(s.material_ids[k:k + nb], ball.material_ids + len(room.materials))
    # camera: the first motion state of its entity, fov in radians
    assert s.camera["fov_y"] == pytest.approx(math.radians(40.0))
    assert np.allclose(s.camera["position"], [0.5, 0.5, 2.5])
    cam = sf.device_camera(s, 64, 48)
    expect = scenes.make_camera([0.5, 0.5, 2.5], [0.5, 0.4, 0.0], 40.0, 64 / 48)
    assert np.allclose(cam, expect, atol=2e-6)


def test_entities_without_a_transform(assets):
    text = """
scene:
    - components:
        - type: Transform
          translation: [0.0, 0.0, 5.0]
          scale: [1.0, 1.0, 1.0]
        - type: Camera
          fov-y: 50.0
          near-plane: 0.1
          far-plane: 10.0
    - components:
        - type: Transform
          translation: [1.0, 0.0, 0.0]
          scale: [1.0, 1.0, 1.0]
      children:
        - components:
            - type: Model
              path: Models/Ball/scene.obj
    - components:
        - type: Light
          color: [1.0, 1.0, 1.0]
          intensity: 1.0
      children:
        - components:
            - type: Model
              path: Models/Ball/scene.obj
        - components:
            - type: Transform
              translation: [0.0, 3.0, 0.0]
              scale: [1.0, 1.0, 1.0]
            - type: Model
              path: Models/Ball/scene.obj
"""
    s = sf.load_scene(write_scene(assets, text))
    ball = pathtracer.load_obj(str(assets / "Models/Ball/scene.obj"))
    nb = ball.triangle_count
    # a child without a Transform takes its parent's matrix
    assert np.allclose(s.positions[:nb], ball.positions + np.float32([1, 0, 0]), atol=1e-6)
    # a root without a Transform is not propagated: it and its whole subtree stay at identity
    assert np.allclose(s.positions[nb:2 * nb], ball.positions, atol=1e-6)
    assert np.allclose(s.positions[2 * nb:], ball.positions, atol=1e-6)
    assert np.allclose(s.camera["rotation"], [1, 0, 0, 0])


CAMERA = """    - components:
        - type: Transform
          translation: [0.0, 0.0, 5.0]
          scale: [1.0, 1.0, 1.0]
        - type: Camera
          fov-y: 50.0
          near-plane: 0.1
          far-plane: 10.0
"""
MODEL = """    - components:
        - type: Transform
          translation: [0.0, 0.0, 0.0]
          scale: [1.0, 1.0, 1.0]
        - type: Model
          path: Models/Ball/scene.obj
"""


@pytest.mark.parametrize("text,message", [
    ("scene:\n" + MODEL, "exactly one camera"),
    ("scene:\n" + CAMERA + CAMERA + MODEL, "exactly one camera"),
    ("scene:\n" + CAMERA.replace("fov-y: 50.0", "fov-y: 180.0") + MODEL, "fov-y"),
    ("scene:\n" + CAMERA.replace("near-plane: 0.1", "near-plane: 0.0") + MODEL, "near-plane"),
    ("scene:\n" + CAMERA.replace("far-plane: 10.0", "far-plane: 0.05") + MODEL, "far-plane"),
    ("scene:\n" + CAMERA.replace("scale: [1.0, 1.0, 1.0]", "scale: [1.0, 1.0, 1.0]\n          target: [0.0, 0.0, 5.0]") + MODEL,
     "'target' must differ"),
    ("scene:\n" + CAMERA.replace("scale: [1.0, 1.0, 1.0]", "scale: [1.0, 1.0, 1.0]\n          target: [0.0, 0.0, 0.0]\n"
                                 "          euler-degrees: [0.0, 0.0, 0.0]") + MODEL, "only have one of"),
    ("scene:\n" + CAMERA.replace("          translation: [0.0, 0.0, 5.0]\n", "") + MODEL, "translation"),
    ("scene:\n" + CAMERA + MODEL.replace("type: Model", "type: Spline"), "no builder"),
    ("scene:\n" + CAMERA + MODEL.replace("Ball", "Missing"), "not found"),
    ("scripts:\n    - phase: Late\n      name: X\nscene:\n" + CAMERA + MODEL, "Invalid script phase"),
    ("scene: {}\n", "scene root sequence"),
    ("scene:\n" + CAMERA + MODEL.replace("scale: [1.0, 1.0, 1.0]", "scale: [1.0, 1.0, 1.0]\n        - type: Transform\n"
                                         "          translation: [0.0, 0.0, 0.0]\n          scale: [1.0, 1.0, 1.0]"),
     "more than one Transform"),
    ("scene:\n" + CAMERA + MODEL + "        - type: Model\n          path: Models/Ball/scene.obj\n", "more than one Model or Grid"),
    ("scene:\n" + CAMERA + MODEL + "      children:\n" + MODEL.replace("    - ", "        - ", 1).replace("\n    ", "\n        "),
     "cannot also list 'children'"),
])
def test_scene_file_errors(assets, text, message):
    with pytest.raises(sf.SceneFileError, match=message):
        sf.load_scene(write_scene(assets, text))


def test_camera_entity_needs_a_transform(assets):
    text = "scene:\n    - components:\n        - type: Camera\n          fov-y: 50.0\n          near-plane: 0.1\n" \
           "          far-plane: 10.0\n" + MODEL
    with pytest.raises(sf.SceneFileError, match="must have a Transform"):
        sf.load_scene(write_scene(assets, text))
