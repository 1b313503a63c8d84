"""Tangent frames of imported meshes (gpt_generate_tangents, Mikkelsen's method) against the
reference's own MikkTSpace (External/mikktspace/mikktspace.c compiled from the reference tree into
oracle/_ref/ and driven as TangentSpace.cpp:66-89 drives it): bit for bit on meshes with uv seams,
mirrored uvs, degenerate and zero-uv-area triangles and non-manifold edges. Host code, no GPU."""
import numpy as np
import pytest

import pathtracer
import ref_harness


def uv_sphere(nu=24, nv=12, mirror=False):
    P, T, idx = [], [], []
    for j in range(nv + 1):
        th = np.pi * j / nv
        for i in range(nu + 1):
            ph = 2 * np.pi * i / nu
            P.append([np.sin(th) * np.cos(ph), np.cos(th), np.sin(th) * np.sin(ph)])
            u = i / nu
            T.append([1 - abs(2 * u - 1) if mirror else u, j / nv])
    for j in range(nv):
        for i in range(nu):
            a = j * (nu + 1) + i
            b, c = a + 1, a + nu + 1
            idx += [[a, c, b], [b, c, c + 1]]
    P = np.array(P, np.float32)
    return P, P.copy(), np.array(T, np.float32), np.array(idx, np.uint32)


def random_mesh(seed, n=400):
    rng = np.random.default_rng(seed)
    P = rng.normal(size=(n, 3)).astype(np.float32)
    N = rng.normal(size=(n, 3))
    N = (N / np.linalg.norm(N, axis=1, keepdims=True)).astype(np.float32)
    T = rng.uniform(size=(n, 2)).astype(np.float32)
    idx = rng.integers(0, n, size=(2 * n, 3)).astype(np.uint32)
    idx[::37, 1] = idx[::37, 0]           # degenerate triangles
    T[::11] = T[::11][:, :1].repeat(2, 1)  # uv on a line: no uv area
    return P, N, T, idx


MESHES = {"sphere": lambda: uv_sphere(), "sphere-mirrored-uv": lambda: uv_sphere(mirror=True),
          "sphere-fine": lambda: uv_sphere(96, 48), "random-1": lambda: random_mesh(1), "random-2": lambda: random_mesh(2)}


@pytest.mark.skipif(not ref_harness.mikk_available(), reason="oracle/_ref not built (needs the reference sources)")
@pytest.mark.parametrize("name", sorted(MESHES))
def test_tangents_bit_exact_with_the_reference_mikktspace(name):
    mesh = MESHES[name]()
    got = pathtracer.generate_tangents(*mesh)
    ref = ref_harness.mikk_tangents(*mesh)
    used = np.zeros(len(got), bool)
    used[mesh[3].reshape(-1)] = True
    assert np.array_equal(got[used].view(np.uint32), ref[used].view(np.uint32))


def test_tangent_frames_are_unit_and_orthogonal_on_a_smooth_mesh():
    P, N, T, idx = uv_sphere(48, 24)
    t = pathtracer.generate_tangents(P, N, T, idx)
    inner = np.ones(len(P), bool)
    inner[:49] = inner[-49:] = False  # the poles' fans
    assert np.allclose(np.linalg.norm(t[inner, :3], axis=1), 1.0, atol=1e-6)
    assert np.max(np.abs((t[inner, :3] * N[inner]).sum(1))) < 1e-5
    # u increases with the azimuth: the tangent points along +phi (-sin, 0, cos)
    phi = np.arctan2(P[inner, 2], P[inner, 0])
    along = np.stack([-np.sin(phi), np.zeros_like(phi), np.cos(phi)], 1)
    assert np.min((t[inner, :3] * along).sum(1)) > 0.99
    assert set(np.unique(t[:, 3]).tolist()) <= {-1.0, 1.0}
    # mirrored uvs flip the handedness on the mirrored half
    _, _, Tm, _ = uv_sphere(48, 24, mirror=True)
    tm = pathtracer.generate_tangents(P, N, Tm, idx)
    assert (tm[inner, 3] < 0).any() and (tm[inner, 3] > 0).any()


def test_tangent_argument_checks():
    P, N, T, idx = uv_sphere()
    bad = idx.copy()
    bad[0, 0] = len(P)
    with pytest.raises(pathtracer.GptError):
        pathtracer.generate_tangents(P, N, T, bad)
