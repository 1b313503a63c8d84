"""Camera-path resampling (gpt_resample_motion) against the oracle's restatement of
Capture::ResampleMotion (Core/Source/Capture/Resampling.cpp:17-55); host code, no GPU."""
import math

import numpy as np
import pytest

import oracle
import pathtracer


def axis_angle(axis, deg):
    a = np.asarray(axis, np.float64)
    a = a / np.linalg.norm(a)
    h = math.radians(deg) / 2
    return (math.cos(h), *(a * math.sin(h)))


PATH = [
    ((0.0, 1.0, 4.0), axis_angle((0, 1, 0), 0), 0.0),
    ((0.5, 1.1, 3.8), axis_angle((0, 1, 0), 20), 0.37),
    ((1.2, 1.0, 3.1), axis_angle((0.2, 1, 0), 55), 0.81),
    ((2.0, 0.8, 2.0), axis_angle((0.2, 1, 0.1), 90), 1.30),
    ((2.1, 0.8, 1.9), axis_angle((0.2, 1, 0.1), 90.0001), 1.31),   # nearly parallel rotations: linear branch
    ((3.0, 0.5, 0.0), tuple(-np.asarray(axis_angle((0, 1, 0), 170))), 2.02),  # opposite hemisphere: shorter arc
]


@pytest.mark.parametrize("interval", [1 / 60, 0.1, 0.25, 0.5, 3.0])
def test_resample_motion_matches_the_restatement(interval):
    got = pathtracer.resample_motion(PATH, interval)
    ref = oracle.resample_motion(PATH, interval)
    assert len(got) == len(ref) == int(math.floor((2.02 - 0.0) / np.float32(interval) + 1e-6)) + 1
    for (gp, gq), (rp, rq) in zip(got, ref):
        assert np.allclose(gp, rp, rtol=0, atol=2e-6)
        assert np.allclose(gq, rq, rtol=0, atol=2e-6)
        assert abs(np.linalg.norm(gq) - 1.0) < 1e-6
    # the first state is the first sample's, unchanged
    assert got[0][0] == tuple(np.float32(PATH[0][0])) and np.allclose(got[0][1], PATH[0][1])


def test_resample_takes_the_shorter_arc():
    states = pathtracer.resample_motion(PATH[4:], 0.05)
    q0 = np.asarray(PATH[4][1])
    for _, q in states:
        # every interpolated rotation stays on the start's hemisphere (angle to it at most 90 degrees)
        assert np.dot(q, q0) > 0.0


def test_resample_edge_cases():
    assert pathtracer.resample_motion([], 0.1) == []
    one = pathtracer.resample_motion(PATH[:1], 0.1)
    assert len(one) == 1 and np.allclose(one[0][1], PATH[0][1])
    assert len(pathtracer.resample_motion(PATH[:2], 10.0)) == 1
    with pytest.raises(pathtracer.GptError) as e:
        pathtracer.resample_motion(PATH[:2], 0.0)
    assert e.value.code == 1
    bad = [PATH[0], (PATH[1][0], PATH[1][1], 0.0)]
    with pytest.raises(pathtracer.GptError) as e:
        pathtracer.resample_motion(bad, 0.1)
    assert e.value.code == 1
    # capacity: the count comes back with GPT_ERR_CAPACITY and nothing is written
    import ctypes
    arr = (pathtracer.gpt_motion_sample * 2)()
    arr[1].time = 1.0
    arr[0].state.rotation[0] = arr[1].state.rotation[0] = 1.0
    n = ctypes.c_uint32()
    out = (pathtracer.gpt_motion_state * 2)()
    assert pathtracer.lib().gpt_resample_motion(arr, 2, ctypes.c_float(0.25), out, 2, ctypes.byref(n)) == 6
    assert n.value == 5
