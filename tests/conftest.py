import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for sub in ("gpu-path-tracer_b200", "oracle"):
    path = os.path.join(ROOT, sub)
    if path not in sys.path:
        sys.path.insert(0, path)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


_scene_cache = {}


def get_scene(name):
    import scenes
    if name not in _scene_cache:
        _scene_cache[name] = scenes.config_scene(name)
    return _scene_cache[name]


@pytest.fixture(scope="session")
def scene_factory():
    return get_scene


_oracle_cache = {}


@pytest.fixture(scope="session")
def oracle_scene():
    import oracle

    def get(name):
        if name not in _oracle_cache:
            _oracle_cache[name] = oracle.OracleScene(get_scene(name))
        return _oracle_cache[name]
    return get


@pytest.fixture(scope="session")
def gpu_renderer():
    """The deterministic build (libgpt_b200_det.so): bit-for-bit comparable with the oracle."""
    import pathtracer
    r = pathtracer.Renderer(0, variant="det")
    yield r
    r.close()


@pytest.fixture(scope="session")
def gpu_renderer_product():
    """The product build (libgpt_b200.so): the reference build's arithmetic."""
    import pathtracer
    r = pathtracer.Renderer(0, variant="product")
    yield r
    r.close()
