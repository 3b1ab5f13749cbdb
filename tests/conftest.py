"""Shared fixtures. GPU tests are marked ``gpu``; everything else runs on CPU."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def cuda_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if cuda_available():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


@pytest.fixture(scope="session")
def halton_perm():
    from ymrt_b200 import scenes
    return scenes.halton_permutations()


@pytest.fixture(scope="session")
def scene_dir(tmp_path_factory):
    d = os.environ.get("YMRT_SCENE_CACHE")
    if d:
        return d
    return str(tmp_path_factory.mktemp("scenes"))


@pytest.fixture(scope="session")
def cornell_path(scene_dir):
    from ymrt_b200 import scenes
    return scenes.scene_path("cornell", 0, scene_dir)


@pytest.fixture(scope="session")
def instanced_path(scene_dir):
    from ymrt_b200 import scenes
    return scenes.scene_path("instanced", 0, scene_dir)


@pytest.fixture(scope="session")
def volumetric_path(scene_dir):
    from ymrt_b200 import scenes
    return scenes.scene_path("volumetric", 0, scene_dir)


@pytest.fixture(scope="session")
def oracle():
    """The reference built for the host (oracle/_ref); skips when absent."""
    from oracle import ref
    if not ref.available():
        try:
            from oracle import build_ref
            build_ref.build()
        except Exception as e:  # reference sources absent (e.g. on a GPU machine without the prebuilt library)
            pytest.skip(f"oracle library unavailable: {e}")
    return ref


@pytest.fixture(scope="session")
def ctx():
    import ymrt_b200 as Y
    c = Y.Context(0)
    yield c
    c.close()
