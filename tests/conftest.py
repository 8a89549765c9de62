"""Shared fixtures.  GPU tests are marked ``gpu``; everything else runs on CPU."""
import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session", autouse=True)
def native_libs():
    """Build libatrc_cuda.so and the oracle in-tree if they are missing."""
    from atrc_b200 import build
    build.build_library()
    build.build_oracle()
    yield


@pytest.fixture(scope="session")
def scene_dir(tmp_path_factory):
    d = tmp_path_factory.mktemp("scenes")
    os.environ.setdefault("ATRC_SCENE_CACHE", str(d))
    return d


@pytest.fixture(scope="session")
def cornell_path(scene_dir):
    from atrc_b200.scenes import cornell_box
    return cornell_box(scene_dir / "cornell", spp=16)
