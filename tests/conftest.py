import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the device kernels")
    config.addinivalue_line("markers", "slow: long-running CPU test")


@pytest.fixture(scope="session")
def scene_dir(tmp_path_factory):
    return tmp_path_factory.mktemp("scenes")


@pytest.fixture(scope="session")
def mixed_nls(scene_dir):
    from lambda_b200 import synth
    return synth.mixed(os.path.join(str(scene_dir), "mixed"))


@pytest.fixture(scope="session")
def mixed2_nls(scene_dir):
    from lambda_b200 import synth
    return synth.mixed(os.path.join(str(scene_dir), "mixed2"), lights=("direction", "ambient", "quaddir"),
                       seed=11)


@pytest.fixture(scope="session")
def box_nls(scene_dir):
    from lambda_b200 import synth
    return synth.box_room(os.path.join(str(scene_dir), "box"), width=64)
