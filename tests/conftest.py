import os
import sys

import numpy
import pytest
import torch

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def pytest_collection_modifyitems(config, items):
    if torch.cuda.is_available():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


def load_golden(name):
    return dict(numpy.load(os.path.join(GOLDEN, name), allow_pickle=False))


@pytest.fixture(scope="session")
def term():
    from tmol_b200.score.ljlk_energy_term import LJLKEnergyTerm

    return LJLKEnergyTerm()


@pytest.fixture(scope="session")
def ubq_golden():
    return load_golden("ubq.npz")


@pytest.fixture(scope="session")
def ubq_pose_stack(ubq_golden):
    from tmol_b200.pose.builder import build_pose_stack, PoseTopology

    names = [str(n) for n in ubq_golden["block_type_names"]]
    topo = PoseTopology(names, [(i, "up", i + 1, "down") for i in range(len(names) - 1)])
    return build_pose_stack([topo], [ubq_golden["coords"]])


@pytest.fixture(scope="session")
def synthetic_golden():
    return load_golden("synthetic.npz")


@pytest.fixture(scope="session")
def synthetic_pose_stack_golden(synthetic_golden):
    from tmol_b200.pose.synthetic import synthetic_pose_stack

    ps = synthetic_pose_stack(list(synthetic_golden["sizes"]), list(synthetic_golden["seeds"]))
    # the fixture's coordinates are the ones the reference scored
    ps.coords = torch.tensor(synthetic_golden["coords"])
    return ps
