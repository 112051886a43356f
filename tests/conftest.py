import os
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.join(REPO, "oracle"))
GOLDEN = os.path.join(REPO, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and libpq3d.so")


@pytest.fixture(scope="session")
def gf_golden():
    return dict(np.load(os.path.join(GOLDEN, "gf_cases.npz")))


@pytest.fixture(scope="session")
def tiny_golden():
    return dict(np.load(os.path.join(GOLDEN, "tiny_case.npz")))


@pytest.fixture(scope="session")
def tiny_files(tmp_path_factory, tiny_golden):
    """The reference's tiny case written back to disk (msh, dat, parameter.txt)."""
    d = tmp_path_factory.mktemp("tiny")
    (d / "tiny.msh").write_text(str(tiny_golden["msh"]))
    (d / "tinyparam.dat").write_text(str(tiny_golden["param_dat"]))
    (d / "parameter.txt").write_text(str(tiny_golden["parameter_txt"]))
    return str(d / "tiny.msh"), str(d / "parameter.txt")


@pytest.fixture(scope="session")
def tiny_sim(tiny_files):
    from pyquake3d_b200 import QDsim, read_mshV2
    msh, para = tiny_files
    nodes, tris = read_mshV2(msh)
    return QDsim(tris, nodes, para)
