import os
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)
GOLDEN = os.path.join(REPO, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def fixture_names(prefix=""):
    return sorted(f[:-4] for f in os.listdir(GOLDEN) if f.endswith(".npz") and f.startswith(prefix))


def load_fixture(name):
    from jaxley_pytorch_b200.problem import load_problem

    return load_problem(os.path.join(GOLDEN, f"{name}.npz"))


@pytest.fixture(scope="session")
def cuda_device():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from jaxley_pytorch_b200 import _lib

    _lib.load()  # fail loudly if the library is missing on a GPU machine
    return torch.device("cuda:0")


def import_reference():
    """The reference package (jaxley-pytorch) for the drop-in tests: from
    `JXB_REFERENCE` when set, else the copy installed under `baseline/_ref`; its
    module-level matplotlib import (plotting only) is served by the stand-in package
    under `tests/golden/_mpl_stub`. Skips when neither is present."""
    import importlib

    path = os.environ.get("JXB_REFERENCE") or os.path.join(REPO, "baseline", "_ref")
    if not os.path.isdir(os.path.join(path, "jaxley_pytorch")):
        pytest.skip("the reference package is not installed here")
    for p in (os.path.join(GOLDEN, "_mpl_stub"), path):
        if p not in sys.path:
            sys.path.insert(0, p)
    return importlib.import_module("jaxley_pytorch")
