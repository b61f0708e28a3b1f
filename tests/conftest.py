import os
import pathlib
import sys

import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
for p in (ROOT, ROOT / "tca-spmm_b200" / "python"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))

# The reference project's tree (only for the tests that read its files; they
# skip when it is not given): the environment variable TCA_REFERENCE_ROOT.
_ref_env = os.environ.get("TCA_REFERENCE_ROOT")
REFERENCE_TREE = pathlib.Path(_ref_env) if _ref_env else None


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def golden():
    import numpy as np
    return np.load(ROOT / "tests" / "golden" / "golden.npz")


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")
