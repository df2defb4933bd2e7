"""Shared pytest configuration: the ``gpu`` marker and fixture loading."""

import json
import os
import sys

# one BLAS thread, as the golden fixtures were made: the oracle then
# reproduces the reference's floating-point trajectory exactly
os.environ.setdefault("OPENBLAS_NUM_THREADS", "1")

import numpy as np  # noqa: E402
import pytest
from threadpoolctl import threadpool_limits

# a pytest plugin may have loaded NumPy before this file, so the variable
# above can come too late; cap the BLAS pool directly as well
threadpool_limits(1)

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def load_golden(name: str) -> dict:
    """Load ``tests/golden/<name>.npz`` into a plain dict."""
    with np.load(os.path.join(GOLDEN, f"{name}.npz"), allow_pickle=False) as f:
        data = {k: f[k] for k in f.files}
    data["args"] = json.loads(str(data.pop("args_json")))
    return data


def golden_train(data: dict, name: str):
    """Cores and orthogonality centre of train ``name`` from a fixture."""
    n = int(data[f"{name}_n"])
    oc = int(data[f"{name}_oc"])
    return [data[f"{name}_{k}"] for k in range(n)], (None if oc < 0 else oc)


@pytest.fixture
def golden():
    return load_golden
