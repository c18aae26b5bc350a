"""Shared fixtures.  ``-m gpu`` tests need a CUDA device and the built library."""

import pathlib
import sys

import numpy as np
import pytest
import torch

REPO = pathlib.Path(__file__).resolve().parent.parent
if str(REPO) not in sys.path:
    sys.path.insert(0, str(REPO))

GOLDEN = pathlib.Path(__file__).resolve().parent / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libpygrog_b200.so")


def golden(name: str) -> dict:
    with np.load(GOLDEN / name, allow_pickle=False) as z:
        return {k: z[k] for k in z.files}


def golden_plan_cases():
    return sorted(p.name for p in GOLDEN.glob("plan_*.npz"))


def parse_meta(arr):
    import ast

    return ast.literal_eval(str(arr[0]))


@pytest.fixture
def rng():
    return np.random.default_rng(42)


@pytest.fixture(scope="session")
def cuda():
    if not torch.cuda.is_available():
        pytest.skip("CUDA not available")
    import pygrog_b200

    pygrog_b200.load_library()
    return torch.device("cuda")


def rel_l2(a, b) -> float:
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-30))
