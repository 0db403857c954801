import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def oracle():
    import pyoracle
    pyoracle.build()
    return pyoracle


@pytest.fixture(scope="session")
def gpu_ctx():
    if not has_gpu():
        pytest.skip("no CUDA device")
    from gerjoii_b200 import _native
    ctx = _native.Context(0)
    yield ctx
    ctx.close()


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


def edge_cells(a):
    """The model's edge cells (first and last row and column) of an m x n
    array (or of the last two axes): the cells whose eps_r the PML replicates
    (w_exp2pml.m:21-33), where the exact gradient collects the derivatives of
    the PML coefficients."""
    a = np.asarray(a)
    m, n = a.shape[-2:]
    msk = np.zeros((m, n), bool)
    msk[0, :] = msk[-1, :] = msk[:, 0] = msk[:, -1] = True
    return a[..., msk]


def cosine(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    return float(a @ b / (np.linalg.norm(a) * np.linalg.norm(b)))
