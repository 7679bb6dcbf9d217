"""Shared fixtures.  GPU tests carry @pytest.mark.gpu and run only on a B200
box (``pytest -m gpu``); everything else runs on CPU (``-m "not gpu"``)."""
from __future__ import annotations

import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def _cuda_ok() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _cuda_ok():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


def _cases(npz):
    names = sorted({k.split("/")[0] for k in npz.files})
    return {nm: {k.split("/", 1)[1]: npz[k] for k in npz.files if k.startswith(nm + "/")}
            for nm in names}


@pytest.fixture(scope="session")
def spmv_golden():
    return _cases(np.load(os.path.join(GOLDEN, "spmv_cases.npz")))


@pytest.fixture(scope="session")
def cg_golden():
    return _cases(np.load(os.path.join(GOLDEN, "cg_cases.npz")))


@pytest.fixture(scope="session")
def rcm_golden():
    return _cases(np.load(os.path.join(GOLDEN, "rcm_cases.npz")))


@pytest.fixture(scope="session")
def full_golden():
    with open(os.path.join(GOLDEN, "full_sizes.json")) as f:
        return json.load(f)


def cond_scaled_err(y, y_ref, rowptr, rowind, rowval, x):
    """max_i |y_i - yref_i| / sum_k |a_ik x_k|  (rows with an all-zero scale
    must match exactly: their scaled error is reported as |diff| / tiny)."""
    import scipy.sparse as sp
    n = len(rowptr) - 1
    A = sp.csr_matrix((np.abs(rowval).astype(np.float64), rowind.astype(np.int64),
                       rowptr.astype(np.int64)), shape=(n, len(x)))
    scale = A @ np.abs(x.astype(np.float64))
    diff = np.abs(y.astype(np.float64) - y_ref.astype(np.float64))
    return float(np.max(diff / np.maximum(scale, 1e-300))) if n else 0.0
