"""Shared fixtures. GPU tests carry ``@pytest.mark.gpu``; everything else runs
on a CPU-only machine."""
from __future__ import annotations

import importlib
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built libwinds_bs.so")


@pytest.fixture(scope="session")
def wb():
    pkg = importlib.import_module("winds-master_b200")
    pkg.lib()  # raises when the library is not built
    return pkg


@pytest.fixture(scope="session")
def synth():
    return importlib.import_module("winds-master_b200.synth")


@pytest.fixture(scope="session")
def oracle():
    import oracle as orc
    return orc


@pytest.fixture(scope="session")
def ref():
    import biot_savart_ref
    return biot_savart_ref


def load_golden(name):
    return dict(np.load(os.path.join(GOLDEN, name), allow_pickle=False))


def per_target_rel(u, u_ref):
    """max_i |u_i - u_ref_i| / |u_ref_i| over targets of [n,3,...] arrays."""
    a = np.stack([np.asarray(u)[:, c].ravel(order="F") for c in range(3)], 1)
    b = np.stack([np.asarray(u_ref)[:, c].ravel(order="F") for c in range(3)], 1)
    num = np.linalg.norm(a - b, axis=1)
    den = np.linalg.norm(b, axis=1)
    ok = den > 0
    worst = np.max(num[ok] / den[ok]) if ok.any() else 0.0
    zero_err = np.max(num[~ok]) if (~ok).any() else 0.0
    return max(worst, zero_err)
