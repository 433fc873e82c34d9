import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "ispm-sparse-lib_b200")
for p in (PKG, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def ispm():
    import ispm as m
    m.lib_handle()  # fails loudly when libispm_b200.so is missing
    return m


@pytest.fixture(scope="session")
def gen():
    import ispm.gen as g
    return g


@pytest.fixture(scope="session")
def oracle():
    import oracle as o
    o.orc()
    return o


@pytest.fixture(scope="session")
def ref(oracle):
    """The reference's host code compiled in place (oracle/_ref)."""
    if not oracle.have_ref():
        try:
            oracle.build()
        except Exception:
            pass
    if not oracle.have_ref():
        pytest.skip("oracle/_ref not built (reference source tree absent)")
    oracle.ref()
    return oracle


@pytest.fixture(scope="session")
def cuda(ispm):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    torch.cuda.init()
    ispm.ispm_initialize()
    return torch


def copy_csr(ispm, A):
    return ispm.csr_matrix(A.n_rows, A.n_cols, A.row_ptr.copy(), A.cols.copy(), A.elms.copy())
