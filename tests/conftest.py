"""Shared fixtures.  Tests marked ``gpu`` need a CUDA device (B200); all
others run on the CPU.  The oracle (``oracle/``) is the checker here."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden", "golden.npz")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (runs on the B200)")


@pytest.fixture(scope="session")
def cuda_include():
    """The CUDA toolkit's include directory (beside the nvcc the library is
    built with), for host-only test builds of headers that include it."""
    from autom2_b200 import build
    inc = os.path.join(os.path.dirname(os.path.dirname(os.path.realpath(build.nvcc()))),
                       "include")
    assert os.path.exists(os.path.join(inc, "cuda_runtime.h")), inc
    return inc


@pytest.fixture(scope="session")
def golden():
    with np.load(GOLDEN) as z:
        return {k: z[k] for k in z.files}


@pytest.fixture(scope="session")
def restatement():
    import oracle
    return oracle.Restatement()


@pytest.fixture(scope="session")
def reference():
    import oracle
    if not oracle.reference_available():
        pytest.skip("oracle/_ref (the compiled reference) is not built here")
    return oracle.Reference()


@pytest.fixture(scope="session")
def engine():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("gpu test collected without a CUDA device")
    from autom2_b200 import build
    build.build_lib()
    from autom2_b200.tiltrec import Engine
    eng = Engine(0)
    yield eng
    eng.close()
