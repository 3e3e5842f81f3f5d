"""The C-ABI library: symbols, host-only geometry and error behaviour (CPU)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from autom2_b200 import build, tiltrec

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def lib():
    build.build_lib()
    return tiltrec.load_library()


def _declared(header):
    text = open(os.path.join(ROOT, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(tr_\w+)\s*\(", text)))


def test_exports_every_declared_symbol(lib):
    names = []
    for h in os.listdir(os.path.join(ROOT, "include")):
        if h.endswith(".h"):
            names += _declared(h)
    assert len(names) >= 15
    for n in names:
        assert hasattr(lib, n), n


def test_header_constants_match_the_wrapper():
    """The method codes and the zero-start flag the Python wrapper passes are
    the header's."""
    from autom2_b200 import tiltrec as T
    text = open(os.path.join(ROOT, "include", "tiltrec_b200.h")).read()
    flag = re.search(r"#define\s+TR_RECON_ZERO_START\s+(0x[0-9a-fA-F]+|\d+)", text)
    assert flag and int(flag.group(1), 0) == T.RECON_ZERO_START
    for name, code in re.findall(r"TR_METHOD_(\w+)\s*=\s*(\d+)", text):
        assert T.METHODS[name] == int(code), name
    assert not (T.RECON_ZERO_START & max(T.METHODS.values()))


def test_geometry_matches_reference_vectors(golden, lib):
    ang = golden["geom/angles"]
    for par, c20 in zip(golden["geom/params"], golden["geom/coeff20"]):
        c8 = tiltrec.geometry_from_angles(ang, *par)
        np.testing.assert_array_equal(c8, c20[:, [0, 1, 2, 3, 10, 11, 12, 13]])


def test_status_strings(lib):
    for s in range(0, -8, -1):
        assert lib.tr_status_string(s)
    assert lib.tr_version() >= 10000


def test_errors_without_device_or_problem(lib):
    h = C.c_void_p()
    assert lib.tr_create(-1, 0, C.byref(h)) == -1  # TR_ERR_ARG, no exit
    assert lib.tr_geometry_from_angles(None, 3, 0, 0, 0, None) == -1
    assert lib.tr_set_problem(None, 8, 8, 1, 4, 0, None, 0, 0, 0) == -1
    assert lib.tr_sirt(None, None, None, 1, 0.5, None) == -1
    lib.tr_sched_set_aging.argtypes = [C.c_void_p, C.c_double]
    assert lib.tr_sched_set_aging(None, 1.0) == -1
    assert lib.tr_sched_set_policy(None, 1) == -1
    lib.tr_set_deterministic.argtypes = [C.c_void_p, C.c_int]
    assert lib.tr_set_deterministic(None, 1) == -1
    lib.tr_sirt_gated.argtypes = [C.c_void_p] * 3 + [C.c_int, C.c_float, C.c_double,
                                                   C.c_void_p, C.c_void_p, C.c_void_p]
    assert lib.tr_sirt_gated(None, None, None, 3, 0.5, 0.0, None, None, None) == -1
    lib.tr_sirt_host_zslabs.argtypes = [C.c_void_p] * 3 + [C.c_int, C.c_int, C.c_float,
                                                         C.c_int, C.c_void_p]
    assert lib.tr_sirt_host_zslabs(None, None, None, 1, 2, 0.5, 0, None) == -1
    lib.tr_host_alloc.argtypes = [C.c_size_t, C.c_void_p]
    assert lib.tr_host_alloc(16, None) == -1
    lib.tr_sirt_zslabs.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_int,
                                   C.c_void_p, C.c_int, C.c_int, C.c_float, C.c_int,
                                   C.c_void_p]
    assert lib.tr_sirt_zslabs(None, None, 0, None, 0, None, 0, 1, 0.5, 32, None) == -1


def test_engine_fails_loudly_without_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(tiltrec.TiltRecError):
        tiltrec.Engine(0)
