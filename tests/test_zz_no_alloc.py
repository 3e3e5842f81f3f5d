"""tr_sirt_static: the SIRT entry point that allocates no device memory.

It serves callers that cannot call cudaMalloc where they reconstruct (a
process whose memory pool already owns its device memory, or a stream-ordered
pipeline that must not take an allocation's device-wide synchronisation).
Its scratch is a 64 MiB static device array shared by every call.  This file
is collected last so that a failure here comes after every other test; it
passes alone in a fresh process as well as after the rest."""
import numpy as np
import pytest
import torch

import oracle as O
from autom2_b200 import tiltrec as T

pytestmark = pytest.mark.gpu
TOL = 1e-5  # the parity tolerance used by every GPU test


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()


def test_static_sirt_matches_context_sirt_twice(golden):
    nx, ny, nt, th = (int(v) for v in golden["cfg0s4/dims"])
    org = tuple(float(v) for v in golden["cfg0s4/origin"])
    c8 = golden["cfg0s4/coeff8"]
    proj = _dev(golden["cfg0s4/proj"])
    eng = T.Engine(0)
    eng.set_problem(nx, ny, nt, th, c8, T.LAYOUT_Y, org)
    want = torch.zeros((ny, th, nx), device="cuda")
    eng.sirt(proj, want, 5, 0.5)
    torch.cuda.synchronize()
    want = want.cpu().numpy()
    eng.close()
    vol = torch.zeros((ny, th, nx), device="cuda")
    for k in range(2):  # the second call starts from the first call's scratch
        vol.zero_()
        torch.cuda.synchronize()
        # Device memory free before and after the call (driver view: every
        # cudaMalloc of the process shows; torch allocates nothing here, the
        # tensors exist already).
        free0 = torch.cuda.mem_get_info()[0]
        T.sirt_static(proj, vol, c8, 5, 0.5, T.LAYOUT_Y, org)
        torch.cuda.synchronize()
        free1 = torch.cuda.mem_get_info()[0]
        if k == 1:  # the first call may load the library's device code
            assert free1 == free0, f"the call changed free device memory by {free0 - free1} B"
        got = vol.cpu().numpy()
        assert O.rel_l2(got, want) < TOL
        assert O.rel_l2(got, golden["cfg0s4/sirt5"]) < TOL
    assert T.static_take_timeout() == 0  # no device wait gave up


def test_static_sirt_rejects_problems_beyond_its_scratch():
    limit = T.static_scratch_limit()
    assert limit == 64 << 20
    nx = ny = 1024
    nt, th = 61, 64  # 2*61*1024^2*4 B of projection scratch alone > 64 MiB
    proj = torch.zeros((nt, 1, 1), device="cuda")  # never touched: rejected first
    vol = torch.zeros((1, 1, 1), device="cuda")
    c8 = np.tile([0, 1, 0, 0, 0, 0, 1, 0.0], (nt, 1))
    lib = T.load_library()
    fn = lib.tr_sirt_static
    import ctypes as C
    fn.argtypes = [C.c_int] * 6 + [C.POINTER(C.c_double)] + [C.c_float] * 3 + \
        [C.c_void_p, C.c_void_p, C.c_int, C.c_float, C.c_void_p]
    st = fn(0, nx, ny, nt, th, 0, np.ascontiguousarray(c8).ctypes.data_as(C.POINTER(C.c_double)),
            512.0, 32.0, 32.0, proj.data_ptr(), vol.data_ptr(), 1, 0.5, None)
    assert st == -3  # TR_ERR_BUDGET


def test_static_sirt_reports_a_device_wait_that_gave_up():
    # A bounded wait on a barrier nothing completes (50 ms), reporting through
    # the static scratch as a back-projection does; the report stays until it
    # is read, and reading clears it.
    assert T.static_selftest_wait(50_000) == -5  # TR_ERR_TIMEOUT
    assert T.static_take_timeout() == 0


def test_static_sirt_rejects_non_finite_coefficients():
    nt, ny, nx, th = 3, 8, 16, 4
    c8 = np.tile([0, 1, 0, 0, 0, 0, 1, 0.0], (nt, 1))
    c8[1, 3] = np.nan
    proj = torch.zeros((nt, ny, nx), device="cuda")
    vol = torch.zeros((ny, th, nx), device="cuda")
    with pytest.raises(T.TiltRecError) as e:
        T.sirt_static(proj, vol, c8, 1, 0.5, T.LAYOUT_Y)
    assert e.value.status == -1  # TR_ERR_ARG, as tr_set_problem
