"""The R-weighting filter's host-side spectrum (tr_filter_host.h), on the CPU.

WBP's filter (ApplyFilterInplace mode 2, src/TiltRec/src/filter/
filter_prj.cpp:674-736) pads each row to N = nx + nx/10 with a linear ramp,
weights its length-N spectrum and crops.  That is a circular convolution of
the padded row with a fixed kernel h, and the device evaluates it as a linear
convolution through an M-point power-of-two FFT, multiplying by a kernel
spectrum that the host forms in double precision (rweight_spectrum).  Here
the header is compiled as host C++, the device's convolution is replayed in
numpy with that spectrum, and the result is compared with the oracle's direct
double-precision evaluation of the reference's chain (itself pinned to the
reference's own filter).  The Stockham twiddle tables are checked too.
"""
import ctypes as C
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

import oracle as O

CSRC = Path(__file__).resolve().parents[1] / "autom2_b200" / "csrc"

PROBE = r"""
#include "tr_filter_host.h"
extern "C" int probe_spectrum(int nx, size_t smem_max, int *npad, int *log2m,
                              float *ghat, int ghat_cap, float *tw, int tw_cap, int *ntw) {
  trb::RweightSpectrum s;
  if (!trb::rweight_spectrum(nx, smem_max, &s)) return 0;
  *npad = s.npad;
  *log2m = s.log2m;
  if ((int)s.ghat.size() > ghat_cap || (int)s.tw.size() > tw_cap) return -1;
  for (size_t i = 0; i < s.ghat.size(); ++i) {
    ghat[2 * i] = s.ghat[i].x;
    ghat[2 * i + 1] = s.ghat[i].y;
  }
  for (size_t i = 0; i < s.tw.size(); ++i) {
    tw[2 * i] = s.tw[i].x;
    tw[2 * i + 1] = s.tw[i].y;
  }
  *ntw = (int)s.tw.size();
  return 1;
}
"""

CAP = 1 << 16


@pytest.fixture(scope="module")
def spectrum(tmp_path_factory, cuda_include):
    cxx = shutil.which("g++")
    assert cxx, "g++ is needed to compile the filter header for this test"
    d = tmp_path_factory.mktemp("rwprobe")
    (d / "p.cpp").write_text(PROBE)
    so = d / "p.so"
    subprocess.run([cxx, "-O2", "-std=c++17", "-shared", "-fPIC", f"-I{CSRC}",
                    f"-I{cuda_include}", str(d / "p.cpp"), "-o", str(so)], check=True)
    lib = C.CDLL(str(so))

    def get(nx, smem_max=227 * 1024):
        npad, log2m, ntw = C.c_int(), C.c_int(), C.c_int()
        g = np.zeros(2 * CAP, np.float32)
        tw = np.zeros(2 * CAP, np.float32)
        ok = lib.probe_spectrum(nx, C.c_size_t(smem_max), C.byref(npad), C.byref(log2m),
                                g.ctypes.data_as(C.c_void_p), CAP,
                                tw.ctypes.data_as(C.c_void_p), CAP, C.byref(ntw))
        if ok != 1:
            return None
        m = 1 << log2m.value
        return (npad.value, log2m.value, g[:2 * m].view(np.complex64).astype(np.complex128),
                tw[:2 * ntw.value].view(np.complex64))
    return get


def device_filter(rows, npad, ghat):
    """The device's evaluation: the ramp-padded row, zero-extended to M
    points, times the kernel spectrum, inverse transformed (the spectrum
    carries 1/(M nx)), first nx outputs."""
    nrow, nx = rows.shape
    m = ghat.size
    x = np.zeros((nrow, m))
    x[:, :nx] = rows
    nxp = npad - nx + 1
    j = np.arange(nx, npad)
    x[:, nx:npad] = ((j - nx + 1) / nxp)[None, :] * rows[:, :1] + \
        ((npad - j) / nxp)[None, :] * rows[:, -1:]
    y = np.fft.ifft(np.fft.fft(x, axis=1) * ghat[None, :], axis=1) * m
    return y[:, :nx].real


@pytest.mark.parametrize("nx", [16, 100, 256, 257, 1000, 1024, 2048, 4096])
def test_spectrum_reproduces_the_reference_filter(spectrum, nx):
    s = spectrum(nx)
    assert s is not None
    npad, log2m, ghat, _ = s
    assert npad == nx + nx // 10
    assert (1 << log2m) >= npad + nx - 1 > (1 << (log2m - 1)) or log2m == 4
    rng = np.random.default_rng(nx)
    rows = rng.normal(size=(4, nx)).astype(np.float32)
    rows[1] += 3.0  # an offset row: the ramp pad matters
    want = O.Restatement().filter_rweight(rows.copy())
    got = device_filter(rows.astype(np.float64), npad, ghat)
    err = np.linalg.norm(got - want) / np.linalg.norm(want)
    assert err < 2e-6, f"nx {nx}: rel-L2 {err:.2e} against the oracle's direct evaluation"


def test_twiddle_tables(spectrum):
    for nx in (256, 1024, 4096):
        npad, log2m, _, tw = spectrum(nx)
        want = []
        for ls in range(log2m & 3, log2m, 4):
            if ls == 0:
                continue
            ns = 1 << ls
            r, k = np.meshgrid(np.arange(1, 16), np.arange(ns), indexing="ij")
            want.append(np.exp(-2j * np.pi * r * k / (16 * ns)).ravel())
        want = np.concatenate(want) if want else np.array([1 + 0j])
        np.testing.assert_allclose(tw, want, atol=1e-7)


def test_sizes_beyond_the_device_fft_are_refused(spectrum):
    assert spectrum(4096) is not None
    assert spectrum(9000) is None  # M = 2^15 is beyond the largest FFT
    assert spectrum(4096, smem_max=64 * 1024) is None  # 16384 points need ~136 KB
