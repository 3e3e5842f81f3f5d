"""MRC file handling of the drop-in executables (autom2_b200/cli/mrc_io.cpp)
on the CPU.

The executables read the reference's input stacks (MRC modes 0, 1 and 2, with
or without an extended header) and write volumes whose headers carry the
reference's InitializeHeader fields and UpdateHeader statistics
(src/TiltRec/src/mrcmx/mrcstack.cpp:57-86, 104-142).  mrc_io.cpp is compiled
here into a small test library and checked against numpy on files written in
a temporary directory; the GPU CLI tests compare whole output files with the
reference executables.
"""
import ctypes as C
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

CLI = Path(__file__).resolve().parents[1] / "autom2_b200" / "cli"

WRAP = r"""
#include <string.h>
#include "mrc_io.h"
using namespace trcli;
static std::string g_err;
extern "C" {
const char *probe_err() { return g_err.c_str(); }
int probe_read_header(const char *p, MrcHeader *h) { return read_header(p, h, &g_err); }
int probe_read_sections(const char *p, const MrcHeader *h, int z0, int z1, int sgn,
                        float *out) {
  return read_sections(p, *h, z0, z1, sgn != 0, out, &g_err);
}
void probe_new_header(int nx, int ny, int nz, int byte_mode, MrcHeader *h) {
  *h = new_volume_header(nx, ny, nz, byte_mode != 0);
}
void probe_update_stats(MrcHeader *h, const float *s, size_t n) { update_stats(h, s, n); }
int probe_write_volume(const char *p, const MrcHeader *h, const void *d, size_t b) {
  return write_volume(p, *h, d, b, &g_err);
}
int probe_write_ext(const char *p, const MrcHeader *h, const float *d, size_t n) {
  return write_with_extended(p, *h, d, n, &g_err);
}
int probe_read_angles(const char *p, float *out, int cap) {
  std::vector<float> a;
  if (!read_angles(p, &a, &g_err)) return -1;
  for (int i = 0; i < (int)a.size() && i < cap; ++i) out[i] = a[i];
  return (int)a.size();
}
int probe_header_size() { return (int)sizeof(MrcHeader); }
}
"""

# The MRC header's fields as numpy reads them (1024 bytes, little endian).
HDR = np.dtype([
    ("nx", "<i4"), ("ny", "<i4"), ("nz", "<i4"), ("mode", "<i4"),
    ("start", "<i4", 3), ("m", "<i4", 3), ("len", "<f4", 3), ("ang", "<f4", 3),
    ("map", "<i4", 3), ("amin", "<f4"), ("amax", "<f4"), ("amean", "<f4"),
    ("ispg", "<i2"), ("nsymbt", "<i2"), ("next", "<i4"), ("creatid", "<i2"),
    ("blank", "V30"), ("nint", "<i2"), ("nreal", "<i2"), ("sub", "<i2"), ("zfac", "<i2"),
    ("mm", "<f4", 6), ("idtype", "<i2", 6), ("tilt", "<f4", 6), ("org", "<f4", 3),
    ("cmap", "S4"), ("stamp", "S4"), ("rms", "<f4"), ("nlabl", "<i4"), ("labels", "V800"),
])


class Hdr(C.Structure):
    _fields_ = [("raw", C.c_ubyte * 1024)]

    def view(self):
        return np.frombuffer(bytes(self.raw), HDR)[0]


@pytest.fixture(scope="module")
def mrc(tmp_path_factory):
    cxx = shutil.which("g++")
    assert cxx, "g++ is needed to compile the MRC module for this test"
    d = tmp_path_factory.mktemp("mrcprobe")
    (d / "wrap.cpp").write_text(WRAP)
    so = d / "mrc.so"
    subprocess.run([cxx, "-O2", "-std=c++17", "-shared", "-fPIC", f"-I{CLI}",
                    str(d / "wrap.cpp"), str(CLI / "mrc_io.cpp"), "-o", str(so)], check=True)
    lib = C.CDLL(str(so))
    lib.probe_err.restype = C.c_char_p
    lib.probe_update_stats.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t]
    lib.probe_write_volume.argtypes = [C.c_char_p, C.c_void_p, C.c_void_p, C.c_size_t]
    lib.probe_write_ext.argtypes = [C.c_char_p, C.c_void_p, C.c_void_p, C.c_size_t]
    assert lib.probe_header_size() == 1024 == HDR.itemsize
    return lib


def write_stack(path, data, mode, next_bytes=0):
    """An input stack as another program would write it: header, `next`
    bytes of extended header, then sections [nz][ny][nx]."""
    h = np.zeros((), HDR)
    h["nz"], h["ny"], h["nx"] = data.shape
    h["mode"], h["next"] = mode, next_bytes
    dt = {0: np.uint8, 1: "<i2", 2: "<f4"}[mode]
    with open(path, "wb") as f:
        f.write(h.tobytes())
        f.write(b"\x7f" * next_bytes)
        f.write(np.ascontiguousarray(data).astype(dt).tobytes())


@pytest.mark.parametrize("mode,next_bytes", [(0, 0), (1, 0), (2, 0), (2, 3072), (0, 131)])
def test_read_sections(mrc, tmp_path, mode, next_bytes):
    rng = np.random.default_rng(mode * 10 + next_bytes)
    nz, ny, nx = 7, 5, 9
    if mode == 0:
        data = rng.integers(0, 256, (nz, ny, nx))
    elif mode == 1:
        data = rng.integers(-32768, 32768, (nz, ny, nx))
    else:
        data = rng.normal(size=(nz, ny, nx)).astype(np.float32)
    p = str(tmp_path / "s.mrc").encode()
    write_stack(p.decode(), data, mode, next_bytes)
    h = Hdr()
    assert mrc.probe_read_header(p, C.byref(h)) == 1, mrc.probe_err()
    assert (h.view()["nx"], h.view()["ny"], h.view()["nz"]) == (nx, ny, nz)
    for z0, z1 in ((0, nz), (2, 5), (6, 7)):
        for sgn in (0, 1):
            out = np.full((z1 - z0, ny, nx), np.nan, np.float32)
            assert mrc.probe_read_sections(p, C.byref(h), z0, z1, sgn,
                                           out.ctypes.data_as(C.c_void_p)) == 1
            want = data[z0:z1].astype(np.float64)
            if mode == 0 and sgn:  # mode 0 bytes as signed char
                want = np.where(want > 127, want - 256, want)
            np.testing.assert_array_equal(out, want.astype(np.float32))


def test_bad_files_are_errors(mrc, tmp_path):
    h = Hdr()
    p = tmp_path / "x.mrc"
    p.write_bytes(b"\0" * 100)
    assert mrc.probe_read_header(str(p).encode(), C.byref(h)) == 0
    assert b"short" in mrc.probe_err()
    write_stack(str(p), np.zeros((2, 2, 2)), 2)
    raw = bytearray(p.read_bytes())
    raw[12:16] = np.int32(6).tobytes()  # mode 6 is not read by the reference either
    p.write_bytes(bytes(raw))
    assert mrc.probe_read_header(str(p).encode(), C.byref(h)) == 0
    assert b"mode" in mrc.probe_err()
    assert mrc.probe_read_header(str(tmp_path / "missing.mrc").encode(), C.byref(h)) == 0
    # a stack shorter than its header says
    write_stack(str(p), np.zeros((2, 2, 2)), 2)
    raw = bytearray(p.read_bytes())
    raw[8:12] = np.int32(3).tobytes()
    p.write_bytes(bytes(raw))
    assert mrc.probe_read_header(str(p).encode(), C.byref(h)) == 1
    out = np.zeros((3, 2, 2), np.float32)
    assert mrc.probe_read_sections(str(p).encode(), C.byref(h), 0, 3, 0,
                                   out.ctypes.data_as(C.c_void_p)) == 0


def test_new_volume_header_is_initialize_header(mrc):
    h = Hdr()
    for byte_mode in (0, 1):
        mrc.probe_new_header(11, 13, 17, byte_mode, C.byref(h))
        v = h.view()
        assert (v["nx"], v["ny"], v["nz"], v["mode"]) == (11, 13, 17, 0 if byte_mode else 2)
        assert list(v["m"]) == [1, 1, 1] and list(v["len"]) == [1, 1, 1]
        assert list(v["ang"]) == [90, 90, 90] and list(v["map"]) == [1, 2, 3]
        assert (v["amin"], v["amax"], v["amean"]) == (0, 255, 128)
        assert v["creatid"] == 1000 and v["next"] == 0


def test_update_stats_quirks(mrc):
    """UpdateHeader's statistics: the running maximum starts at FLT_MIN, the
    smallest positive float, so a section of negative values reports it; the
    mean accumulates in long double."""
    h = Hdr()
    mrc.probe_new_header(4, 4, 4, 0, C.byref(h))
    rng = np.random.default_rng(0)
    s = rng.normal(size=1000).astype(np.float32)
    mrc.probe_update_stats(C.byref(h), s.ctypes.data, s.size)
    v = h.view()
    assert v["amin"] == s.min() and v["amax"] == s.max()
    assert v["amean"] == np.float32(np.sum(s.astype(np.longdouble)) / s.size)
    neg = -np.abs(s) - 1
    mrc.probe_update_stats(C.byref(h), neg.ctypes.data, neg.size)
    v = h.view()
    assert v["amax"] == np.finfo(np.float32).tiny and v["amin"] == neg.min()


def test_write_then_read(mrc, tmp_path):
    h = Hdr()
    vol = np.random.default_rng(1).normal(size=(3, 4, 5)).astype(np.float32)
    mrc.probe_new_header(5, 4, 3, 0, C.byref(h))
    p = str(tmp_path / "v.mrc").encode()
    assert mrc.probe_write_volume(p, C.byref(h), vol.ctypes.data, vol.nbytes) == 1
    raw = open(p, "rb").read()
    assert len(raw) == 1024 + vol.nbytes
    np.testing.assert_array_equal(np.frombuffer(raw[1024:], "<f4").reshape(vol.shape), vol)
    # with an extended header of zeros
    raw_h = bytearray(bytes(h.raw))
    raw_h[92:96] = np.int32(256).tobytes()  # next
    h2 = Hdr.from_buffer_copy(bytes(raw_h))
    assert h2.view()["next"] == 256
    assert mrc.probe_write_ext(p, C.byref(h2), vol.ctypes.data, vol.size) == 1
    raw = open(p, "rb").read()
    assert raw[1024:1280] == b"\0" * 256
    out = np.zeros_like(vol)
    assert mrc.probe_read_sections(p, C.byref(h2), 0, 3, 0, out.ctypes.data_as(C.c_void_p)) == 1
    np.testing.assert_array_equal(out, vol)


def test_read_angles_stops_at_the_first_bad_token(mrc, tmp_path):
    p = tmp_path / "a.tlt"
    p.write_text("-60.0\n -57.5\t-55\n1e1 x 12\n")
    out = np.zeros(16, np.float32)
    n = mrc.probe_read_angles(str(p).encode(), out.ctypes.data_as(C.c_void_p), 16)
    assert n == 4 and list(out[:4]) == [-60.0, -57.5, -55.0, 10.0]
    assert mrc.probe_read_angles(str(tmp_path / "none.tlt").encode(),
                                 out.ctypes.data_as(C.c_void_p), 16) == -1
