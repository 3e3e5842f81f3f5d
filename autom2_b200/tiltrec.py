"""Python host binding of the TiltRec B200 engine (ctypes over the C ABI in
``include/tiltrec_b200.h``).

It mirrors the reference's reconstruction interface for this path:

==========================  ==================================================
reference                   here
==========================  ==================================================
TranslateAngleToCoefficients + DecorateCoefficients
  (main/main-mpi.cpp:85-183)  :func:`geometry_from_angles`
ApplyFilterInplace mode 2    :meth:`Engine.filter_rweight`
  (filter/filter_prj.cpp:738)
BackProject                  :meth:`Engine.backproject`
  (main-mpi.cpp:411; main-mpiz.cpp:322)
Reproject                    :meth:`Engine.forward_project`
  (main-mpi.cpp:286; main-mpiz.cpp:197)
SIRT / SART                  :meth:`Engine.sirt` / :meth:`Engine.sart`
  (main-mpi.cpp:614 / :578)
WBP (filter + BackProject)   :meth:`Engine.wbp` (main-mpi.cpp:841-846)
==========================  ==================================================

Device arrays are torch CUDA tensors (float32, contiguous); torch supplies
memory and streams only, all arithmetic runs in the library's sm_100a kernels.
There is no CPU fallback: constructing an :class:`Engine` without the built
library or without a CUDA device raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import build as _build

LAYOUT_Y, LAYOUT_Z = 0, 1
METHOD_BPT, METHOD_WBP, METHOD_SIRT, METHOD_SART, METHOD_FBP = 0, 1, 2, 3, 4
RECON_ZERO_START = 0x100  # tr_reconstruct_host: start from zeros
METHODS = {"BPT": METHOD_BPT, "WBP": METHOD_WBP, "SIRT": METHOD_SIRT,
           "SART": METHOD_SART, "FBP": METHOD_FBP}
DTYPE_F32, DTYPE_F16, DTYPE_BF16 = 0, 1, 2
DTYPES = {"f32": DTYPE_F32, "f16": DTYPE_F16, "bf16": DTYPE_BF16}


def _dtype_code(t) -> int:
    """tr_dtype of a torch tensor's element type."""
    import torch
    return {torch.float32: DTYPE_F32, torch.float16: DTYPE_F16,
            torch.bfloat16: DTYPE_BF16}[t.dtype]

_lib = None


class TiltRecError(RuntimeError):
    """A C-ABI call returned a non-zero tr_status."""

    def __init__(self, status: int, message: str):
        super().__init__(f"tr_status {status}: {message}")
        self.status = status


def library_path() -> str:
    return _build.LIB


def load_library(path: str | None = None) -> C.CDLL:
    """Load ``libtiltrec_b200.so``; raises if it has not been built."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    path = path or library_path()
    if not os.path.exists(path):
        raise FileNotFoundError(
            f"{path} is missing: build it with `python -m autom2_b200.build`")
    lib = C.CDLL(path)
    vp, i, f, d, sz = C.c_void_p, C.c_int, C.c_float, C.c_double, C.c_size_t
    dp = C.POINTER(C.c_double)
    fp = C.POINTER(C.c_float)
    lib.tr_version.restype = i
    lib.tr_status_string.argtypes = [i]
    lib.tr_status_string.restype = C.c_char_p
    lib.tr_geometry_from_angles.argtypes = [fp, i, f, f, f, dp]
    lib.tr_create.argtypes = [i, sz, C.POINTER(vp)]
    lib.tr_destroy.argtypes = [vp]
    lib.tr_last_error.argtypes = [vp]
    lib.tr_last_error.restype = C.c_char_p
    lib.tr_scratch_bytes.argtypes = [vp]
    lib.tr_scratch_bytes.restype = sz
    lib.tr_set_problem.argtypes = [vp, i, i, i, i, i, dp, f, f, f]
    lib.tr_update_geometry.argtypes = [vp, dp, vp]
    lib.tr_filter_rweight.argtypes = [vp, vp, vp]
    lib.tr_filter_fbp.argtypes = [vp, vp, i, vp]
    lib.tr_admm.argtypes = [vp, vp, vp, i, i, f, f, vp]
    lib.tr_admm_host.argtypes = [vp, vp, vp, i, i, f, f]
    lib.tr_backproject.argtypes = [vp, vp, vp, i, i, vp]
    lib.tr_forward_project.argtypes = [vp, vp, i, i, vp, vp, vp]
    lib.tr_sirt.argtypes = [vp, vp, vp, i, f, vp]
    lib.tr_sart.argtypes = [vp, vp, vp, i, f, vp]
    lib.tr_wbp.argtypes = [vp, vp, vp, vp]
    lib.tr_reconstruct_host.argtypes = [vp, i, vp, vp, i, f]
    lib.tr_forward_project_tilts.argtypes = [vp, vp, i, i, i, i, vp, vp, vp]
    lib.tr_residual.argtypes = [vp, vp, vp, vp, i, vp]
    lib.tr_sirt_update.argtypes = [vp, vp, vp, i, i, f, vp]
    lib.tr_sart_update.argtypes = [vp, vp, i, vp, i, i, f, vp]
    lib.tr_quantize.argtypes = [vp, vp, i, vp, vp, vp]
    lib.tr_backproject_lp.argtypes = [vp, vp, i, vp, vp, i, i, vp]
    lib.tr_sirt_lp.argtypes = [vp, vp, i, vp, i, vp, i, f, vp]
    lib.tr_sirt_zslabs.argtypes = [vp, vp, i, vp, i, vp, i, i, f, i, vp]
    lib.tr_set_deterministic.argtypes = [vp, i]
    lib.tr_sirt_gated.argtypes = [vp, vp, vp, i, f, d, vp, C.POINTER(i), vp]
    lib.tr_sirt_host_zslabs.argtypes = [vp, vp, vp, i, i, f, i, C.POINTER(i)]
    lib.tr_autotune_zslab.argtypes = [vp, vp, i, vp, i, vp, i, C.POINTER(i), dp]
    lib.tr_synchronize.argtypes = [vp]
    lib.tr_selftest_wait.argtypes = [vp, i]
    for name in ("tr_create", "tr_destroy", "tr_set_problem", "tr_update_geometry",
                 "tr_filter_rweight",
                 "tr_backproject", "tr_forward_project", "tr_sirt", "tr_sart",
                 "tr_wbp", "tr_reconstruct_host", "tr_synchronize",
                 "tr_geometry_from_angles"):
        getattr(lib, name).restype = i
    if path == library_path():
        _lib = lib
    return lib


def geometry_from_angles(angles, offset=0.0, pitch=0.0, zshift=0.0) -> np.ndarray:
    """Per-tilt coefficients [ntilt][8] (a0..a3, b0..b3), bit-identical to the
    reference's TranslateAngleToCoefficients + DecorateCoefficients."""
    lib = load_library()
    a = np.ascontiguousarray(angles, np.float32)
    out = np.zeros((a.size, 8), np.float64)
    st = lib.tr_geometry_from_angles(a.ctypes.data_as(C.POINTER(C.c_float)), a.size,
                                     float(offset), float(pitch), float(zshift),
                                     out.ctypes.data_as(C.POINTER(C.c_double)))
    if st:
        raise TiltRecError(st, "tr_geometry_from_angles")
    return out


def default_origin(layout: int, nx: int, ny: int, th: int):
    """The float origin the reference CLIs use: TiltRec-mpi (Y layout) takes
    (nx/2, th/2, th/2) (main-mpi.cpp:743-745, mrcvol.Y() is the thickness);
    TiltRecZ (Z layout) takes (nx/2, ny/2, th/2) (main-mpiz.cpp:1078-1080)."""
    if layout == LAYOUT_Y:
        return (nx * 0.5, th * 0.5, th * 0.5)
    return (nx * 0.5, ny * 0.5, th * 0.5)


def _ptr(t) -> int:
    return t.data_ptr() if t is not None else 0


def _stream(device: int):
    import torch
    return torch.cuda.current_stream(device).cuda_stream


class Engine:
    """One C-ABI context (``tr_ctx``) bound to a CUDA device."""

    def __init__(self, device: int = 0, hbm_budget: int = 0):
        self.lib = load_library()
        self.device = device
        h = C.c_void_p()
        st = self.lib.tr_create(device, hbm_budget, C.byref(h))
        if st:
            raise TiltRecError(st, f"tr_create(device={device}) failed "
                                   f"({self.lib.tr_status_string(st).decode()})")
        self.h = h
        self.shape = None

    def close(self):
        if getattr(self, "h", None):
            self.lib.tr_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st: int, what: str):
        if st:
            msg = self.lib.tr_last_error(self.h).decode()
            raise TiltRecError(st, f"{what}: {msg}")

    @property
    def scratch_bytes(self) -> int:
        return int(self.lib.tr_scratch_bytes(self.h))

    def set_problem(self, nx, ny, ntilt, thickness, coeff8, layout=LAYOUT_Y,
                    origin=None):
        c = np.ascontiguousarray(coeff8, np.float64).reshape(ntilt, 8)
        ox, oy, oz = origin if origin is not None else default_origin(layout, nx, ny, thickness)
        self._check(self.lib.tr_set_problem(self.h, nx, ny, ntilt, thickness, layout,
                                            c.ctypes.data_as(C.POINTER(C.c_double)),
                                            ox, oy, oz), "tr_set_problem")
        self.shape = (nx, ny, ntilt, thickness, layout)

    def update_geometry(self, coeff8):
        nt = self.shape[2]
        c = np.ascontiguousarray(coeff8, np.float64).reshape(nt, 8)
        self._check(self.lib.tr_update_geometry(self.h, c.ctypes.data_as(C.POINTER(C.c_double)),
                                                _stream(self.device)), "tr_update_geometry")

    def vol_shape(self):
        nx, ny, nt, th, layout = self.shape
        return (ny, th, nx) if layout == LAYOUT_Y else (th, ny, nx)

    def proj_shape(self):
        nx, ny, nt, th, _ = self.shape
        return (nt, ny, nx)

    def filter_rweight(self, proj):
        self._check(self.lib.tr_filter_rweight(self.h, _ptr(proj), _stream(self.device)),
                    "tr_filter_rweight")

    def filter_fbp(self, proj, mode=0):
        """FBP row filter in place: mode 0 Shepp-Logan, 1 Ram-Lak."""
        self._check(self.lib.tr_filter_fbp(self.h, _ptr(proj), mode, _stream(self.device)),
                    "tr_filter_fbp")

    def backproject(self, proj, vol, z0=0, nz=None):
        nz = self.shape[3] - z0 if nz is None else nz
        self._check(self.lib.tr_backproject(self.h, _ptr(proj), _ptr(vol), z0, nz,
                                            _stream(self.device)), "tr_backproject")

    def forward_project(self, vol, val, wt=None, z0=0, nz=None):
        nz = self.shape[3] - z0 if nz is None else nz
        self._check(self.lib.tr_forward_project(self.h, _ptr(vol), z0, nz, _ptr(val),
                                                _ptr(wt), _stream(self.device)),
                    "tr_forward_project")

    def forward_project_tilts(self, vol, t0, ntilts, val, wt=None, z0=0, nz=None):
        """Forward projection of tilts [t0, t0+ntilts); val/wt hold those
        tilts' planes only."""
        nz = self.shape[3] - z0 if nz is None else nz
        self._check(self.lib.tr_forward_project_tilts(self.h, _ptr(vol), z0, nz, t0, ntilts,
                                                      _ptr(val), _ptr(wt),
                                                      _stream(self.device)),
                    "tr_forward_project_tilts")

    def residual(self, proj, val, wt):
        """val <- proj - val/wt (val where wt == 0), over proj.shape[0]
        planes."""
        self._check(self.lib.tr_residual(self.h, _ptr(proj), _ptr(val), _ptr(wt),
                                         proj.shape[0], _stream(self.device)), "tr_residual")

    def sirt_update(self, resid, vol, gamma, z0=0, nz=None):
        nz = self.shape[3] - z0 if nz is None else nz
        self._check(self.lib.tr_sirt_update(self.h, _ptr(resid), _ptr(vol), z0, nz, gamma,
                                            _stream(self.device)), "tr_sirt_update")

    def sart_update(self, resid_plane, tilt, vol, gamma, z0=0, nz=None):
        nz = self.shape[3] - z0 if nz is None else nz
        self._check(self.lib.tr_sart_update(self.h, _ptr(resid_plane), tilt, _ptr(vol), z0, nz,
                                            gamma, _stream(self.device)), "tr_sart_update")

    def sirt(self, proj, vol, iters, gamma):
        self._check(self.lib.tr_sirt(self.h, _ptr(proj), _ptr(vol), iters, gamma,
                                     _stream(self.device)), "tr_sirt")

    def sart(self, proj, vol, iters, gamma):
        self._check(self.lib.tr_sart(self.h, _ptr(proj), _ptr(vol), iters, gamma,
                                     _stream(self.device)), "tr_sart")

    def admm(self, proj, vol, outer, cg_iters, mu, soft):
        """ADMM with a soft threshold, in place on vol (see tr_admm)."""
        self._check(self.lib.tr_admm(self.h, _ptr(proj), _ptr(vol), outer, cg_iters, mu, soft,
                                     _stream(self.device)), "tr_admm")

    def admm_host(self, proj: np.ndarray, vol: np.ndarray, outer, cg_iters, mu, soft):
        assert proj.dtype == np.float32 and proj.flags.c_contiguous
        assert vol.dtype == np.float32 and vol.flags.c_contiguous
        self._check(self.lib.tr_admm_host(self.h, proj.ctypes.data, vol.ctypes.data, outer,
                                          cg_iters, mu, soft), "tr_admm_host")

    def wbp(self, proj, vol):
        self._check(self.lib.tr_wbp(self.h, _ptr(proj), _ptr(vol), _stream(self.device)),
                    "tr_wbp")

    def reconstruct_host(self, method, proj: np.ndarray, vol: np.ndarray, iters=0,
                         gamma=0.0, zero_start=False):
        """Host buffers in, host volume out (vol is updated in place).
        zero_start: start from a zero volume without reading vol."""
        m = METHODS[method] if isinstance(method, str) else int(method)
        if zero_start:
            m |= RECON_ZERO_START
        assert proj.dtype == np.float32 and proj.flags.c_contiguous
        assert vol.dtype == np.float32 and vol.flags.c_contiguous
        self._check(self.lib.tr_reconstruct_host(self.h, m, proj.ctypes.data,
                                                 vol.ctypes.data, iters, gamma),
                    "tr_reconstruct_host")

    def quantize(self, proj, dtype):
        """FP32 stack -> (16-bit stack, per-tilt power-of-two scales), new
        CUDA tensors; dtype is torch.float16 or torch.bfloat16."""
        import torch
        out = torch.empty(proj.shape, dtype=dtype, device=proj.device)
        scale = torch.empty(proj.shape[0], dtype=torch.float32, device=proj.device)
        self._check(self.lib.tr_quantize(self.h, _ptr(proj), _dtype_code(out), _ptr(out),
                                         _ptr(scale), _stream(self.device)), "tr_quantize")
        return out, scale

    def backproject_lp(self, proj, scale, vol, z0=0, nz=None):
        nz = self.shape[3] - z0 if nz is None else nz
        self._check(self.lib.tr_backproject_lp(self.h, _ptr(proj), _dtype_code(proj),
                                               _ptr(scale), _ptr(vol), z0, nz,
                                               _stream(self.device)), "tr_backproject_lp")

    def sirt_lp(self, proj, scale, vol, iters, gamma, resid_dtype="bf16"):
        """SIRT from a 16-bit stack (see :meth:`quantize`); resid_dtype is
        'f32', 'f16' or 'bf16'."""
        self._check(self.lib.tr_sirt_lp(self.h, _ptr(proj), _dtype_code(proj), _ptr(scale),
                                        DTYPES[resid_dtype], _ptr(vol), iters, gamma,
                                        _stream(self.device)), "tr_sirt_lp")

    @staticmethod
    def _slab_vol(vol):
        """(pointer, on_host) of a z-slab volume: a CUDA tensor, or host
        memory (a CPU tensor, page-locked for overlapped copies, or a float32
        C-contiguous numpy array)."""
        if isinstance(vol, np.ndarray):
            assert vol.dtype == np.float32 and vol.flags.c_contiguous
            return vol.ctypes.data, 1
        assert vol.is_contiguous()
        return vol.data_ptr(), 0 if vol.is_cuda else 1

    def sirt_zslabs(self, proj, vol, iters, gamma, depth, scale=None, resid_dtype="f32"):
        """tr_sirt_zslabs: SIRT over z-slabs of `depth` sections; `vol` on
        the device or host-resident (see :meth:`_slab_vol`); proj FP32 or a
        16-bit stack with its scales."""
        vp, host = self._slab_vol(vol)
        self._check(self.lib.tr_sirt_zslabs(self.h, _ptr(proj), _dtype_code(proj), _ptr(scale),
                                            DTYPES[resid_dtype], vp, host, iters, gamma, depth,
                                            _stream(self.device)), "tr_sirt_zslabs")

    def autotune_zslab(self, proj, vol, scale=None, resid_dtype="f32"):
        """tr_autotune_zslab: (slab depth, sweep ms)."""
        vp, host = self._slab_vol(vol)
        d, ms = C.c_int(), C.c_double()
        self._check(self.lib.tr_autotune_zslab(self.h, _ptr(proj), _dtype_code(proj),
                                               _ptr(scale), DTYPES[resid_dtype], vp, host,
                                               C.byref(d), C.byref(ms)), "tr_autotune_zslab")
        return d.value, ms.value

    def sirt_host_zslabs(self, proj: np.ndarray, vol: np.ndarray, iters, gamma, depth=0,
                         zero_start=True) -> int:
        """tr_sirt_host_zslabs: SIRT with the volume kept in host memory,
        streamed in z-slabs (depth 0: autotuned); returns the depth run."""
        assert proj.dtype == np.float32 and proj.flags.c_contiguous
        assert vol.dtype == np.float32 and vol.flags.c_contiguous
        used = C.c_int()
        self._check(self.lib.tr_sirt_host_zslabs(self.h, proj.ctypes.data, vol.ctypes.data,
                                                 int(zero_start), iters, gamma, depth,
                                                 C.byref(used)), "tr_sirt_host_zslabs")
        return used.value

    def sirt_gated(self, proj, vol, max_iters, gamma, rel_tol=0.0):
        """tr_sirt_gated: (iterations applied, FP64 residual norms)."""
        norms = np.zeros(max(1, max_iters), np.float64)
        done = C.c_int()
        self._check(self.lib.tr_sirt_gated(self.h, _ptr(proj), _ptr(vol), max_iters, gamma,
                                           rel_tol, norms.ctypes.data, C.byref(done),
                                           _stream(self.device)), "tr_sirt_gated")
        n = min(max_iters, done.value + 1) if max_iters else 0
        return done.value, norms[:n]

    def set_deterministic(self, on: bool = True):
        """tr_set_deterministic: int64 fixed-point forward-projection sums,
        bitwise repeatable."""
        self._check(self.lib.tr_set_deterministic(self.h, int(bool(on))),
                    "tr_set_deterministic")

    def synchronize(self):
        self._check(self.lib.tr_synchronize(self.h), "tr_synchronize")

    def volume_to_bytes(self, vol, slab, alpha=0.9):
        """tr_volume_to_bytes: a uint8 CUDA tensor of vol's byte mapping."""
        import torch
        out = torch.empty(vol.numel(), dtype=torch.uint8, device=vol.device)
        self.lib.tr_volume_to_bytes.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, C.c_size_t,
                                               C.c_float, C.c_void_p, C.c_void_p]
        self._check(self.lib.tr_volume_to_bytes(self.h, vol.data_ptr(), vol.numel(), slab,
                                                alpha, out.data_ptr(), _stream(self.device)),
                    "tr_volume_to_bytes")
        return out

    def selftest_wait(self, budget_us: int) -> int:
        """tr_selftest_wait's status (TR_ERR_TIMEOUT = -5 when the bounded
        wait gave up, as it should)."""
        return int(self.lib.tr_selftest_wait(self.h, budget_us))


def sirt_static(proj, vol, coeff8, iters, gamma, layout=LAYOUT_Y, origin=None,
                device=0):
    """SIRT through tr_sirt_static, the entry point that allocates no device
    memory (its scratch is a 64 MiB static device array; see the header).
    proj, vol: CUDA tensors; vol is updated in place."""
    lib = load_library()
    fn = lib.tr_sirt_static
    vp, i, f = C.c_void_p, C.c_int, C.c_float
    fn.argtypes = [i, i, i, i, i, i, C.POINTER(C.c_double), f, f, f, vp, vp, i, f, vp]
    fn.restype = i
    nt, ny, nx = proj.shape
    th = vol.shape[1] if layout == LAYOUT_Y else vol.shape[0]
    c = np.ascontiguousarray(coeff8, np.float64).reshape(nt, 8)
    ox, oy, oz = origin if origin is not None else default_origin(layout, nx, ny, th)
    st = fn(device, nx, ny, nt, th, layout, c.ctypes.data_as(C.POINTER(C.c_double)),
            ox, oy, oz, proj.data_ptr(), vol.data_ptr(), iters, gamma, _stream(device))
    if st:
        raise TiltRecError(st, "tr_sirt_static: " + lib.tr_status_string(st).decode())


def static_scratch_limit() -> int:
    lib = load_library()
    lib.tr_static_scratch_limit.restype = C.c_size_t
    return int(lib.tr_static_scratch_limit())


def static_take_timeout(device=0) -> int:
    """tr_static_take_timeout's status: TR_ERR_TIMEOUT (-5) when a
    tr_sirt_static back-projection gave up a device wait since the last read."""
    lib = load_library()
    lib.tr_static_take_timeout.argtypes = [C.c_int]
    return int(lib.tr_static_take_timeout(device))


def static_selftest_wait(budget_us: int, device=0) -> int:
    """tr_static_selftest_wait's status (-5 when the bounded wait gave up and
    the report came back through the static scratch, as it should)."""
    lib = load_library()
    lib.tr_static_selftest_wait.argtypes = [C.c_int, C.c_int]
    return int(lib.tr_static_selftest_wait(device, budget_us))


# ------------------------------------------------------------ batched jobs

class Job(C.Structure):
    """tr_job: one reconstruction for the scheduler."""
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("ntilt", C.c_int), ("thickness", C.c_int),
                ("layout", C.c_int), ("coeff8", C.POINTER(C.c_double)),
                ("ox", C.c_float), ("oy", C.c_float), ("oz", C.c_float),
                ("proj", C.c_void_p), ("vol", C.c_void_p), ("vol_in", C.c_int),
                ("host", C.c_int),
                ("wbp", C.c_int), ("sirt_iters", C.c_int), ("gamma", C.c_float)]


class SchedInfo(C.Structure):
    _fields_ = [("steps", C.c_longlong), ("bp_items", C.c_longlong),
                ("fp_items", C.c_longlong), ("peak_bytes", C.c_size_t),
                ("grid_bp", C.c_int), ("grid_fp", C.c_int), ("smem_bp", C.c_size_t),
                ("queued", C.c_int), ("active", C.c_int)]


class Scheduler:
    """tr_sched: many reconstructions on one device, advanced together one
    batched step at a time (see include/tiltrec_b200.h).

    Jobs take torch CUDA tensors (device jobs: the volume is updated in
    place) or numpy arrays (host jobs: pinned memory overlaps the copies)."""

    def __init__(self, device=0, hbm_budget=0, proj_dtype="f32", resid_dtype="f32"):
        self.lib = load_library()
        L = self.lib
        vp, i, sz = C.c_void_p, C.c_int, C.c_size_t
        L.tr_sched_create.argtypes = [i, sz, i, i, C.POINTER(vp)]
        L.tr_sched_submit.argtypes = [vp, C.POINTER(Job), C.POINTER(C.c_ulonglong)]
        L.tr_sched_wait.argtypes = [vp, C.c_ulonglong, C.POINTER(C.c_double)]
        L.tr_sched_drain.argtypes = [vp]
        L.tr_sched_stats.argtypes = [vp, C.POINTER(SchedInfo)]
        L.tr_sched_last_error.argtypes = [vp]
        L.tr_sched_last_error.restype = C.c_char_p
        L.tr_sched_configure.argtypes = [vp, sz, i]
        L.tr_sched_set_policy.argtypes = [vp, i]
        L.tr_sched_set_aging.argtypes = [vp, C.c_double]
        L.tr_sched_autotune.argtypes = [vp, C.POINTER(Job), i, C.POINTER(sz), C.POINTER(i)]
        L.tr_sched_destroy.argtypes = [vp]
        h = vp()
        st = L.tr_sched_create(device, hbm_budget, DTYPES[proj_dtype], DTYPES[resid_dtype],
                               C.byref(h))
        if st:
            raise TiltRecError(st, "tr_sched_create failed")
        self.h = h
        self.device = device

    def _check(self, st, what):
        if st:
            raise TiltRecError(st, f"{what}: {self.lib.tr_sched_last_error(self.h).decode()}")

    def job(self, proj, vol, coeff8, layout=LAYOUT_Y, origin=None, wbp=False, sirt_iters=0,
            gamma=0.0, vol_in=False):
        """A tr_job over proj [nt][ny][nx] and vol (the layout's shape); the
        reconstruction starts from vol's contents when vol_in, else from
        zeros."""
        nt, ny, nx = proj.shape
        th = vol.shape[1] if layout == LAYOUT_Y else vol.shape[0]
        c = np.ascontiguousarray(coeff8, np.float64).reshape(nt, 8)
        ox, oy, oz = origin if origin is not None else default_origin(layout, nx, ny, th)
        host = isinstance(proj, np.ndarray)
        if host:
            assert proj.dtype == np.float32 and vol.dtype == np.float32
            assert proj.flags.c_contiguous and vol.flags.c_contiguous
            pp, vv = proj.ctypes.data, vol.ctypes.data
        else:
            pp, vv = proj.data_ptr(), vol.data_ptr()
        j = Job(nx, ny, nt, th, layout, c.ctypes.data_as(C.POINTER(C.c_double)), ox, oy, oz,
                pp, vv, int(bool(vol_in)), int(host), int(bool(wbp)), sirt_iters, gamma)
        j._c = c  # keeps the coefficients alive until submission copies them
        return j

    def submit(self, job: Job) -> int:
        jid = C.c_ulonglong()
        self._check(self.lib.tr_sched_submit(self.h, C.byref(job), C.byref(jid)),
                    "tr_sched_submit")
        return jid.value

    def wait(self, jid: int) -> float:
        """Blocks until job jid is done; returns its latency in seconds."""
        lat = C.c_double()
        self._check(self.lib.tr_sched_wait(self.h, jid, C.byref(lat)), "tr_sched_wait")
        return lat.value

    def drain(self):
        self._check(self.lib.tr_sched_drain(self.h), "tr_sched_drain")

    def stats(self) -> dict:
        info = SchedInfo()
        self._check(self.lib.tr_sched_stats(self.h, C.byref(info)), "tr_sched_stats")
        return {k: getattr(info, k) for k, _ in SchedInfo._fields_}

    def configure(self, smem_bp: int, bp_ctas_per_sm: int = 0):
        self._check(self.lib.tr_sched_configure(self.h, smem_bp, bp_ctas_per_sm),
                    "tr_sched_configure")

    def set_policy(self, policy: str):
        """'batched' (all admitted jobs per step, persistent graph-replayed
        launches) or 'srpt' (shortest remaining work first, per-job
        kernels)."""
        self._check(self.lib.tr_sched_set_policy(self.h, {"batched": 0, "srpt": 1}[policy]),
                    "tr_sched_set_policy")

    def set_aging(self, aging_s: float):
        """SRPT aging time in seconds (0: pure shortest remaining work)."""
        self._check(self.lib.tr_sched_set_aging(self.h, aging_s), "tr_sched_set_aging")

    def autotune(self, probe: Job, iters: int = 2):
        sm, ct = C.c_size_t(), C.c_int()
        self._check(self.lib.tr_sched_autotune(self.h, C.byref(probe), iters, C.byref(sm),
                                               C.byref(ct)), "tr_sched_autotune")
        return sm.value, ct.value

    def close(self):
        if getattr(self, "h", None):
            self.lib.tr_sched_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def resample_bin(stack, bin_factor: int):
    """Area binning of a CUDA tensor [nt][ny][nx] by an integer factor
    (tr_resample_bin); returns a new tensor [nt][ny/bin][nx/bin]."""
    import torch
    lib = load_library()
    lib.tr_resample_bin.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int,
                                    C.c_void_p, C.c_void_p]
    nt, ny, nx = stack.shape
    out = torch.empty((nt, ny // bin_factor, nx // bin_factor), dtype=torch.float32,
                      device=stack.device)
    st = lib.tr_resample_bin(stack.data_ptr(), nx, ny, nt, bin_factor, out.data_ptr(),
                             _stream(stack.device.index or 0))
    if st:
        raise TiltRecError(st, "tr_resample_bin: " + lib.tr_status_string(st).decode())
    return out
