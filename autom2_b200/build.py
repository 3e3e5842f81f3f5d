"""Build the TiltRec B200 engine in-tree.

Outputs:
  autom2_b200/lib/libtiltrec_b200.so   C-ABI library (include/tiltrec_b200.h)
  autom2_b200/bin/TiltRec-cuda         drop-in CLI, Y layout
  autom2_b200/bin/TiltRecZ-cuda        drop-in CLI, Z layout
  autom2_b200/bin/TiltRec-mpi          the same, mpi option dialect, Y layout
  autom2_b200/bin/TiltRecZ-mpi         the same, mpi option dialect, Z layout
  autom2_b200/bin/resample             drop-in binning step

Kernels are compiled for sm_100a only.  Run: python -m autom2_b200.build
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
CLI = os.path.join(PKG, "cli")
INCLUDE = os.path.join(ROOT, "include")
LIBDIR = os.path.join(PKG, "lib")
BINDIR = os.path.join(PKG, "bin")
LIB = os.path.join(LIBDIR, "libtiltrec_b200.so")

GENCODE = ["-gencode", "arch=compute_100a,code=sm_100a"]
CU_SOURCES = ["tr_kernels.cu", "tr_filter.cu", "tr_api.cu", "tr_static.cu", "tr_sched.cu",
              "tr_admm.cu", "tr_output.cu"]
CLI_SOURCES = ["mrc_io.cpp", "tiltrec_cli.cpp"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _newer(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(d) <= t for d in deps)


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("build step failed: " + " ".join(cmd))


def _tmp(out: str) -> str:
    """A build output's temporary name, private to this process: ranks that
    build at the same time (one process per GPU) each write their own file
    and move it into place atomically, so none loads a half-written one."""
    return f"{out}.tmp{os.getpid()}"


def _build_to(out: str, cmd_for) -> None:
    tmp = _tmp(out)
    try:
        _run(cmd_for(tmp))
        os.replace(tmp, out)
    finally:
        if os.path.exists(tmp):
            os.remove(tmp)


def build_lib(force: bool = False, verbose_ptxas: bool = False) -> str:
    srcs = [os.path.join(CSRC, s) for s in CU_SOURCES]
    deps = srcs + [os.path.join(CSRC, "tr_internal.cuh"), os.path.join(CSRC, "tr_geom.h"),
                   os.path.join(CSRC, "tr_filter_host.h"),
                   os.path.join(INCLUDE, "tiltrec_b200.h")]
    if not force and _newer(LIB, deps):
        return LIB
    os.makedirs(LIBDIR, exist_ok=True)
    def cmd(tmp):
        c = [nvcc(), *GENCODE, "-O3", "-lineinfo", "-std=c++17", "-shared",
             "-Xcompiler", "-fPIC,-fvisibility=hidden", "-I", INCLUDE, "-I", CSRC,
             "--expt-relaxed-constexpr", "-o", tmp, *srcs]
        if verbose_ptxas:
            c.insert(1, "-Xptxas=-v")
        return c
    _build_to(LIB, cmd)
    return LIB


def build_cli(force: bool = False) -> list[str]:
    srcs = [os.path.join(CLI, s) for s in CLI_SOURCES]
    if not all(os.path.exists(s) for s in srcs):
        return []
    os.makedirs(BINDIR, exist_ok=True)
    outs = []
    for name, layout, mpi in (("TiltRec-cuda", 0, 0), ("TiltRecZ-cuda", 1, 0),
                              ("TiltRec-mpi", 0, 1), ("TiltRecZ-mpi", 1, 1)):
        out = os.path.join(BINDIR, name)
        deps = srcs + [os.path.join(CLI, "mrc_io.h"), LIB]
        if force or not _newer(out, deps):
            _build_to(out, lambda tmp, layout=layout, mpi=mpi: [
                "g++", "-std=c++17", "-O2", f"-DTR_CLI_LAYOUT={layout}",
                f"-DTR_CLI_MPI_DIALECT={mpi}", "-I", INCLUDE, "-I", CLI, "-o", tmp, *srcs,
                "-L", LIBDIR, "-ltiltrec_b200", "-Wl,-rpath,$ORIGIN/../lib"])
        outs.append(out)
    out = os.path.join(BINDIR, "resample")
    srcs_r = [os.path.join(CLI, "mrc_io.cpp"), os.path.join(CLI, "resample_cli.cpp")]
    if force or not _newer(out, srcs_r + [os.path.join(CLI, "mrc_io.h"), LIB]):
        _build_to(out, lambda tmp: [
            "g++", "-std=c++17", "-O2", "-I", INCLUDE, "-I", CLI, "-o", tmp, *srcs_r,
            "-L", LIBDIR, "-ltiltrec_b200", "-Wl,-rpath,$ORIGIN/../lib"])
    outs.append(out)
    return outs


def build(force: bool = False) -> None:
    build_lib(force)
    build_cli(force)


if __name__ == "__main__":
    build(force="--force" in sys.argv)
    print(LIB)
