"""Drop-in executables: option handling and error exits (CPU; no device)."""
import os
import subprocess

import numpy as np
import pytest

from autom2_b200 import build
from mrc_util import write_angles, write_mrc

BIN = os.path.join(os.path.dirname(build.LIB), "..", "bin")


@pytest.fixture(scope="module")
def exes():
    build.build()
    return {n: os.path.join(BIN, n) for n in ("TiltRec-cuda", "TiltRecZ-cuda")}


def run(exe, *args, env=None):
    return subprocess.run([exe, *args], capture_output=True, text=True, env=env, timeout=120)


@pytest.mark.parametrize("name", ["TiltRec-cuda", "TiltRecZ-cuda"])
def test_help_and_bad_options(exes, name):
    r = run(exes[name], "--help")
    assert r.returncode == 0 and "--geometry" in r.stdout
    r = run(exes[name], "--bogus")
    assert r.returncode == 1 and "WRONG INPUT" in r.stdout


def test_argument_errors(exes, tmp_path):
    exe = exes["TiltRec-cuda"]
    stack = tmp_path / "s.mrc"
    write_mrc(stack, np.zeros((3, 8, 8), np.float32))
    tlt = tmp_path / "a.tlt"
    write_angles(tlt, [-3, 0, 3])
    base = ["-i", str(stack), "-o", str(tmp_path / "v.mrc"), "-t", str(tlt)]
    r = run(exe, *base, "-g", "0,0,0,0", "-m", "BPT")
    assert r.returncode == 1 and "thickness" in r.stderr
    r = run(exe, *base, "-g", "0,0,0,4", "-m", "SIRT")
    assert r.returncode == 1 and "needs iterations" in r.stderr
    r = run(exe, *base, "-g", "0,0,0,4", "-m", "ADMM")
    assert r.returncode == 1 and "ADMM needs" in r.stderr
    r = run(exe, *base, "-g", "0,0,0,4,9", "-m", "BPT")
    assert r.returncode == 1
    write_angles(tlt, [0, 3])
    r = run(exe, *base, "-g", "0,0,0,4", "-m", "BPT")
    assert r.returncode == 1 and "tilt angles" in r.stderr


def test_no_device_is_an_error(exes, tmp_path):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    stack = tmp_path / "s.mrc"
    write_mrc(stack, np.zeros((2, 8, 8), np.float32))
    tlt = tmp_path / "a.tlt"
    write_angles(tlt, [0, 3])
    r = run(exes["TiltRec-cuda"], "-i", str(stack), "-o", str(tmp_path / "v.mrc"), "-t", str(tlt),
            "-g", "0,0,0,4", "-m", "WBP")
    assert r.returncode == 1 and "no CUDA device" in r.stderr


def test_only_rank_zero_works(exes, tmp_path):
    env = dict(os.environ, OMPI_COMM_WORLD_RANK="1")
    r = run(exes["TiltRec-cuda"], "-i", "missing.mrc", "-o", "x", "-t", "y", "-g", "0,0,0,4",
            "-m", "BPT", env=env)
    assert r.returncode == 0


def test_concurrent_builds_leave_whole_binaries(exes):
    """One process per GPU may build at the same time: each writes its own
    temporary file and moves it into place, so two concurrent rebuilds leave
    complete executables and no temporaries."""
    import sys
    code = "from autom2_b200 import build; build.build_cli(force=True)"
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    procs = [subprocess.Popen([sys.executable, "-c", code], cwd=root) for _ in range(2)]
    assert all(p.wait(timeout=300) == 0 for p in procs)
    assert not [f for f in os.listdir(BIN) if ".tmp" in f]
    for name in ("TiltRec-cuda", "TiltRecZ-cuda", "TiltRec-mpi", "TiltRecZ-mpi"):
        r = run(os.path.join(BIN, name), "--help")
        assert r.returncode == 0 and "--geometry" in r.stdout
