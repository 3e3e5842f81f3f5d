"""bench.py's reference arm, on the CPU.

`bench.py --impl reference` times the reference's own SIRT (the unmodified
reference sources built into oracle/_ref) on the host cores, on the same
metric and workload as the GPU arm.  It must never load this project's
engine library: its geometry comes from the reference's own
TranslateAngleToCoefficients / DecorateCoefficients.  This runs the arm for
one short step in a child process, checks its JSON line against the
benchmark contract and lists the project libraries the process mapped.
"""
import json
import os
import subprocess
import sys
from pathlib import Path

import pytest

import oracle as O

ROOT = Path(__file__).resolve().parents[1]

CHILD = r"""
import atexit, runpy, sys
root = sys.argv[1]
def maps():
    libs = sorted({l.split()[-1] for l in open('/proc/self/maps')
                   if '.so' in l and l.split()[-1].startswith(root)})
    print('MAPPED ' + ' '.join(libs), flush=True)
atexit.register(maps)
sys.argv = ['bench.py', '--impl', 'reference', '--steps', '1', '--warmup', '1']
runpy.run_path('bench.py', run_name='__main__')
"""


@pytest.mark.skipif(not O.reference_available(), reason="oracle/_ref is not built")
def test_reference_arm_line_and_libraries():
    env = dict(os.environ)
    env.pop("RANK", None)
    env.pop("WORLD_SIZE", None)
    out = subprocess.run([sys.executable, "-c", CHILD, str(ROOT)], cwd=ROOT, env=env,
                         capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, out.stdout
    line = json.loads(lines[0])
    assert line["impl"] == "reference"
    assert line["metric"] == "voxel-proj updates/s" and line["unit"] == "VPU/s"
    assert line["higher_is_better"] is True and line["value"] > 0
    cb = line["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["sample"]
    assert cb["value"] == line["value"]
    assert line["e2e"] == {"value": line["value"], "unit": "VPU/s",
                           "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    mapped = [l for l in out.stdout.splitlines() if l.startswith("MAPPED")][0].split()[1:]
    assert mapped, "the reference libraries were not loaded"
    assert all("/oracle/_ref/" in p for p in mapped), mapped
    assert not any("libtiltrec_b200" in p for p in mapped)


def test_reference_arm_other_ranks_exit_without_work():
    """Under torchrun rank 0 alone times the reference; the other ranks exit 0
    and print nothing."""
    env = dict(os.environ, RANK="1", LOCAL_RANK="1", WORLD_SIZE="2")
    out = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--gpus", "2",
                          "--steps", "1", "--warmup", "1"], cwd=ROOT, env=env,
                         capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr[-2000:]
    assert not [l for l in out.stdout.splitlines() if l.startswith("{")]
