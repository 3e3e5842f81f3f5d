"""Generate the golden fixtures in tests/golden/ from the reference itself.

The reference ships no tests or golden vectors for TiltRec.  These fixtures
are the outputs of the unmodified reference CPU routines (compiled by
``oracle/Makefile`` into ``oracle/_ref/``) on seeded inputs, so that parity
can be checked where the reference sources are absent (the GPU host).

Run from the repository root (needs oracle/_ref built):
    python tests/golden/make_golden.py
Writes tests/golden/golden.npz and tests/golden/MANIFEST.json (SHA-256 of
every array).
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle as O  # noqa: E402
from autom2_b200 import synth  # noqa: E402
from autom2_b200.tiltrec import geometry_from_angles  # noqa: E402

OUT = os.path.join(ROOT, "tests", "golden")


def small_case(name, rng, nx, ny, nt, th, pitch=0.0, rot_deg=0.0, shift=1.0,
               amax=63.0):
    ang = np.linspace(-amax, amax - 6.0, nt).astype(np.float32)
    c8 = geometry_from_angles(ang, 0.7, pitch, 1.25).copy()
    if rot_deg:
        psi = np.deg2rad(rng.normal(0, rot_deg, nt))
        a, b = c8[:, :4].copy(), c8[:, 4:].copy()
        c8[:, :4] = np.cos(psi)[:, None] * a - np.sin(psi)[:, None] * b
        c8[:, 4:] = np.sin(psi)[:, None] * a + np.cos(psi)[:, None] * b
    c8[:, 0] += rng.normal(0, shift, nt)
    c8[:, 4] += rng.normal(0, shift, nt)
    proj = rng.normal(size=(nt, ny, nx)).astype(np.float32)
    return dict(name=name, nx=nx, ny=ny, nt=nt, th=th, angles=ang, coeff8=c8,
                proj=proj)


def main():
    ref = O.Reference()
    rng = np.random.default_rng(20241203)
    out = {}

    def put(prefix, **arrs):
        for k, v in arrs.items():
            out[f"{prefix}/{k}"] = np.asarray(v)

    # Y layout cases: separable (shifts only) and general (XTILT + rotations).
    for case in (small_case("ysep", rng, 61, 23, 9, 13),
                 small_case("ygen", rng, 53, 29, 7, 11, pitch=4.0, rot_deg=2.0)):
        nx, ny, nt, th = case["nx"], case["ny"], case["nt"], case["th"]
        c20 = O.coeff20(case["coeff8"])
        org = (nx * 0.5, th * 0.5, th * 0.5)
        zero = np.zeros((ny, th, nx), np.float32)
        vol0 = rng.normal(size=(ny, th, nx)).astype(np.float32)
        bpt = ref.y_backproject(nx, ny, nt, th, c20, org, case["proj"], zero)
        filt = ref.filter_rweight(case["proj"])
        wbp = ref.y_backproject(nx, ny, nt, th, c20, org, filt, zero)
        sirt = ref.y_sirt(nx, ny, nt, th, c20, org, case["proj"], vol0, 3, 0.5)
        sart = ref.y_sirt(nx, ny, nt, th, c20, org, case["proj"], vol0, 1, 0.5, sart=True)
        fpv, fpw = ref.y_reproject(nx, ny, th, c20[nt // 2], org, vol0)
        put(case["name"], dims=np.array([nx, ny, nt, th]), origin=np.array(org, np.float32),
            angles=case["angles"], coeff8=case["coeff8"], proj=case["proj"], vol0=vol0,
            bpt=bpt, filtered=filt, wbp=wbp, sirt3=sirt, sart1=sart, fp_val=fpv, fp_wt=fpw)

    # Z layout (TiltRecZ-mpi routines).
    case = small_case("zsep", rng, 47, 31, 8, 12)
    nx, ny, nt, th = case["nx"], case["ny"], case["nt"], case["th"]
    c20 = O.coeff20(case["coeff8"])
    org = (nx * 0.5, ny * 0.5, th * 0.5)
    vol0 = rng.normal(size=(th, ny, nx)).astype(np.float32)
    bpt = ref.z_run(0, nx, ny, nt, th, c20, org, case["proj"], vol0)
    sirt = ref.z_run(3, nx, ny, nt, th, c20, org, case["proj"], vol0, 2, 0.7)
    wbp = ref.z_run(2, nx, ny, nt, th, c20, org, case["proj"], vol0)
    put("zsep", dims=np.array([nx, ny, nt, th]), origin=np.array(org, np.float32),
        angles=case["angles"], coeff8=case["coeff8"], proj=case["proj"], vol0=vol0,
        bpt=bpt, sirt2=sirt, wbp=wbp)

    # cfg0 geometry and phantom at 1/4 scale: reference forward model, noise,
    # then the reference WBP and SIRT-5 reconstructions.
    cfg = synth.config("cfg0", scale=4)
    c8 = synth.coefficients(cfg)
    c20 = O.coeff20(c8)
    nx, ny, nt, th = cfg.nx, cfg.ny, cfg.ntilt, cfg.thickness
    org = (nx * 0.5, th * 0.5, th * 0.5)
    ph = synth.phantom(cfg).numpy()
    proj = np.zeros((nt, ny, nx), np.float32)
    for t in range(nt):
        v, w = ref.y_reproject(nx, ny, th, c20[t], org, ph)
        proj[t] = np.where(w != 0, v / np.where(w != 0, w, 1), 0)
    proj = synth.add_noise(proj, cfg)
    zero = np.zeros((ny, th, nx), np.float32)
    wbp = ref.y_backproject(nx, ny, nt, th, c20, org, ref.filter_rweight(proj), zero)
    sirt = ref.y_sirt(nx, ny, nt, th, c20, org, proj, zero, 5, 0.5)
    put("cfg0s4", dims=np.array([nx, ny, nt, th]), origin=np.array(org, np.float32),
        angles=cfg.angles, coeff8=c8, phantom=ph, proj=proj, wbp=wbp, sirt5=sirt)

    # Reference coefficients (TranslateAngleToCoefficients + DecorateCoefficients)
    # for a few --geometry settings, 20 doubles per tilt.
    geo_ang = np.concatenate([np.arange(-60, 61, 3), [-89.5, -70.25, 0.001, 45.0, 89.9]]
                             ).astype(np.float32)
    geo_par = np.array([[0, 0, 0], [1.5, 0.3, 3.0], [-2.0, -5.0, -1.0],
                        [0.7, 12.0, -7.5], [-11.0, 0.3, 40.0]], np.float32)
    put("geom", angles=geo_ang, params=geo_par,
        coeff20=np.stack([ref.coeffs20(geo_ang, *g) for g in geo_par]))

    np.savez_compressed(os.path.join(OUT, "golden.npz"), **out)
    manifest = {k: hashlib.sha256(np.ascontiguousarray(v).tobytes()).hexdigest()
                for k, v in sorted(out.items())}
    with open(os.path.join(OUT, "MANIFEST.json"), "w") as f:
        json.dump(manifest, f, indent=1)
    print(f"wrote {len(out)} arrays")


if __name__ == "__main__":
    main()
