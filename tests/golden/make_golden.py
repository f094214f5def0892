"""Regenerate the golden J(t) fixtures from the reference's own code.

Runs the reference build ``oracle/_ref/libwannier.so`` (compiled from the reference's unmodified
sources by ``oracle/Makefile``) through the reference's own, unmodified ctypes wrapper
``pySWE/pyswe.py`` loaded from the reference checkout, so the fixtures are exactly what a user of
the reference would get.  The ``ks_*`` fixtures come from the reference's k-space solver
(src/solver_kspace.cpp), which none of its entry points reach: ``oracle/ref_probe.cpp`` drives its
compiled objects the way SWESim drives the real-space solver.  Needs the reference checkout
(``--ref``); the GPU box never runs this.

    python tests/golden/make_golden.py [--ref /root/reference] [--only NAME ...]
"""
from __future__ import annotations

import argparse
import contextlib
import hashlib
import importlib.util
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "hhg-solids_b200"))
import tbgen  # noqa: E402

PULSE = {"tmax": 90.0, "dt": 21.97e-3, "intensity": 1e12, "lambda": 3000.0, "tmax_field": 80.0,
         "pol_vec": [0.0, 1.0, 0.0], "phi_vec": [0.0, 0.0, 0.0]}


def case(model, n, **over):
    p = dict(PULSE, nr1=n, nr2=n, nr3=1)
    p.update(over)
    return {"model": model, "param": p}


# name -> model + pySWE parameters.  "c0" is the full 60x60 pulse, "c1" the full 200x200 pulse,
# "c2_prefix" the first steps of the 11-orbital 150x150 case (a complete run with a short tmax).
CASES = {
    "haldane_8_y": case("haldane", 8, tmax=2.0),
    "haldane_12_pol": case("haldane", 12, tmax=4.0, pol_vec=[0.6, 0.8, 0.0], phi_vec=[0.3, 0.0, 0.0]),
    "haldane_16_rect": case("haldane", 16, nr2=10, tmax=3.0, pol_vec=[1.0, 0.0, 0.0], intensity=3e12),
    "tmd6_8": case("tmd6_s1", 8, tmax=1.0, pol_vec=[0.3, 1.0, 0.0]),
    "tmd11_10": case("tmd11_s7", 10, tmax=0.5),
    "tmd12_6": case("tmd12_s3", 6, tmax=0.4, pol_vec=[0.5, 0.5, 0.0], lambda_=2000.0),
    "c0": case("haldane", 60),
    "c2_prefix": case("tmd11_s7", 150, tmax=2.2),
    "c1": case("haldane", 200),
    # Full pulses of the 11- and 12-orbital models on a small grid: where the mixed form's per-harmonic
    # error is measured on models whose mixed kernels differ from the FP64 ones.
    "tmd11_12_full": case("tmd11_s7", 12),
    "tmd12_12_full": case("tmd12_s2", 12, pol_vec=[0.6, 0.8, 0.0], intensity=2e12),
    "w90_tmd6_deg_8": case("tmd6_deg_equiv", 8, tmax=1.0, pol_vec=[0.6, 0.8, 0.0], intensity=2e12),
    "ks_haldane_12_pol": case("haldane", 12, tmax=4.0, pol_vec=[0.6, 0.8, 0.0], phi_vec=[0.3, 0.0, 0.0],
                              solver="kspace"),
    "ks_tmd6_8": case("tmd6_s1", 8, tmax=1.0, pol_vec=[0.3, 1.0, 0.0], solver="kspace"),
    "ks_tmd11_10": case("tmd11_s7", 10, tmax=0.5, solver="kspace"),
    "ks_c0": case("haldane", 60, solver="kspace"),
    "ks_c1": case("haldane", 200, solver="kspace"),
}


def load_reference_pyswe(ref: str):
    spec = importlib.util.spec_from_file_location("reference_pyswe", os.path.join(ref, "pySWE", "pyswe.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def run_case(pyswe, lib: str, name: str, spec: dict) -> dict:
    p = dict(spec["param"])
    if "lambda_" in p:
        p["lambda"] = p.pop("lambda_")
    solver = p.pop("solver", "rspace")
    tb = tbgen.model_path(spec["model"])
    param = dict(p, path_lib=lib, path_tb=tb)
    param["pol_vec"] = np.array(p["pol_vec"], dtype=np.float64)
    param["phi_vec"] = np.array(p["phi_vec"], dtype=np.float64)
    t0 = time.time()
    if solver == "kspace":
        sys.path.insert(0, os.path.join(REPO, "oracle"))
        import oracle  # noqa: E402

        t, J = oracle.ref_kspace_run(tb, param)
        jx, jy, jz = J
        t_init = 0.0
        p["solver"] = solver
    else:
        with open(os.devnull, "w") as devnull, contextlib.redirect_stdout(devnull):
            settings = pyswe.Settings(param)
            swe = pyswe.SWE(settings)
            t_init = time.time() - t0
            swe.run_simulation()
            t, jx, jy, jz = swe.get_current()
            swe.delete()
    t_run = time.time() - t0 - t_init
    out = os.path.join(HERE, f"{name}.npz")
    np.savez_compressed(out, t=np.real(t), J=np.stack([jx, jy, jz]).astype(np.complex128))
    meta = {"model": spec["model"], "param": p,
            "model_sha256": hashlib.sha256(open(tb, "rb").read()).hexdigest(),
            "nt": int(len(t)), "reference_seconds_init": round(t_init, 3), "reference_seconds_run": round(t_run, 3)}
    with open(os.path.join(HERE, f"{name}.json"), "w") as f:
        json.dump(meta, f, indent=1)
    return meta


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("HHG_REFERENCE", "/root/reference"))
    ap.add_argument("--only", nargs="*")
    args = ap.parse_args()
    lib = os.path.join(REPO, "oracle", "_ref", "libwannier.so")
    if not os.path.exists(lib):
        raise SystemExit("build the reference first: make -C oracle")
    os.environ.setdefault("OPENBLAS_NUM_THREADS", "1")
    pyswe = load_reference_pyswe(args.ref)
    for name, spec in CASES.items():
        if args.only and name not in args.only:
            continue
        meta = run_case(pyswe, lib, name, spec)
        print(name, json.dumps(meta), flush=True)


if __name__ == "__main__":
    main()
