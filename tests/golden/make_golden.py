"""Generate the committed golden fixtures of the parity tests.

Run in a checkout that has the reference project (its directory given by
--ref or the environment variable CCFD_REFERENCE_DIR) and the compiled reference oracle (``make -C oracle``):

    python tests/golden/make_golden.py --ref /path/to/ccfd

Outputs (small, committed):
  sod_check.json    the reference's own regression suite (check/*.ini with
                    check/targetOutput/*.csv): per case the .ini text and the
                    golden x, density, velocity columns at t = 0.25
  ref_small.npz     outputs of the compiled reference (oracle/_ref) on small
                    synthetic cases: residuals at seeded random states for
                    every flux function and limiter, every boundary type,
                    Navier-Stokes, and short explicit runs
  ref_output.json   the compiled reference's own solution files (curve /
                    CSV, with the exact-solution file) of small runs
The synthetic cases themselves are described by CASES below and rebuilt by
the tests from the same generators and seeds.
"""
from __future__ import annotations

import argparse
import glob
import json
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from tests.golden import cases as CASES  # noqa: E402
from oracle import refdump  # noqa: E402


def sod_check(ref: str) -> dict:
    out = {}
    for ini in sorted(glob.glob(os.path.join(ref, "check", "*.ini"))):
        name = os.path.basename(ini)[:-4]
        tgt = sorted(glob.glob(os.path.join(ref, "check", "targetOutput", f"{name}_*")))[-1]
        data = np.genfromtxt(tgt, skip_header=1, delimiter=",")[:, 0:3]
        with open(ini) as f:
            text = f.read()
        out[name] = {"ini": text, "target": os.path.basename(tgt),
                     "x": data[:, 0].tolist(), "rho": data[:, 1].tolist(),
                     "u": data[:, 2].tolist()}
    return out


def ref_small(only: str | None = None) -> dict:
    """Reference outputs of every case, or of the cases whose key starts
    with ``only``."""
    arrays = {}
    pick = lambda d: {k: v for k, v in d.items() if only is None or k.startswith(only)}
    with tempfile.TemporaryDirectory() as tmp:
        for key, spec in pick(CASES.residual_cases()).items():
            ini, files = CASES.materialise(spec, tmp)
            prim = CASES.random_state(spec, tmp)
            d = refdump.run_ref(ini, "residual", spec["time"], state=prim, eqn=spec["eqn"],
                                files=files)
            arrays[f"{key}/u_t"] = d["u_t"]
            arrays[f"{key}/u_x"] = d["u_x"]
            arrays[f"{key}/u_y"] = d["u_y"]
            arrays[f"{key}/prim"] = prim.ravel()
        for key, spec in pick(CASES.run_cases()).items():
            ini, files = CASES.materialise(spec, tmp)
            d = refdump.run_ref(ini, "run", spec["steps"], eqn=spec["eqn"], files=files)
            arrays[f"{key}/pvar"] = d["pvar"]
            arrays[f"{key}/info"] = d["run_info"]
            arrays[f"{key}/history"] = d["history"]
            if "errors_printed" in d:
                arrays[f"{key}/errors_printed"] = d["errors_printed"]
                arrays[f"{key}/err_u_x"] = d["err_u_x"]
                arrays[f"{key}/err_u_y"] = d["err_u_y"]
        for key, spec in pick(CASES.implicit_cases()).items():
            ini, files = CASES.materialise(spec, tmp)
            d = refdump.run_ref(ini, "coef", spec["steps"], eqn=spec["eqn"], files=files,
                                rel_abort=spec.get("rel_abort"))
            arrays[f"{key}/pvar"] = d["pvar"]
            arrays[f"{key}/info"] = d["run_info"]
            arrays[f"{key}/history"] = d["history"]
            for name in ("clcd", "cp_pressure", "cp_suction"):
                if name in d:  # cases with calcWing
                    arrays[f"{key}/{name}"] = d[name]
    return arrays


def ref_output() -> dict:
    """The reference's own output files (and final state) of the output
    cases."""
    out = {}
    with tempfile.TemporaryDirectory() as tmp:
        for key, spec in CASES.output_cases().items():
            ini, files = CASES.materialise(spec, tmp)
            d = refdump.run_ref(ini, "run", 0, eqn=spec["eqn"], output=True, files=files)
            out[key] = {"files": d["output_files"], "pvar": d["pvar"].tolist(),
                        "history": d["history"].tolist(),
                        "t": float(d["run_info"][0]), "iterations": int(d["run_info"][1])}
    return out


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("CCFD_REFERENCE_DIR"),
                    help="reference project directory (default: $CCFD_REFERENCE_DIR)")
    ap.add_argument("--only", default=None,
                    help="regenerate only the cases whose key starts with this prefix and "
                         "merge them into the existing ref_small.npz")
    a = ap.parse_args()
    if not a.ref or not os.path.isdir(a.ref):
        print("reference project not found: pass --ref or set CCFD_REFERENCE_DIR", file=sys.stderr)
        return 1
    if not refdump.have_ref("euler") or not refdump.have_ref("navierstokes"):
        print("compiled reference missing: run `make -C oracle` first", file=sys.stderr)
        return 1
    npz = os.path.join(HERE, "ref_small.npz")
    if a.only == "out":
        with open(os.path.join(HERE, "ref_output.json"), "w") as f:
            json.dump(ref_output(), f)
        print("wrote ref_output.json")
        return 0
    if a.only:
        with np.load(npz) as old:
            arrays = {k: old[k] for k in old.files}
        arrays.update(ref_small(a.only))
        np.savez_compressed(npz, **arrays)
        print(f"updated ref_small.npz ({a.only}*)")
        return 0
    with open(os.path.join(HERE, "sod_check.json"), "w") as f:
        json.dump(sod_check(a.ref), f)
    np.savez_compressed(npz, **ref_small())
    with open(os.path.join(HERE, "ref_output.json"), "w") as f:
        json.dump(ref_output(), f)
    print("wrote sod_check.json, ref_small.npz, ref_output.json")
    return 0


if __name__ == "__main__":
    sys.exit(main())
