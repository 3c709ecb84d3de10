"""Precision study of the population storage forms.

    python -m komegafoulingmodel_b200.precision --workload komega_straight_16384x1024 \
        --steps 20000 [--forms fp32,fp16,bf16,fp16neq]

Runs the same seeded channel once per storage form (FP64 throughout; FP32 /
FP16 / BF16 deviations f - w_i; FP16 non-equilibrium parts f - feq with
FP64 or FP32 collide arithmetic) and
reports, for every other form, the rel-L2 of u_x, k and omega over the fluid
nodes against the reference form -- the FP64 form when it is among the forms
(the reference's own precision, held to the FP64 oracle by the test suite),
else the FP32 form -- (u_y, ~0 in a straight channel, relative to |u|), the
mass drift (sum rho at the end over sum rho at the start, minus 1) of every
form, and each form's device-resident throughput.  Prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import _abi
from . import workloads as W
from .lattice import Lattice

FORMS = {"fp64": _abi.STORE_FP64, "fp32": _abi.STORE_FP32, "fp16": _abi.STORE_FP16_DEV,
         "bf16": _abi.STORE_BF16_DEV, "fp16neq": _abi.STORE_FP16_NEQ,
         "fp16neq32": _abi.STORE_FP16_NEQ32, "fp16row": _abi.STORE_FP16_ROW}


def rel_l2(a, b, mask):
    d = np.linalg.norm((a - b)[mask])
    n = np.linalg.norm(b[mask])
    return float(d / n) if n > 0 else float(d)


def run_form(w, form: str, steps: int, chunk: int = 500):
    d = W.descriptor(w, storage=FORMS[form])
    with Lattice(d) as L:
        W.apply(L, w)
        L.step(1)
        m0 = L.reduce(_abi.FIELD_RHO)
        L.sync()
        t0 = time.perf_counter()
        left = steps - 1
        while left > 0:
            n = min(chunk, left)
            L.step(n)
            left -= n
        L.sync()
        secs = time.perf_counter() - t0
        m1 = L.reduce(_abi.FIELD_RHO)
        rho, ux, uy = L.get_macro()
        _, k, o, _, _ = L.get_state() if w.komega else (None, None, None, None, None)
    return {"ux": ux, "uy": uy, "k": k, "omega": o, "mass_drift": m1 / m0 - 1.0,
            "mlups": w.nodes * max(steps - 1, 1) / secs / 1e6}


def study(workload: str, steps: int, forms=("fp64", "fp32", "fp16", "bf16", "fp16neq", "fp16neq32")) -> dict:
    w = W.by_name(workload)
    fl = w.channel.fluid_mask().ravel()
    ref_form = "fp64" if "fp64" in forms else "fp32"
    res = {f: run_form(w, f, steps) for f in forms}  # one form on the device at a time
    out = {"workload": workload, "steps": steps, "reference_form": ref_form, "forms": {}}
    base = res.get(ref_form)
    for f, r in res.items():
        e = {"mass_drift": r["mass_drift"], "mlups_wall": r["mlups"]}
        if base is not None and f != ref_form:
            for key in ("ux", "k", "omega"):
                if r[key] is not None:
                    e[f"rel_l2_{key}"] = rel_l2(r[key], base[key], fl)
            # u_y is ~0 in a straight channel: its error relative to |u|
            e["l2_uy_over_l2_u"] = float(np.linalg.norm((r["uy"] - base["uy"])[fl]) /
                                         np.linalg.norm(np.hypot(base["ux"], base["uy"])[fl]))
        out["forms"][f] = e
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="komega_straight_16384x1024")
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--forms", default="fp64,fp32,fp16,bf16,fp16neq,fp16neq32")
    args = ap.parse_args()
    print(json.dumps(study(args.workload, args.steps, tuple(args.forms.split(",")))), flush=True)


if __name__ == "__main__":
    main()
