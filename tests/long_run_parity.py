"""Long-run FP64 parity of the production jet (4400 x 640, Mach 1.5, Re 5000, shock
capturing on, reference dt): per-field relative L2 error after many RK4 steps.

Two modes:

  calibrate   the oracle (no FMA contraction) against the same C source built with FMA
              contraction (liboracle_axj_fma.so). Both are correct FP64 evaluations of
              the reference's arithmetic that differ only in rounding, as the device
              path and the oracle do; their spread after N steps is how far two correct
              builds drift apart. Needs no GPU. Writes the spread per checkpoint.
  check       the device path (libaxj.so through the C-ABI, graph-replayed steps) against
              the oracle on the same initial state; every path computes its own dt
              (ComputeTimeStep, ModInputOutput.f90:389-438) and runs RK4
              (ModRungeKutta.f90:5-171). Writes the per-field relative L2 per checkpoint
              and, with --calibration, the tolerance: TOL_FACTOR x the calibrated spread
              at the same step, or the FP64 unit roundoff (2.2e-16) if that is larger
              (the first steps, where the spread is below it). Exits 1 if a field is out
              of tolerance.
  verdict     applies the same tolerance to a recorded check (--check) and rewrites it.

    python tests/long_run_parity.py calibrate --steps 1000 --out tests/golden/long_run_calibration.json
    python tests/long_run_parity.py check --steps 1000 --calibration tests/golden/long_run_calibration.json \\
        --out long_run_check.json
    python tests/long_run_parity.py verdict --check long_run_check.json \\
        --calibration tests/golden/long_run_calibration.json --out long_run_check.json

Fields: rho, V_r, V_z, T, relative L2 = ||a - b|| / ||b|| over the
grid; V_r is taken relative to the norm of V_z (V_r's own norm is the perturbation's).
The oracle is test infrastructure: only this script runs it.
"""
import argparse
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)

FIELDS = {"rho": 0, "V_r": 1, "V_z": 3, "T": 4}
TOL_FACTOR = 10.0
# a relative L2 below the FP64 unit roundoff is below what a norm of the field resolves:
# the floor for the first steps, where the spread is smaller still
FLOOR = 2.2e-16


def rel_l2(a, b):
    out = {}
    for name, k in FIELDS.items():
        ref = b[3] if name == "V_r" else b[k]
        out[name] = float(np.linalg.norm(a[k] - b[k]) / np.linalg.norm(ref))
    return out


def checkpoints(steps, every):
    pts = list(range(every, steps + 1, every))
    for s in (1, 3, 10):
        if s <= steps and s not in pts:
            pts.append(s)
    if steps not in pts:
        pts.append(steps)
    return sorted(pts)


def make_pair(kind, case_name):
    import oracle
    from axisymmetricjet_b200 import fixtures
    c = fixtures.case(case_name)
    op = oracle.patches_from_records(c["records"], c["Nz"], c["Nr"])
    a = oracle.Oracle(c["params"], c["zvec"], c["rvec"], c["ibval"], op)
    if kind == "calibrate":
        b = oracle.Oracle(c["params"], c["zvec"], c["rvec"], c["ibval"], op, variant="fma")
    else:
        import axisymmetricjet_b200 as axj
        gp = axj.patches_from_records(c["records"], c["Nz"], c["Nr"])
        assert gp == op
        b = axj.AxiJetSolver(c["params"], c["zvec"], c["rvec"], c["ibval"], gp)
    a.set_state(c["pv"], c["target"])
    b.set_state(c["pv"], c["target"])
    return c, a, b


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("mode", choices=["calibrate", "check", "verdict"])
    ap.add_argument("--check", default=None)
    ap.add_argument("--case", default="jet4400x640")
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--every", type=int, default=100)
    ap.add_argument("--calibration", default=None)
    ap.add_argument("--out", required=True)
    args = ap.parse_args(argv)

    if args.mode == "verdict":
        out = json.load(open(args.check))
        rows = out["checkpoints"]
    else:
        c, ora, other = make_pair(args.mode, args.case)
        pts = checkpoints(args.steps, args.every)
        rows = []
        max_dt_rel = 0.0
        t0 = time.time()
        done = 0
        for p in pts:
            for _ in range(p - done):
                d_o = ora.compute_time_step()
                d_b = other.compute_time_step()
                max_dt_rel = max(max_dt_rel, abs(d_b - d_o) / abs(d_o))
                ora.rk4(d_o)
                other.rk4(d_b)
            done = p
            err = rel_l2(other.get_state(), ora.get_state())
            rows.append(dict(step=p, time=ora.get_time()[1], l2=err, max_dt_rel=max_dt_rel))
            print(json.dumps(rows[-1]), f"{time.time() - t0:.0f}s", flush=True)
        out = dict(mode=args.mode, case=args.case, Nz=c["Nz"], Nr=c["Nr"], steps=args.steps,
                   compared=("oracle vs oracle built with FMA contraction" if args.mode == "calibrate"
                             else "device FP64 path vs oracle"), checkpoints=rows, seconds=time.time() - t0)
    rc = 0
    if args.mode in ("check", "verdict") and args.calibration:
        cal = json.load(open(args.calibration))
        spread = {r["step"]: r["l2"] for r in cal["checkpoints"]}
        verdict = []
        for r in rows:
            if r["step"] not in spread:
                continue
            tol = {k: max(TOL_FACTOR * spread[r["step"]][k], FLOOR) for k in FIELDS}
            ok = all(r["l2"][k] <= tol[k] for k in FIELDS)
            verdict.append(dict(step=r["step"], tol=tol, ok=ok,
                                margin=min(tol[k] / max(r["l2"][k], 1e-300) for k in FIELDS)))
            rc |= 0 if ok else 1
        out["tolerance_rule"] = (f"per field: max({TOL_FACTOR:g} x the calibrated spread at the step, "
                                 f"{FLOOR:g})")
        out["verdict"] = verdict
        out["pass"] = rc == 0
    with open(args.out, "w") as f:
        json.dump(out, f, indent=1)
    return rc


if __name__ == "__main__":
    sys.exit(main())
