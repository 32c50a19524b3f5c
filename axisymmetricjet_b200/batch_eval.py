"""Batched uneven jets against the same jets run one after another on the plain FP64 path.

64 instances (Nz in [256, 2048], Nr in [96, 384], both multiples of 32; Mach in
[0.9, 1.5], Re in [1000, 5000]; harmonic inflow forcing with amplitude up to 0.02 U_j and
Strouhal number in [0.2, 0.6]) advance `--steps` steps as one batch in the
mixed-precision + learned-sensor form (tile order and CTAs per SM picked by the
autotuner), and the same instances advance the same number of steps one after another
on the plain FP64 path. Reports both throughputs (RK4 grid-point updates/s, CUDA-event
device time), their ratio, and each instance's relative L2 error of rho and p against
its FP64 run.

    python -m axisymmetricjet_b200.batch_eval --instances 64 --steps 500
"""
import argparse
import json
import sys
import time

import numpy as np

import axisymmetricjet_b200 as axj
from axisymmetricjet_b200 import accuracy, fixtures


def make_solvers(cases, model=None):
    out = []
    for c in cases:
        patches = axj.patches_from_records(c["records"], c["Nz"], c["Nr"])
        s = axj.AxiJetSolver(c["params"], c["zvec"], c["rvec"], c["ibval"], patches)
        if model is not None:
            s.mlp_set(model)
        s.set_state(c["pv"], c["target"])
        out.append(s)
    return out


def evaluate(n=64, steps=500, seed=2024, warmup=3, tune_steps=3, precision=1, sensor=1, model=None, log=print,
             accuracy_check=True, judge_every=50, judge_stages=4, forms=None):
    """forms (optional): a list of dicts of (precision, sensor, judge_every, judge_stages) run as
    batches against one set of sequential FP64 runs; returns {"forms": [...], ...} then."""
    from axisymmetricjet_b200.train_sensor import load_model
    if sensor == 1 and model is None:
        model = load_model()
    base = fixtures.batch_instances(n, seed=seed)
    npts = sum(c["Nz"] * c["Nr"] for c in base)
    if forms is None:
        forms = [dict(precision=precision, sensor=sensor, judge_every=judge_every, judge_stages=judge_stages)]
    if len(forms) > 1:
        reps = [_batched(base, fm, n, steps, seed, warmup, tune_steps, model, log) for fm in forms]
        seq = _sequential(base, [r.pop("_states") for r in reps], steps, warmup, npts, accuracy_check, log)
        for r, errs in zip(reps, seq.pop("errs")):
            _attach(r, seq, errs)
        return {"instances": n, "steps": steps, "points": npts, "sequential_fp64": seq["sequential_fp64"],
                "forms": reps}
    fm = forms[0]
    precision, sensor = fm["precision"], fm["sensor"]
    fast = fixtures.batch_instances(n, seed=seed, precision=precision, sensor=sensor,
                                    judge_every=fm["judge_every"], judge_stages=fm["judge_stages"])
    rep = {"instances": n, "steps": steps, "points": npts, "precision": precision, "sensor": sensor,
           "judge_every": fm["judge_every"], "judge_stages": fm["judge_stages"]}

    # batched mixed + learned
    t0 = time.time()
    solvers = make_solvers(fast, model if sensor == 1 else None)
    batch = axj.AxjBatch(solvers)
    chosen, trials = batch.autotune(steps_per_trial=tune_steps)
    rep["tuning"] = chosen
    rep["autotune_trials_ms"] = trials
    batch.run(warmup)
    ms_b = batch.run_timed(steps - warmup) if steps > warmup else 0.0
    rep["batched"] = {"ms": ms_b, "ms_per_step": ms_b / max(steps - warmup, 1),
                      "value": npts * (steps - warmup) / (ms_b / 1e3) if ms_b > 0 else None}
    log(f"batched: {rep['batched']} (setup + run {time.time() - t0:.1f} s)")
    if sensor == 1:
        st = [s.learned_stats() for s in solvers]
        rep["judge"] = {"judged_outputs": sum(x["judged_outputs"] for x in st),
                        "fallbacks": sum(x["fallbacks"] for x in st)}
    fast_states = [s.get_state() for s in solvers]
    batch.close()
    for s in solvers:
        s.close()

    # the same instances one after another, plain FP64 (graph-captured steps each)
    t0 = time.time()
    seq_ms = 0.0
    errs = []
    for k, c in enumerate(base):
        s = make_solvers([c])[0]
        s.run(warmup)
        seq_ms += s.run_timed(steps - warmup) if steps > warmup else 0.0
        if accuracy_check:
            ref = s.get_state()
            e = accuracy.field_errors(fast_states[k], ref)
            errs.append({"Nz": c["Nz"], "Nr": c["Nr"], "rho": e["rho"]["rel_l2"], "p": e["p"]["rel_l2"]})
        s.close()
    rep["sequential_fp64"] = {"ms": seq_ms, "value": npts * (steps - warmup) / (seq_ms / 1e3) if seq_ms > 0 else None}
    log(f"sequential FP64: {rep['sequential_fp64']} ({time.time() - t0:.1f} s)")
    if rep["batched"]["value"] and rep["sequential_fp64"]["value"]:
        rep["speedup"] = rep["batched"]["value"] / rep["sequential_fp64"]["value"]
    if errs:
        rep["rel_l2_vs_fp64"] = {"rho_max": max(e["rho"] for e in errs), "p_max": max(e["p"] for e in errs),
                                 "rho_median": float(np.median([e["rho"] for e in errs])),
                                 "p_median": float(np.median([e["p"] for e in errs]))}
    return rep


def _batched(base, fm, n, steps, seed, warmup, tune_steps, model, log):
    from axisymmetricjet_b200.train_sensor import load_model
    sensor = fm["sensor"]
    if sensor == 1 and model is None:
        model = load_model()
    fast = fixtures.batch_instances(n, seed=seed, precision=fm["precision"], sensor=sensor,
                                    judge_every=fm["judge_every"], judge_stages=fm["judge_stages"])
    npts = sum(c["Nz"] * c["Nr"] for c in base)
    solvers = make_solvers(fast, model if sensor == 1 else None)
    batch = axj.AxjBatch(solvers)
    chosen, trials = batch.autotune(steps_per_trial=tune_steps)
    batch.run(warmup)
    ms_b = batch.run_timed(steps - warmup)
    rep = dict(fm, tuning=chosen, ms_per_step=ms_b / (steps - warmup), value=npts * (steps - warmup) / (ms_b / 1e3))
    if sensor == 1:
        st = [s.learned_stats() for s in solvers]
        rep["judge"] = {"judged_outputs": sum(x["judged_outputs"] for x in st),
                        "fallbacks": sum(x["fallbacks"] for x in st)}
    rep["_states"] = [s.get_state() for s in solvers]
    batch.close()
    for s in solvers:
        s.close()
    log(f"batched {fm}: {rep['value']:.3e}")
    return rep


def _sequential(base, states_per_form, steps, warmup, npts, accuracy_check, log):
    seq_ms = 0.0
    errs = [[] for _ in states_per_form]
    for k, c in enumerate(base):
        s = make_solvers([c])[0]
        s.run(warmup)
        seq_ms += s.run_timed(steps - warmup)
        if accuracy_check:
            ref = s.get_state()
            for f, states in enumerate(states_per_form):
                e = accuracy.field_errors(states[k], ref)
                errs[f].append({"rho": e["rho"]["rel_l2"], "p": e["p"]["rel_l2"]})
        s.close()
    value = npts * (steps - warmup) / (seq_ms / 1e3)
    log(f"sequential FP64: {value:.3e}")
    return {"sequential_fp64": {"ms": seq_ms, "value": value}, "errs": errs}


def _attach(rep, seq, errs):
    rep["speedup"] = rep["value"] / seq["sequential_fp64"]["value"]
    if errs:
        rep["rel_l2_vs_fp64"] = {"rho_max": max(e["rho"] for e in errs), "p_max": max(e["p"] for e in errs),
                                 "rho_median": float(np.median([e["rho"] for e in errs])),
                                 "p_median": float(np.median([e["p"] for e in errs]))}


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--instances", type=int, default=64)
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--precision", type=int, default=1)
    ap.add_argument("--sensor", type=int, default=1)
    ap.add_argument("--judge-every", type=int, default=50)
    ap.add_argument("--judge-stages", type=int, default=4)
    ap.add_argument("--report", default=None)
    args = ap.parse_args(argv)
    rep = evaluate(args.instances, args.steps, args.seed, precision=args.precision, sensor=args.sensor,
                   judge_every=args.judge_every, judge_stages=args.judge_stages,
                   log=lambda m: print(m, file=sys.stderr, flush=True))
    print(json.dumps(rep), flush=True)
    if args.report:
        with open(args.report, "w") as f:
            json.dump(rep, f, indent=1)
    return 0


if __name__ == "__main__":
    sys.exit(main())
