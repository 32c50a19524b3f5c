"""Train the learned artificial-diffusivity sensor on snapshots the solver generates.

Runs the plain FP64 solver (shock capturing on) on one grid at several jet Mach
numbers, adds a snapshot (feature channels + the plain sensor's betastar, kappastar)
every `--every` steps to the device data set, then trains the MLP with Adam on the
device and writes the model to an .npz file (the fields of axj_mlp plus the loss
history and the run's settings).

    python -m axisymmetricjet_b200.train_sensor --case jet4400x640 --machs 1.2,1.5,1.8 \\
        --snapshots 200 --every 15 --steps 2000 --batch 65536 --out sensor_mlp.npz
"""
import argparse
import json
import os
import sys
import time

import numpy as np

import axisymmetricjet_b200 as axj
from axisymmetricjet_b200 import fixtures

MODEL_FILE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "sensor_mlp_jet4400x640.npz")


def load_model(path=MODEL_FILE):
    """The model dict stored by save_model (the fields of axj_mlp)."""
    with np.load(path) as z:
        return {k: z[k].astype(np.float32) for k in axj.AxjMlp.SHAPES}


def save_model(path, model, **extra):
    arrays = {k: np.asarray(v, dtype=np.float32) for k, v in model.items()}
    meta = {k: v for k, v in extra.items() if not isinstance(v, np.ndarray)}
    arrays.update({k: v for k, v in extra.items() if isinstance(v, np.ndarray)})
    arrays["meta_json"] = np.frombuffer(json.dumps(meta).encode(), dtype=np.uint8)
    np.savez(path, **arrays)


def generate(case, machs, nsnap, every, seed=12345, log=print):
    """A solver handle of `case` whose data set holds nsnap snapshots spread over the
    Mach numbers; returns (solver, seconds)."""
    spec = dict(fixtures.CASES[case])
    c = fixtures.case(case, Mj=machs[0], seed=seed)
    patches = axj.patches_from_records(c["records"], c["Nz"], c["Nr"])
    s = axj.AxiJetSolver(c["params"], c["zvec"], c["rvec"], c["ibval"], patches)
    s.dataset_reserve(nsnap)
    t0 = time.time()
    per = [nsnap // len(machs) + (1 if k < nsnap % len(machs) else 0) for k in range(len(machs))]
    for Mj, n in zip(machs, per):
        cm = fixtures.make_case(**dict(spec, Mj=Mj, seed=seed))
        s.set_state(cm["pv"], cm["target"])
        for _ in range(n):
            s.run(every)
            s.dataset_add()
        log(f"Mach {Mj}: {n} snapshots, every {every} steps")
    return s, time.time() - t0


SENSORS = {"plain": 0, "learned": 1, "held": 2}


def evaluate(model, case, Mj, steps, seed=777, judge_every=50, threshold=0.1, precision=0, timing_steps=50,
             log=print):
    """Advance the same initial state `steps` steps with the plain sensor, the learned
    sensor and the held-coefficient baseline (same dt sequence, from the plain run) and
    report each one's error against the plain run and its graph-replayed step time."""
    from axisymmetricjet_b200 import accuracy
    spec = dict(fixtures.CASES[case], Mj=Mj, seed=seed)
    solvers, report = {}, {"case": case, "Mj": Mj, "steps": steps, "judge_every": judge_every,
                           "threshold": threshold, "precision": precision, "modes": {}}
    for name, kind in SENSORS.items():
        c = fixtures.make_case(**dict(spec, sensor=kind, judge_every=judge_every, judge_threshold=threshold,
                                      precision=precision if name != "plain" else 0))
        patches = axj.patches_from_records(c["records"], c["Nz"], c["Nr"])
        sv = axj.AxiJetSolver(c["params"], c["zvec"], c["rvec"], c["ibval"], patches)
        if name == "learned":
            sv.mlp_set(model)
        sv.set_state(c["pv"], c["target"])
        solvers[name] = (sv, c)
    ref = solvers["plain"][0]
    for _ in range(steps):
        dt = ref.compute_time_step()
        for sv, _ in solvers.values():
            sv.rk4(dt)
    base = ref.get_state()
    for name, (sv, c) in solvers.items():
        entry = {}
        if name != "plain":
            entry["errors_vs_plain"] = accuracy.field_errors(sv.get_state(), base)
        if name == "learned":
            entry["judge"] = sv.learned_stats()
        # step time: graph-replayed steps on the same handle from its current state
        sv.run(5)
        entry["ms_per_step"] = sv.run_timed(timing_steps) / timing_steps
        report["modes"][name] = entry
        log(f"{name}: {json.dumps(entry)[:300]}")
        sv.close()
    return report


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--case", default="jet4400x640")
    ap.add_argument("--machs", default="1.2,1.5,1.8")
    ap.add_argument("--snapshots", type=int, default=200)
    ap.add_argument("--every", type=int, default=15)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--batch", type=int, default=65536)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--out", default=MODEL_FILE)
    ap.add_argument("--evaluate-steps", type=int, default=0,
                    help="after training, compare plain / learned / held sensors over this many steps")
    ap.add_argument("--eval-mach", type=float, default=1.5)
    ap.add_argument("--eval-precision", type=int, default=0)
    ap.add_argument("--report", default=None, help="write the training and evaluation summary (JSON) here")
    args = ap.parse_args(argv)
    machs = [float(m) for m in args.machs.split(",")]

    def log(msg):
        print(msg, file=sys.stderr, flush=True)

    s, t_gen = generate(args.case, machs, args.snapshots, args.every, log=log)
    s.mlp_set(axj.mlp_init(args.seed))
    t0 = time.time()
    loss = s.mlp_train(steps=args.steps, batch=args.batch, lr=args.lr, seed=args.seed, fit_normalization=1)
    t_train = time.time() - t0
    model = s.mlp_get()
    s.close()
    save_model(args.out, model, loss=loss, case=args.case, machs=machs, snapshots=args.snapshots,
               every=args.every, steps=args.steps, batch=args.batch, lr=args.lr, seed=args.seed)
    tail = float(np.mean(loss[-50:])) if len(loss) else None
    summary = {"case": args.case, "machs": machs, "snapshots": args.snapshots, "every": args.every,
               "steps": args.steps, "batch": args.batch, "generate_s": t_gen, "train_s": t_train,
               "loss_first": float(loss[0]) if len(loss) else None, "loss_last50": tail,
               "loss_at": {str(k): float(loss[k]) for k in (0, 10, 100, 500, 1000, 1999) if k < len(loss)},
               "out": args.out}
    if args.evaluate_steps > 0:
        summary["evaluation"] = evaluate(model, args.case, args.eval_mach, args.evaluate_steps,
                                         precision=args.eval_precision, log=log)
    print(json.dumps(summary), flush=True)
    if args.report:
        with open(args.report, "w") as f:
            json.dump(summary, f, indent=1)
    return 0


if __name__ == "__main__":
    sys.exit(main())
