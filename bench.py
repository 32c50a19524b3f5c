"""Throughput of the per-step hot path: RK4 grid-point updates per second.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--case NAME]

Workload (default): jet4400x640 -- Nz=4400 x Nr=640 axisymmetric jet, M_j=1.5, Re=5000,
artificial-diffusivity shock capturing on, SAT/NSCBC faces, sponges, FP64 end to end,
synthetic seeded initial condition. One step = ComputeTimeStep + one RK4 step
(4 right-hand-side evaluations, each with the sensor chain).

Multi-GPU: one process per GPU (torchrun); every rank advances its own jet (replicas,
no data-path collective); the timed region is bracketed by barriers and the device
time is the max over ranks; value = total updates of all ranks / that time.

--impl reference times the CPU implementation of the same step on the host cores:
the reference Fortran cannot be built in this image (no Fortran compiler), so it is
the oracle's line-faithful C restatement (OpenMP over columns, all host threads).
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "RK4 grid-pt updates/s"
UNIT = "grid-pt updates/s"
# Algorithmic bytes of the FP64 path: 680 B per grid point per RK4 step (5 fields x 8 B x
# 17 state accesses), i.e. 170 B per point per RK stage launch.
ALG_BYTES_PER_POINT_STEP = 680.0
ALG_BYTES_PER_POINT_STAGE = ALG_BYTES_PER_POINT_STEP / 4.0
NOUTPUT = 200  # WriteOutput period of the reference (ModuleVariables.f90:69)


def env_int(k, d):
    try:
        return int(os.environ.get(k, d))
    except ValueError:
        return d


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profile_traffic(case):
    """dram bytes per stage-kernel launch from the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", f"stage_kernel_{case}.txt")
    try:
        for line in open(path):
            if line.startswith("traffic_bytes_per_stage_launch"):
                return float(line.split("=")[1].split()[0])
    except Exception:
        pass
    return None


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 50 ms; the summary keeps the
    samples read between mark_start() and mark_end() (the timed region)."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None
        self.t0 = self.t1 = None

    def mark_start(self):
        self.t0 = time.time()

    def mark_end(self):
        self.t1 = time.time()

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append((time.time(), [x.strip() for x in line.split(",")]))

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.1)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = [r for t, r in self.rows
                if self.t0 is None or self.t1 is None or (self.t0 <= t <= self.t1 + 0.06)]
        if not rows:
            rows = [r for _, r in self.rows]
        self.rows = rows
        sm = [float(r[1]) for r in self.rows if len(r) >= 9 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) >= 9 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            if len(r) >= 9:
                for n, v in zip(names, r[5:9]):
                    if v.lower() == "active":
                        reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.rows)}


def host_cpu():
    """(logical CPUs, physical cores, CPU model) of this host."""
    logical = os.cpu_count() or 1
    physical = None
    try:
        import psutil
        physical = psutil.cpu_count(logical=False)
    except Exception:
        pass
    model = None
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                model = line.split(":", 1)[1].strip()
                break
    except Exception:
        pass
    return logical, physical, model


def cpu_step_sample(case, threads, steps=15, warmup=2):
    """Oracle (CPU restatement) on the full workload grid: seconds per RK4 step over
    `steps` steps after `warmup` untimed ones (the first step also touches every page)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    os.environ["OMP_NUM_THREADS"] = str(threads)
    import oracle
    from axisymmetricjet_b200 import fixtures
    c = fixtures.case(case)
    ora = oracle.Oracle(c["params"], c["zvec"], c["rvec"], c["ibval"],
                        oracle.patches_from_records(c["records"], c["Nz"], c["Nr"]))
    ora.set_state(c["pv"], c["target"])
    for _ in range(warmup):
        ora.rk4(ora.compute_time_step())
    t0 = time.perf_counter()
    for _ in range(steps):
        d = ora.compute_time_step()
        ora.rk4(d)
    return (time.perf_counter() - t0) / steps, c["Nz"] * c["Nr"]


def run_reference(args):
    rank = env_int("RANK", 0)
    if rank != 0:
        return 0
    threads, physical, model = host_cpu()
    os.environ["OMP_NUM_THREADS"] = str(threads)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    from axisymmetricjet_b200 import fixtures
    c = fixtures.case(args.case)
    ora = oracle.Oracle(c["params"], c["zvec"], c["rvec"], c["ibval"],
                        oracle.patches_from_records(c["records"], c["Nz"], c["Nr"]))
    ora.set_state(c["pv"], c["target"])
    for _ in range(args.warmup):
        ora.rk4(ora.compute_time_step())
    t0 = time.perf_counter()
    for _ in range(args.steps):
        ora.rk4(ora.compute_time_step())
    sec = time.perf_counter() - t0
    npts = c["Nz"] * c["Nr"]
    value = npts * args.steps / sec
    sample = f"{args.steps} full RK4 steps (ComputeTimeStep + RK4) of {args.case} after {args.warmup} warm-up steps"
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sec / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(args.case, c),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "physical_cores": physical,
                         "cpu_model": model, "kind": "port",
                         "sample": sample + "; CPU restatement of the reference (oracle/axj_oracle.c, -O2 "
                                            "-ffp-contract=off, OpenMP), not the Fortran binary: no Fortran "
                                            "compiler in this image"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def reduce_max(x, world, device):
    """Max of a per-rank time over all ranks (the device time of the slowest replica)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(npts, steps, world, ms_max):
    """Whole-job updates/s: every rank advances its own jet of npts points."""
    return world * npts * steps / (ms_max / 1e3)


def workload_config(name, c):
    p = c["params"]
    return {"workload": f"{name}: axisymmetric jet Nz={c['Nz']} x Nr={c['Nr']}, M_j={c['Mj']}, Re={p.Re:g}, "
                        f"shock capturing {'on' if p.shock_capturing else 'off'}, SAT/NSCBC + sponges, FP64",
            "Nz": c["Nz"], "Nr": c["Nr"], "shock_capturing": bool(p.shock_capturing),
            "l2": "inputs larger than L2 (about 1.6 GB of state, RK and sensor buffers touched per step)"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None,
                    help="timed steps (default 200 on the GPU; 20 for --impl reference, 1.3 s each on the CPU)")
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--case", default="jet4400x640")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--profile-steps", type=int, default=10)
    ap.add_argument("--no-variants", action="store_true",
                    help="skip the timing of the mixed-precision form of the same workload")
    ap.add_argument("--batch-steps", type=int, default=500,
                    help="steps of the batched 64-jet variant (0: skip it)")
    ap.add_argument("--batch-instances", type=int, default=64)
    args = ap.parse_args()
    if args.steps is None:
        args.steps = 20 if args.impl == "reference" else 200
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        return run_reference(args)

    import torch
    import torch.distributed as dist

    import axisymmetricjet_b200 as axj
    from axisymmetricjet_b200 import fixtures

    rank, world, local = env_int("RANK", 0), env_int("WORLD_SIZE", 1), env_int("LOCAL_RANK", 0)
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        return reduce_max(x, world, "cuda")

    c = fixtures.case(args.case, seed=12345 + rank)
    c["params"].device = local
    patches = axj.patches_from_records(c["records"], c["Nz"], c["Nr"])
    npts = c["Nz"] * c["Nr"]
    solver = axj.AxiJetSolver(c["params"], c["zvec"], c["rvec"], c["ibval"], patches)
    solver.set_state(c["pv"], c["target"])

    # warm-up (also builds the CUDA graph)
    solver.run(args.warmup)
    barrier()
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.2)  # the sampler is running before the timed region starts
    barrier()
    clocks.mark_start()
    ms = solver.run_timed(args.steps)
    barrier()
    clocks.mark_end()
    clk = clocks.stop()
    ms_max = max_over_ranks(ms)
    value = replica_throughput(npts, args.steps, world, ms_max)

    # per-kernel breakdown (same kernels launched one group at a time with CUDA events)
    prof_steps = max(1, args.profile_steps)
    pms, plaunch = solver.profile_steps(prof_steps)
    stage_launch_ms = pms["stage"] / (4 * prof_steps)
    peak, peak_kind = measured_peaks()
    alg_bytes = ALG_BYTES_PER_POINT_STAGE * npts
    achieved = alg_bytes / (stage_launch_ms / 1e3) / 1e9
    traffic = profile_traffic(args.case)
    launches_per_step = sum(plaunch.values()) // prof_steps  # the timed graph replays the same launches

    e2e = run_e2e(args, c, patches, npts, world, barrier, max_over_ranks) if not args.no_e2e else None

    variants = None
    if not args.no_variants:
        from axisymmetricjet_b200.train_sensor import MODEL_FILE, load_model
        variants = {"mixed": time_variant(args, c, patches, npts, world, barrier, max_over_ranks, precision=1)}
        if os.path.exists(MODEL_FILE):
            # the timed steps hold the plain sensor's judge steps in proportion: a whole number
            # of judge periods (the judge runs on every judge_every-th iteration)
            je = int(c["params"].judge_every) or 50
            variants["mixed_learned"] = time_variant(args, c, patches, npts, world, barrier, max_over_ranks,
                                                     model=load_model(), steps=je * -(-args.steps // je),
                                                     precision=1, sensor=1)
        for v in variants.values():
            v["speedup_vs_fp64"] = v["value"] / value
        if args.batch_steps > 0:
            variants["batched"] = time_batched(args, rank)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads, physical, model = host_cpu()
        cw, cs = 2, 15
        sec, n = cpu_step_sample(args.case, threads, steps=cs, warmup=cw)
        cpu = {"value": n / sec, "unit": UNIT, "cores": threads, "physical_cores": physical, "cpu_model": model,
               "kind": "port",
               "sample": f"{cs} full RK4 steps (ComputeTimeStep + RK4) of {args.case} after {cw} warm-up steps, "
                         f"by the oracle's C restatement of the reference (OpenMP, {threads} threads on "
                         f"{physical} physical cores): {sec:.2f} s per step"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(args.case, c),
            "parallelism": f"replicas x{world} (one jet per GPU, no data-path collective)",
            "roofline": {"bound": "hbm", "kernel": "stage_kernel (fused RK stage, both tile classes)",
                         "achieved": achieved, "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "alg_bytes_per_launch": alg_bytes, "launch_ms": stage_launch_ms},
            "breakdown_ms_per_step": {k: v / prof_steps for k, v in pms.items()},
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": launches_per_step * args.steps,
            "clocks": clk,
            "variants": variants,
        }
        print(json.dumps(line), flush=True)
    solver.close()
    if world > 1:
        dist.destroy_process_group()
    return 0


def time_batched(args, rank):
    """The batched form of uneven jets: 64 instances (Nz in [256, 2048], Nr in [96, 384],
    Mach in [0.9, 1.5], Re in [1000, 5000], harmonic inflow forcing) in one persistent launch
    per kernel, mixed precision, autotuned (tile order, stage tile shape, CTAs per SM, the
    general tiles' CTAs per SM and stream),
    graph-captured steps; against the same instances one after another on the plain FP64
    path, with each instance's relative L2 error of rho and p against its FP64 run after the
    same number of steps. Forms: the learned sensor judged every 50 steps (the plain sensor
    on all four stages of a judge step), the learned and the held sensor judged on the first
    stage of every second step, and the plain sensor on every stage. Every rank runs its own
    batch (replicas); the figures are rank 0's."""
    from axisymmetricjet_b200 import batch_eval
    forms = [dict(name="learned_judge50", precision=1, sensor=1, judge_every=50, judge_stages=4),
             dict(name="learned_judge2_stage1", precision=1, sensor=1, judge_every=2, judge_stages=1),
             dict(name="held_judge2_stage1", precision=1, sensor=2, judge_every=2, judge_stages=1),
             dict(name="plain", precision=1, sensor=0, judge_every=50, judge_stages=4)]
    names = [f.pop("name") for f in forms]
    rep = batch_eval.evaluate(n=args.batch_instances, steps=args.batch_steps, seed=2024 + rank, forms=forms,
                              log=lambda m: None)
    out = {"instances": rep["instances"], "points": rep["points"], "steps": rep["steps"],
           "timed_steps": rep["steps"] - 3, "unit": UNIT,
           "sequential_fp64_value": rep["sequential_fp64"]["value"], "forms": {}}
    for name, r in zip(names, rep["forms"]):
        out["forms"][name] = {k: r.get(k) for k in ("precision", "sensor", "judge_every", "judge_stages", "tuning",
                                                     "value", "ms_per_step", "speedup", "rel_l2_vs_fp64", "judge")}
    return out


def time_variant(args, c, patches, npts, world, barrier, max_over_ranks, model=None, steps=None, **pkw):
    """The same workload and timing (graph-captured steps, CUDA events, max over ranks)
    with changed solver parameters, e.g. precision = AXJ_MIXED; `model` is installed for
    the learned sensor (its judge steps are part of the timed steps)."""
    steps = steps or args.steps
    import axisymmetricjet_b200 as axj
    from axisymmetricjet_b200._ffi import AxjParams
    prm = AxjParams.from_buffer_copy(c["params"])
    for k, v in pkw.items():
        setattr(prm, k, v)
    s = axj.AxiJetSolver(prm, c["zvec"], c["rvec"], c["ibval"], patches)
    if model is not None:
        s.mlp_set(model)
    s.set_state(c["pv"], c["target"])
    s.run(args.warmup)
    barrier()
    ms = max_over_ranks(s.run_timed(steps))
    barrier()
    out = {"params": dict(pkw), "value": replica_throughput(npts, steps, world, ms), "unit": UNIT,
           "ms_per_step": ms / steps, "steps": steps}
    if model is not None:
        st = s.learned_stats()
        out["judge"] = dict(st, timed_steps=steps, judge_every=int(prm.judge_every))
    s.close()
    return out


def run_e2e(args, c, patches, npts, world, barrier, max_over_ranks):
    """End to end through the public API with host buffers: IC and target upload, every
    step ComputeTimeStep (dt to the host) + RK4(delt), the state downloaded every
    NOUTPUT steps and at the end (ModRungeKutta.f90:161-165)."""
    import torch

    import axisymmetricjet_b200 as axj
    e2e_solver = axj.AxiJetSolver(c["params"], c["zvec"], c["rvec"], c["ibval"], patches)
    pv_h = torch.from_numpy(c["pv"]).pin_memory().numpy()
    tg_h = torch.from_numpy(c["target"]).pin_memory().numpy()
    out_h = torch.empty(c["pv"].shape, dtype=torch.float64).pin_memory().numpy()
    e2e_solver.set_state(pv_h, tg_h)
    for _ in range(args.warmup):
        e2e_solver.rk4(e2e_solver.compute_time_step())
    barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    e2e_solver.set_state(pv_h, tg_h)
    nout = 0
    for s in range(1, args.steps + 1):
        e2e_solver.rk4(e2e_solver.compute_time_step())
        if s % NOUTPUT == 0:
            e2e_solver.get_state(out_h)
            nout += 1
    e2e_solver.get_state(out_h)
    nout += 1
    ev1.record()
    barrier()
    e2e_ms = max_over_ranks(ev0.elapsed_time(ev1))
    state_bytes = 5 * npts * 8
    e2e = {"value": world * npts * args.steps / (e2e_ms / 1e3), "unit": UNIT,
           "h2d_bytes_per_step": (2 * state_bytes + 8 * args.steps) / args.steps,
           "d2h_bytes_per_step": (nout * state_bytes + 12 * args.steps) / args.steps}
    e2e_solver.close()
    return e2e


if __name__ == "__main__":
    sys.exit(main())
