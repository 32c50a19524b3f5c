"""Batches: many uneven jets advanced by one launch per kernel.

The batched kernels run the same per-tile source as a single instance's kernels, but
they are separate compilations, so FMA contraction may differ in the last bit: a batch
must reproduce every instance's own run to 1e-12 relative per field after 7 steps on
the FP64 path (the per-step parity bar), and to 1e-6 with FP32 stage states and the
learned sensor (judge steps included). Both tile orders are checked, and the
autotuner's undo of its trial steps.
"""
import numpy as np
import pytest

import axisymmetricjet_b200 as axj
from axisymmetricjet_b200 import fixtures

SMALL = dict(nz_range=(128, 256), nr_range=(64, 128))  # stable over the test steps (checked with the oracle)


def _solvers(cases, model=None):
    out = []
    for c in cases:
        patches = axj.patches_from_records(c["records"], c["Nz"], c["Nr"])
        s = axj.AxiJetSolver(c["params"], c["zvec"], c["rvec"], c["ibval"], patches)
        if model is not None:
            s.mlp_set(model)
        s.set_state(c["pv"], c["target"])
        out.append(s)
    return out


def test_batch_instances_follow_the_distribution():
    cases = fixtures.batch_instances(64)
    assert len(cases) == 64
    for c in cases:
        assert c["Nz"] % 32 == 0 and 256 <= c["Nz"] <= 2048
        assert c["Nr"] % 32 == 0 and 96 <= c["Nr"] <= 384
        assert 0.9 <= c["Mj"] <= 1.5 and 1000.0 <= c["Re"] <= 5000.0
        assert 0.0 <= c["amp"] <= 0.02 * c["Mj"] and 0.2 <= c["St"] <= 0.6
        assert c["params"].control_forcing == 2 and c["params"].shock_capturing == 1
    again = fixtures.batch_instances(64)
    assert [c["Nz"] for c in cases] == [c["Nz"] for c in again]


def _model(cases):
    m = axj.mlp_init(3)
    m["out_scale"] = np.array([1e-3, 1e-3], dtype=np.float32)
    return m


MODES = {
    "fp64": {},
    "mixed_learned": dict(precision=1, sensor=1, judge_every=3),
    # the plain sensor on the first stage of every second step only (judge_stages = 1)
    "mixed_held_stage1": dict(precision=1, sensor=2, judge_every=2, judge_stages=1),
}


@pytest.mark.gpu
@pytest.mark.parametrize("mode", list(MODES))
@pytest.mark.parametrize("order,rows,gen_ctas,gen_serial", [(0, 16, 1, 0), (1, 16, 2, 1), (0, 8, 2, 0), (1, 8, 1, 1)])
def test_batch_equals_individual_runs(mode, order, rows, gen_ctas, gen_serial):
    kw = MODES[mode]
    cases = fixtures.batch_instances(3, seed=5, **SMALL, **kw)
    model = _model(cases) if mode == "mixed_learned" else None
    single = _solvers(cases, model)
    batched = _solvers(cases, model)
    b = axj.AxjBatch(batched)
    b.set_tuning(tile_order=order, stage_ctas_per_sm=(1 + order) * (16 // rows), stage_rows=rows,
                 general_ctas_per_sm=gen_ctas, general_serial=gen_serial)
    steps = 7
    b.run(steps)
    for s in single:
        s.run(steps)
    tol = 1e-12 if mode == "fp64" else 1e-6
    for k, (s, t) in enumerate(zip(single, batched)):
        a, r = t.get_state(), s.get_state()
        errs = [np.abs(a[f] - r[f]).max() / max(np.abs(r[f]).max(), 1e-300) for f in range(5)]
        assert max(errs) <= tol, (k, errs)
        assert t.get_time()[0] == s.get_time()[0]
        assert abs(t.get_time()[1] - s.get_time()[1]) <= 1e-12 * abs(s.get_time()[1])
    b.close()
    for s in single + batched:
        s.close()


@pytest.mark.gpu
def test_autotune_undoes_its_trials():
    cases = fixtures.batch_instances(4, seed=9, **SMALL, precision=1, sensor=1)
    model = _model(cases)
    batched = _solvers(cases, model)
    ref = _solvers(cases, model)
    b = axj.AxjBatch(batched)
    chosen, trials = b.autotune(steps_per_trial=2)
    assert len(trials) == 19 and all(t > 0 for t in trials)
    assert b.tuning() == chosen
    b.run(3)
    for s in ref:
        s.run(3)
    for s, t in zip(ref, batched):
        a, r = t.get_state(), s.get_state()
        errs = [np.abs(a[f] - r[f]).max() / max(np.abs(r[f]).max(), 1e-300) for f in range(5)]
        assert max(errs) <= 1e-6, errs
    b.close()
    for s in ref + batched:
        s.close()


@pytest.mark.gpu
def test_batch_rejects_mixed_kinds():
    c1 = fixtures.batch_instances(1, seed=1, **SMALL)[0]
    c2 = fixtures.batch_instances(1, seed=2, **SMALL, precision=1)[0]
    s = _solvers([c1, c2])
    with pytest.raises(axj.AxjError):
        axj.AxjBatch(s)
    for x in s:
        x.close()


@pytest.mark.gpu
def test_batch_with_many_tiles_per_cta():
    """Large instances and one persistent CTA per SM: every CTA loops over many tiles, so
    its TMA barriers complete many phases (a batch of small test instances gives each CTA
    about one tile). Three steps must finish and reproduce the individual runs."""
    cases = fixtures.batch_instances(3, seed=2024, nz_range=(1024, 2048), nr_range=(256, 384))
    single = _solvers(cases)
    batched = _solvers(cases)
    b = axj.AxjBatch(batched)
    b.set_tuning(tile_order=0, stage_ctas_per_sm=1, sensor_ctas_per_sm=1)
    b.run(3)
    for s in single:
        s.run(3)
    for k, (s, t) in enumerate(zip(single, batched)):
        a, r = t.get_state(), s.get_state()
        errs = [np.abs(a[f] - r[f]).max() / max(np.abs(r[f]).max(), 1e-300) for f in range(5)]
        assert max(errs) <= 1e-12, (k, errs)
    b.close()
    for s in single + batched:
        s.close()


@pytest.mark.gpu
@pytest.mark.parametrize("sensor", [0, 1, 2])
def test_batch_accuracy_gate_500_steps(sensor):
    """The batched mixed-precision form with the plain sensor on every stage (0), the learned
    sensor (1, the committed model) or the held schedule without the network (2), the last
    two judged by the plain sensor on the first stage of every second step: 8 uneven
    instances, 500 steps, rho and p within 1e-5 relative L2 of each instance's own plain FP64
    run (the gate the batched form is held to). The speed-up over the same instances run one
    after another on the plain FP64 path is printed. (On the 64-instance batch the two judged
    forms exceed the gate in the instances whose shocks move; the plain form stays far below.)"""
    from axisymmetricjet_b200 import batch_eval
    rep = batch_eval.evaluate(n=8, steps=500, seed=2024, forms=[dict(precision=1, sensor=sensor, judge_every=2,
                                                                     judge_stages=1)], log=lambda m: None)
    err = rep["rel_l2_vs_fp64"]
    print("batched gate:", {"sensor": sensor, "speedup": rep["speedup"], "rel_l2": err, "tuning": rep["tuning"]})
    assert err["rho_max"] < 1e-5 and err["p_max"] < 1e-5, err
    assert rep["speedup"] > 1.0, rep
