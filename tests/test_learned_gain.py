"""What the trained network gains over the method without it, measured on the device.

The committed model (sensor_mlp_jet4400x640.npz) stands in for the artificial-diffusivity
sensor of ComputeArtTransCoeffs (ModShockCapturing.f90:18-92) on the production jet
(4400 x 640, Mach 1.5, Re 5000, shock capturing, mixed precision). Three forms run the
same steps from the same state with the same dt sequence:

  plain    the reference's sensor on every RK stage (the method the network replaces);
  held     the schedule without the network: the plain sensor on judge steps, its
           coefficients held in between (AXJ_SENSOR_HELD);
  learned  the network once per step, the plain sensor as judge every judge_every steps,
           its values kept wherever the prediction disagrees by more than the threshold.

The test asserts the network's gain over the plain sensor: the learned run is cheaper per
step and stays within 1e-5 relative L2 of the plain run in rho and p (the accuracy gate)
after 200 steps: cost at a bounded accuracy loss. Against the held schedule it records,
without asserting a direction, the accuracy and the cost (the network costs time on every
step and is judged on the same schedule), and the fraction of judged outputs that fell
back. The numbers are printed for the record.
"""
import json

import numpy as np
import pytest

import axisymmetricjet_b200 as axj
from axisymmetricjet_b200 import accuracy, fixtures
from axisymmetricjet_b200.train_sensor import load_model

pytestmark = pytest.mark.gpu

STEPS = 200   # four judge periods of 50
GATE = 1e-5   # relative L2 of rho and p against the plain sensor's run


def _run(c, patches, dts, model=None, **pkw):
    prm = axj.AxjParams.from_buffer_copy(c["params"])
    for k, v in pkw.items():
        setattr(prm, k, v)
    s = axj.AxiJetSolver(prm, c["zvec"], c["rvec"], c["ibval"], patches)
    if model is not None:
        s.mlp_set(model)
    s.set_state(c["pv"], c["target"])
    for d in dts:
        s.rk4(d)
    state = s.get_state()
    stats = s.learned_stats() if pkw.get("sensor") == 1 else None
    # cost per step: graph-replayed steps of the same form from the same state
    s.set_state(c["pv"], c["target"])
    s.run(3)
    ms = s.run_timed(STEPS) / STEPS
    s.close()
    return state, ms, stats


def test_learned_sensor_gain_over_plain_and_held():
    c = fixtures.case("jet4400x640", precision=1)
    patches = axj.patches_from_records(c["records"], c["Nz"], c["Nr"])
    # one dt sequence for every form: the plain run's (ComputeTimeStep each step)
    s = axj.AxiJetSolver(c["params"], c["zvec"], c["rvec"], c["ibval"], patches)
    s.set_state(c["pv"], c["target"])
    dts = []
    for _ in range(STEPS):
        d = s.compute_time_step()
        s.rk4(d)
        dts.append(d)
    s.close()
    model = load_model()
    plain, ms_plain, _ = _run(c, patches, dts, sensor=0)
    held, ms_held, _ = _run(c, patches, dts, sensor=2)
    lrn, ms_lrn, st = _run(c, patches, dts, model=model, sensor=1)
    e_held = accuracy.field_errors(held, plain)
    e_lrn = accuracy.field_errors(lrn, plain)
    fallback = st["fallbacks"] / max(st["judged_outputs"], 1)
    rec = {"steps": STEPS, "ms_per_step": {"plain": ms_plain, "held": ms_held, "learned": ms_lrn},
           "rel_l2_vs_plain": {"held": {"rho": e_held["rho"]["rel_l2"], "p": e_held["p"]["rel_l2"]},
                               "learned": {"rho": e_lrn["rho"]["rel_l2"], "p": e_lrn["p"]["rel_l2"]}},
           "learned_fallback_fraction": fallback, "judges": st["judges"]}
    print("learned sensor gain:", json.dumps(rec))
    assert np.isfinite(lrn).all()
    # the gain over the plain sensor: cheaper, within the accuracy gate
    assert ms_lrn < ms_plain, rec
    assert e_lrn["rho"]["rel_l2"] < GATE and e_lrn["p"]["rel_l2"] < GATE, rec
    # the network's predictions are used somewhere (not every output falls back)
    assert fallback < 1.0, rec
