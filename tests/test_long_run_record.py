"""The recorded 1000-step FP64 parity run of the production jet (jet4400x640: 4400 x 640,
Mach 1.5, Re 5000, shock capturing, reference dt) against its calibrated tolerance.

tests/golden/long_run_calibration.json: the oracle against the same C source built with
FMA contraction (tests/long_run_parity.py calibrate), i.e. how far two correct FP64
evaluations of the reference's arithmetic drift apart, per field and checkpoint.
tests/golden/long_run_check_jet4400x640.json: the device path against the oracle on a B200
(tests/long_run_parity.py check), every path computing its own dt. The tolerance per field
and checkpoint is 10 x the calibrated spread, or the FP64 unit roundoff if larger.
No GPU needed: this re-applies the rule to the recorded numbers.
"""
import json
import os

import long_run_parity as lrp

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _load(name):
    with open(os.path.join(GOLDEN, name)) as f:
        return json.load(f)


def test_calibration_covers_1000_steps_of_the_production_jet():
    cal = _load("long_run_calibration.json")
    assert cal["case"] == "jet4400x640" and cal["steps"] == 1000
    steps = [r["step"] for r in cal["checkpoints"]]
    assert steps[0] == 1 and steps[-1] == 1000
    for r in cal["checkpoints"]:
        for k in lrp.FIELDS:
            assert 0.0 <= r["l2"][k] < 1e-14


def test_recorded_device_run_is_within_the_calibrated_tolerance():
    cal = _load("long_run_calibration.json")
    chk = _load("long_run_check_jet4400x640.json")
    assert chk["case"] == "jet4400x640" and chk["steps"] == 1000
    assert chk["compared"] == "device FP64 path vs oracle"
    spread = {r["step"]: r["l2"] for r in cal["checkpoints"]}
    seen = 0
    for r in chk["checkpoints"]:
        tol = {k: max(lrp.TOL_FACTOR * spread[r["step"]][k], lrp.FLOOR) for k in lrp.FIELDS}
        for k in lrp.FIELDS:
            assert r["l2"][k] <= tol[k], (r["step"], k, r["l2"][k], tol[k])
        seen += 1
    assert seen == len(cal["checkpoints"])
    assert chk["pass"] is True
