"""Learned artificial-diffusivity sensor: features, tensor-core inference, training
kernels and the judge, against the NumPy oracle (oracle/oracle_mlp.py) and the C oracle.

Tolerances (written per test):
  features        1e-4 of each channel's max (FP32 inputs and stencils vs the FP64 oracle)
  gradients       1e-4 of each tensor's max (FP32 GEMMs with atomics vs FP64)
  Adam step       1e-5 of each tensor's max (same gradient, FP32 vs FP64 update)
  sampler         exact indices; features 1e-6, targets 1e-5 relative
  inference       BF16 operands on both sides; 2e-3 of the prediction's max
"""
import numpy as np
import pytest

import axisymmetricjet_b200 as axj
from axisymmetricjet_b200 import fixtures

import oracle_mlp as om


def _solver(c):
    patches = axj.patches_from_records(c["records"], c["Nz"], c["Nr"])
    s = axj.AxiJetSolver(c["params"], c["zvec"], c["rvec"], c["ibval"], patches)
    s.set_state(c["pv"], c["target"])
    return s, patches


def _oracle(oracle_mod, c):
    op = oracle_mod.patches_from_records(c["records"], c["Nz"], c["Nr"])
    o = oracle_mod.Oracle(c["params"], c["zvec"], c["rvec"], c["ibval"], op)
    o.set_state(c["pv"], c["target"])
    return o


def _rand_model(seed, feat=None):
    m = axj.mlp_init(seed)
    if feat is not None:  # a normalisation that makes the inputs O(1)
        m["feat_mean"] = feat.reshape(4, -1).mean(1).astype(np.float32)
        m["feat_scale"] = (feat.reshape(4, -1).std(1) + 1e-6).astype(np.float32)
    m["out_scale"] = np.array([0.5, 2.0], dtype=np.float32)
    return m


def _relmax(a, b):
    s = np.abs(b).max()
    return float(np.abs(np.asarray(a, np.float64) - b).max() / (s if s > 0 else 1.0))


# ---------------------------------------------------------------- CPU (oracle pins)
def test_oracle_backward_matches_finite_differences():
    rng = np.random.default_rng(3)
    model = {"w1": rng.standard_normal((64, 100)) * 0.1, "b1": rng.standard_normal(64) * 0.1,
             "w2": rng.standard_normal((64, 64)) * 0.1, "b2": rng.standard_normal(64) * 0.1,
             "w3": rng.standard_normal((2, 64)) * 0.1, "b3": rng.standard_normal(2) * 0.1}
    X = rng.standard_normal((7, 100))
    T = rng.standard_normal((7, 2))
    _, g = om.loss_and_grad(model, X, T)
    h = 1e-6
    for k in ("w1", "b2", "w3", "b3"):
        flat = model[k].reshape(-1)
        for idx in rng.choice(flat.size, size=min(5, flat.size), replace=False):
            old = flat[idx]
            flat[idx] = old + h
            lp, _ = om.loss_and_grad(model, X, T)
            flat[idx] = old - h
            lm, _ = om.loss_and_grad(model, X, T)
            flat[idx] = old
            fd = (lp - lm) / (2 * h)
            assert abs(fd - g[k].reshape(-1)[idx]) <= 1e-6 * max(1.0, abs(fd)), (k, idx)


def test_oracle_bf16_rounding():
    x = np.array([1.0, 1.00390625, 1.005859375, -3.14159, 0.0], dtype=np.float32)
    r = om.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0  # tie to even
    assert r[2] == 1.0078125
    assert abs(r[3] + 3.140625) < 1e-12


def test_oracle_sampler_is_deterministic_and_in_range():
    a = om.sample_indices(5, 3, 64, 3, 96, 64)
    b = om.sample_indices(5, 3, 64, 3, 96, 64)
    assert (a == b).all()
    assert a[:, 0].max() < 3 and a[:, 1].max() < 96 and a[:, 2].max() < 64
    assert not (a == om.sample_indices(5, 4, 64, 3, 96, 64)).all()


# ---------------------------------------------------------------- GPU
@pytest.mark.gpu
@pytest.mark.parametrize("name", ["jet96x64sc", "nozzle"])
def test_features_vs_oracle(oracle_mod, name):
    c = fixtures.case(name) if name != "nozzle" else fixtures.nozzle_case(sc=True, Mj=1.5, Re=5000.0)
    dev, _ = _solver(c)
    ora = _oracle(oracle_mod, c)
    # a state with structure: a few steps of the plain solver
    for _ in range(3):
        dev.rk4(dev.compute_time_step())
    pv = dev.get_state()
    got = dev.mlp_features(pv)
    want = om.features(ora, pv, c["z"], c["r"])
    for ch in range(4):
        assert _relmax(got[ch], want[ch]) < 1e-4, ch
    dev.close()


@pytest.mark.gpu
@pytest.mark.parametrize("B", [500, 3000])
def test_gradients_vs_oracle(B):
    c = fixtures.case("jet96x64sc")
    dev, _ = _solver(c)
    model = _rand_model(11)
    dev.mlp_set(model)
    rng = np.random.default_rng(B)
    X = rng.standard_normal((B, 100)).astype(np.float32)
    T = rng.standard_normal((B, 2)).astype(np.float32)
    g, loss = dev.mlp_grad(X, T)
    lo, go = om.loss_and_grad(model, X.astype(np.float64), T.astype(np.float64))
    assert abs(loss - lo) <= 1e-5 * abs(lo)
    for k in ("w1", "b1", "w2", "b2", "w3", "b3"):
        assert _relmax(g[k], go[k]) < 1e-4, k
    dev.close()


def _dataset(dev, nsnap, steps_between):
    dev.dataset_reserve(nsnap)
    states = []
    for _ in range(nsnap):
        for _ in range(steps_between):
            dev.rk4(dev.compute_time_step())
        states.append(dev.get_state())
        dev.dataset_add()
    return states


@pytest.mark.gpu
def test_sampler_vs_oracle(oracle_mod):
    c = fixtures.case("jet96x64sc")
    dev, _ = _solver(c)
    ora = _oracle(oracle_mod, c)
    states = _dataset(dev, 2, 3)
    model = _rand_model(5, dev.mlp_features(states[0]))
    dev.mlp_set(model)
    B, seed, step = 256, 17, 4
    X, T = dev.dataset_sample(B, seed, step)
    idx = om.sample_indices(seed, step, B, 2, c["Nz"], c["Nr"])
    fill = -model["feat_mean"].astype(np.float64) / model["feat_scale"]
    rz = om.ramp(c["z"])
    for s in range(2):
        sel = idx[:, 0] == s
        if not sel.any():
            continue
        feat = om.features(ora, states[s], c["z"], c["r"])
        Xo = om.window_inputs(om.normalise(model, feat), idx[sel, 1], idx[sel, 2], fill)
        assert np.abs(X[sel] - Xo).max() < 1e-3 * max(1.0, np.abs(Xo).max())
        # targets: the plain sensor's betastar, kappastar before the ramp (compared where
        # the ramp is 1 to double precision)
        _, beta, kappa = ora.sensor(states[s])
        ii, jj = idx[sel, 1], idx[sel, 2]
        full = rz[ii] > 1.0 - 1e-12
        for k, ref in enumerate((beta, kappa)):
            want = ref[jj[full], ii[full]] / model["out_scale"][k]
            scale = max(np.abs(ref).max() / model["out_scale"][k], 1e-30)
            assert np.abs(T[sel][full, k] - want).max() <= 1e-5 * scale, k
    dev.close()


@pytest.mark.gpu
def test_adam_step_vs_oracle():
    c = fixtures.case("jet96x64sc")
    dev, _ = _solver(c)
    states = _dataset(dev, 2, 2)
    model = _rand_model(7, dev.mlp_features(states[0]))
    dev.mlp_set(model)
    B, seed = 4096, 23
    X, T = dev.dataset_sample(B, seed, 0)
    dev.mlp_train(steps=1, batch=B, seed=seed, fit_normalization=0)
    got = dev.mlp_get()
    _, g = om.loss_and_grad(model, X.astype(np.float64), T.astype(np.float64))
    want = om.adam_step(model, g, {}, 1)
    for k in ("w1", "b1", "w2", "b2", "w3", "b3"):
        # every weight moves by lr * sign(g) after the first bias-corrected step
        assert _relmax(got[k] - model[k], want[k] - model[k]) < 1e-3, k
    dev.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["jet96x64sc", "jet_ragged"])
def test_tensor_core_inference_vs_oracle(oracle_mod, name):
    c = fixtures.case("jet96x64sc") if name == "jet96x64sc" else fixtures.make_case(77, 45, 30.0, 15.0, 1.5, 5000.0,
                                                                                    sc=True)
    dev, _ = _solver(c)
    for _ in range(3):
        dev.rk4(dev.compute_time_step())
    pv = dev.get_state()
    feat = dev.mlp_features(pv)
    model = _rand_model(9, feat)
    dev.mlp_set(model)
    b, k = dev.mlp_predict(pv)
    bo, ko = om.predict_bf16(model, feat.astype(np.float64), c["z"])
    assert _relmax(b, bo) < 2e-3
    assert _relmax(k, ko) < 2e-3
    dev.close()


@pytest.mark.gpu
def test_judge_vs_oracle_and_learned_steps(oracle_mod):
    """A learned-sensor handle: first step judges (prediction vs plain sensor on the
    stage-1 input), later steps use the prediction with the fallback mask."""
    c = fixtures.case("jet96x64sc", sensor=1, judge_every=5, judge_threshold=0.1)
    dev, _ = _solver(c)
    feat = dev.mlp_features(c["pv"])
    model = _rand_model(13, feat)
    dev.mlp_set(model)
    pv0 = c["pv"]
    dev.rk4(dev.compute_time_step())
    st = dev.learned_stats()
    assert st["judges"] == 1 and st["judged_outputs"] == 2 * c["Nz"] * c["Nr"]
    # the same judge from the oracles
    ora = _oracle(oracle_mod, c)
    _, beta, kappa = ora.sensor(pv0)
    pred = om.predict_bf16(model, om.features(ora, pv0, c["z"], c["r"]), c["z"])
    mask = om.judge(pred, (beta, kappa), 0.1)
    n_fb = int((mask & 1).sum() + ((mask >> 1) & 1).sum())
    # points within rounding of the threshold may go either way
    assert abs(st["fallbacks"] - n_fb) <= 0.01 * 2 * c["Nz"] * c["Nr"], (st, n_fb)
    for _ in range(9):
        dev.rk4(dev.compute_time_step())
    st = dev.learned_stats()
    assert st["judges"] == 2  # iterations 0 and 5
    assert np.isfinite(dev.get_state()).all()
    dev.close()
