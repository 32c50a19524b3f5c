"""NumPy restatement of the learned sensor (TEST INFRASTRUCTURE ONLY).

This is the checker for the device kernels of the learned artificial-diffusivity
sensor: the feature channels, the BF16 tensor-core inference, the judge, the batch
sampler, and the FP32 training step (forward, backward, Adam). It has no counterpart
in the reference; the sensor it learns is the reference's ModShockCapturing.f90:18-92,
whose CPU restatement is the C oracle (oracle.py), used here for the derivatives and
the plain-sensor targets. Only tests/ import this module.

Layouts follow include/axj.h: a model is a dict of float32 arrays w1 (64, 100), b1,
w2 (64, 64), b2, w3 (2, 64), b3, feat_mean (4), feat_scale (4), out_scale (2); input
index ch*25 + (dr+2)*5 + (dz+2); GELU in its tanh form.
"""
import numpy as np

C_GELU = np.sqrt(2.0 / np.pi)
U64 = np.uint64
MASK64 = (1 << 64) - 1


def gelu(x):
    return 0.5 * x * (1.0 + np.tanh(C_GELU * (x + 0.044715 * x ** 3)))


def gelu_grad(x):
    t = np.tanh(C_GELU * (x + 0.044715 * x ** 3))
    return 0.5 * (1.0 + t) + 0.5 * x * (1.0 - t * t) * C_GELU * (1.0 + 3.0 * 0.044715 * x * x)


def deltas(z, r):
    """deltaz(i), deltar(j) of ModShockCapturing.f90:171-189 (central half-differences,
    one-sided at the ends)."""
    z = np.asarray(z, dtype=np.float64)
    r = np.asarray(r, dtype=np.float64)
    dz = np.empty_like(z)
    dr = np.empty_like(r)
    dz[1:-1] = (z[2:] - z[:-2]) / 2.0
    dz[0] = z[1] - z[0]
    dz[-1] = z[-1] - z[-2]
    dr[1:-1] = (r[2:] - r[:-2]) / 2.0
    dr[0] = r[1] - r[0]
    dr[-1] = r[-1] - r[-2]
    return dz, dr


def ramp(z):
    """z ramp of the artificial coefficients, ModShockCapturing.f90:85."""
    return (1.0 + np.tanh(5.0 * (np.asarray(z, dtype=np.float64) - 10.0))) / 2.0


def features(ora, pv, z, r):
    """Feature channels (4, Nr, Nz): dilatation (as ModShockCapturing.f90:117-121),
    |grad rho|, |dVr/dz - dVz/dr| and sqrt(deltaz*deltar). Derivatives are the C
    oracle's Compute1stDerivative (SBP rows from the patches, zero at blanked points)."""
    rho, Vr, Vz = pv[0], pv[1], pv[3]
    dVrdz, dVzdz, drdz = ora.deriv1(Vr, 1), ora.deriv1(Vz, 1), ora.deriv1(rho, 1)
    dVrdr, dVzdr, drdr = ora.deriv1(Vr, 2), ora.deriv1(Vz, 2), ora.deriv1(rho, 2)
    rr = np.asarray(r, dtype=np.float64)[:, None]
    with np.errstate(divide="ignore", invalid="ignore"):
        dil = dVrdr + Vr / rr + dVzdz
    dil[0] = 2.0 * dVrdr[0] + dVzdz[0]
    grad = np.sqrt(drdz ** 2 + drdr ** 2)
    vort = np.abs(dVrdz - dVzdr)
    dz, dr = deltas(z, r)
    h = np.sqrt(dz[None, :] * dr[:, None]) * np.ones_like(dil)
    return np.stack([dil, grad, vort, h])


def normalise(model, feat):
    m = np.asarray(model["feat_mean"], dtype=np.float64)[:, None, None]
    s = np.asarray(model["feat_scale"], dtype=np.float64)[:, None, None]
    return (feat - m) / s


def window_inputs(xn, i, j, fill):
    """Inputs (n, 100) of the points (i, j) from normalised channels xn (4, Nr, Nz);
    outside the grid a channel takes fill[ch] (the normalised value of 0)."""
    _, Nr, Nz = xn.shape
    i = np.asarray(i)
    j = np.asarray(j)
    out = np.empty((i.size, 100), dtype=np.float64)
    for ch in range(4):
        for dr in range(-2, 3):
            for dz in range(-2, 3):
                k = ch * 25 + (dr + 2) * 5 + (dz + 2)
                ii, jj = i + dz, j + dr
                ok = (ii >= 0) & (ii < Nz) & (jj >= 0) & (jj < Nr)
                v = np.full(i.size, fill[ch], dtype=np.float64)
                v[ok] = xn[ch, jj[ok], ii[ok]]
                out[:, k] = v
    return out


def all_inputs(model, feat):
    """Inputs (Nr*Nz, 100) of every point, row-major over (j, i)."""
    _, Nr, Nz = feat.shape
    xn = normalise(model, feat)
    fill = -np.asarray(model["feat_mean"], np.float64) / np.asarray(model["feat_scale"], np.float64)
    jj, ii = np.meshgrid(np.arange(Nr), np.arange(Nz), indexing="ij")
    return window_inputs(xn, ii.ravel(), jj.ravel(), fill)


def forward(model, X):
    """FP64 forward pass: (cache, Y) with Y (n, 2) the normalised outputs."""
    W1, b1 = model["w1"].astype(np.float64), model["b1"].astype(np.float64)
    W2, b2 = model["w2"].astype(np.float64), model["b2"].astype(np.float64)
    W3, b3 = model["w3"].astype(np.float64), model["b3"].astype(np.float64)
    X = np.asarray(X, dtype=np.float64)
    Z1 = X @ W1.T + b1
    H1 = gelu(Z1)
    Z2 = H1 @ W2.T + b2
    H2 = gelu(Z2)
    Y = H2 @ W3.T + b3
    return (X, Z1, H1, Z2, H2), Y


def loss_and_grad(model, X, T):
    """L = sum over the batch and both outputs of (Y - T)^2 / B, and dL/dparams."""
    (X, Z1, H1, Z2, H2), Y = forward(model, X)
    B = X.shape[0]
    D = Y - np.asarray(T, dtype=np.float64)
    L = float((D * D).sum() / B)
    dY = 2.0 * D / B
    g = {"w3": dY.T @ H2, "b3": dY.sum(0)}
    dZ2 = (dY @ model["w3"].astype(np.float64)) * gelu_grad(Z2)
    g["w2"], g["b2"] = dZ2.T @ H1, dZ2.sum(0)
    dZ1 = (dZ2 @ model["w2"].astype(np.float64)) * gelu_grad(Z1)
    g["w1"], g["b1"] = dZ1.T @ X, dZ1.sum(0)
    return L, g


def adam_step(model, grad, state, t, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam step (bias-corrected, t = 1 for the first step) on the weight fields."""
    out = dict(model)
    for k in ("w1", "b1", "w2", "b2", "w3", "b3"):
        m = b1 * state.setdefault("m_" + k, np.zeros_like(grad[k])) + (1 - b1) * grad[k]
        v = b2 * state.setdefault("v_" + k, np.zeros_like(grad[k])) + (1 - b2) * grad[k] ** 2
        state["m_" + k], state["v_" + k] = m, v
        mhat = m / (1 - b1 ** t)
        vhat = v / (1 - b2 ** t)
        out[k] = model[k].astype(np.float64) - lr * mhat / (np.sqrt(vhat) + eps)
    return out


def bf16(x):
    """Round float32 values to bfloat16 (nearest, ties to even), returned as float64."""
    a = np.ascontiguousarray(np.asarray(x, dtype=np.float32))
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def predict_bf16(model, feat, z):
    """Inference as the tensor-core kernel does it: BF16 inputs and weights of both
    hidden layers, FP32-or-better accumulation, BF16 first hidden activations, layer 3
    in full precision; (betastar, kappastar) = output * out_scale * ramp(z)."""
    _, Nr, Nz = feat.shape
    X = bf16(all_inputs(model, feat).astype(np.float32))
    Z1 = X @ bf16(model["w1"]).T + model["b1"].astype(np.float64)
    H1 = bf16(gelu(Z1).astype(np.float32))
    Z2 = H1 @ bf16(model["w2"]).T + model["b2"].astype(np.float64)
    H2 = gelu(Z2)
    Y = H2 @ model["w3"].astype(np.float64).T + model["b3"].astype(np.float64)
    Y = Y * np.asarray(model["out_scale"], dtype=np.float64)
    rz = ramp(z)[None, :]
    return Y[:, 0].reshape(Nr, Nz) * rz, Y[:, 1].reshape(Nr, Nz) * rz


def judge(pred, plain, thr):
    """Fallback mask (bit k for output k) where |pred - plain| > thr * max |plain| over
    the 5 x 5 window (inside the grid)."""
    Nr, Nz = plain[0].shape
    mask = np.zeros((Nr, Nz), dtype=np.uint8)
    for k in range(2):
        a = np.abs(plain[k])
        pad = np.zeros((Nr + 4, Nz + 4))
        pad[2:-2, 2:-2] = a
        lm = np.zeros_like(a)
        for dr in range(5):
            for dz in range(5):
                lm = np.maximum(lm, pad[dr:dr + Nr, dz:dz + Nz])
        mask |= ((np.abs(pred[k] - plain[k]) > thr * lm).astype(np.uint8) << k)
    return mask


def mix64(z):
    z = (int(z) + 0x9E3779B97F4A7C15) & MASK64
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & MASK64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & MASK64
    return z ^ (z >> 31)


def sample_indices(seed, step, B, S, Nz, Nr):
    """(snapshot, i, j) of the B points training step `step` draws."""
    base = mix64((seed + step * 0x9E3779B97F4A7C15) & MASK64)
    out = np.empty((B, 3), dtype=np.int64)
    npts = Nz * Nr
    for b in range(B):
        u = mix64((base + b) & MASK64)
        p = (u >> 32) % npts
        out[b] = (u % S, p % Nz, p // Nz)
    return out
