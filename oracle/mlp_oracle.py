"""FP64 reference of the surrogate MLP (9 -> 256 -> 256 -> 256 -> 1, SiLU) and
of its mean-squared-error gradients, in numpy.

TEST INFRASTRUCTURE ONLY: the checker for the GPU's tcgen05 forward/backward
kernels and for the residual's Black-Scholes base.  The reference library has
no such network; this is the plain mathematics of the architecture the
surrogate specifies.  Parameter order:
W1[256][9], b1, W2[256][256], b2, W3[256][256], b3, w4[256], b4.
"""

import math

import numpy as np

HID, IN = 256, 9
SHAPES = [("W1", (HID, IN)), ("b1", (HID,)), ("W2", (HID, HID)), ("b2", (HID,)),
          ("W3", (HID, HID)), ("b3", (HID,)), ("w4", (HID,)), ("b4", (1,))]
N_PARAMS = sum(int(np.prod(s)) for _, s in SHAPES)


def unpack(p):
    out, k = {}, 0
    for name, shape in SHAPES:
        n = int(np.prod(shape))
        out[name] = np.asarray(p[k:k + n], np.float64).reshape(shape)
        k += n
    return out


def pack(d):
    return np.concatenate([d[name].reshape(-1) for name, _ in SHAPES])


def _sig(z):
    return 1.0 / (1.0 + np.exp(-z))


def forward(p, x):
    w = unpack(p)
    z1 = x @ w["W1"].T + w["b1"]
    h1 = z1 * _sig(z1)
    z2 = h1 @ w["W2"].T + w["b2"]
    h2 = z2 * _sig(z2)
    z3 = h2 @ w["W3"].T + w["b3"]
    h3 = z3 * _sig(z3)
    y = h3 @ w["w4"] + w["b4"][0]
    return y, (z1, h1, z2, h2, z3, h3)


def bf16_round(x):
    """Round to the nearest bf16 value (ties to even), returned as float64."""
    f = np.asarray(x, np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def forward_bf16(p, x):
    """The network as the GPU evaluates it, in FP64 otherwise: weights of the
    three hidden layers rounded to bf16, the activations of layers 1 and 2
    rounded to bf16 after the SiLU (they are the next GEMM's bf16 operand),
    layer 3's activations and the head (w4, b4) in full precision; exact SiLU
    and FP64 sums (the GPU sums in FP32 and takes tanh from the
    special-function unit, so it may round an activation to the neighbouring
    bf16 value)."""
    w = unpack(p)
    h = np.asarray(x, np.float64)
    for name in ("1", "2", "3"):
        z = h @ bf16_round(w["W" + name]).T + w["b" + name]
        h = z * _sig(z)
        if name != "3":
            h = bf16_round(h)
    return h @ w["w4"] + w["b4"][0]


def loss_and_grads(p, x, t):
    """Mean squared error over the batch and its gradient (parameter order)."""
    w = unpack(p)
    y, (z1, h1, z2, h2, z3, h3) = forward(p, x)
    n = x.shape[0]
    loss = float(np.mean((y - t) ** 2))
    dy = 2.0 * (y - t) / n

    def dsilu(z):
        s = _sig(z)
        return s * (1.0 + z * (1.0 - s))

    g = {"w4": h3.T @ dy, "b4": np.array([dy.sum()])}
    dz3 = np.outer(dy, w["w4"]) * dsilu(z3)
    g["W3"], g["b3"] = dz3.T @ h2, dz3.sum(0)
    dz2 = (dz3 @ w["W3"]) * dsilu(z2)
    g["W2"], g["b2"] = dz2.T @ h1, dz2.sum(0)
    dz1 = (dz2 @ w["W2"]) * dsilu(z1)
    g["W1"], g["b1"] = dz1.T @ x, dz1.sum(0)
    return loss, pack(g)


def bsm_mean_var_base(f):
    """The residual's base for feature rows f (n x 9: S/K, T, r, q, v0, kappa,
    theta, sigma, rho): the Black-Scholes call / S at the Heston mean variance
    over [0, T], theta + (v0 - theta)(1 - exp(-kappa T))/(kappa T), in FP64."""
    f = np.asarray(f, np.float64)
    out = np.empty(f.shape[0])
    for i, (m, T, r, q, v0, kappa, theta) in enumerate(f[:, :7]):
        x = kappa * T
        w = -math.expm1(-x) / x if x > 1e-12 else 1.0
        vbar = max(theta + (v0 - theta) * w, 0.0)
        sd = math.sqrt(vbar * T)
        dq, dk = math.exp(-q * T), math.exp(-r * T) / m
        if not sd > 1e-12:
            out[i] = max(dq - dk, 0.0)
            continue
        d1 = (math.log(m) + (r - q) * T) / sd + 0.5 * sd
        out[i] = dq * 0.5 * math.erfc(-d1 / math.sqrt(2.0)) - dk * 0.5 * math.erfc(-(d1 - sd) / math.sqrt(2.0))
    return out


def bf16_bits_to_float(bits):
    """bf16 bit patterns (uint16) to float64."""
    return (np.asarray(bits, np.uint16).astype(np.uint32) << 16).view(np.float32).astype(np.float64)
