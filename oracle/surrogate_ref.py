"""CPU reference of the surrogate MLP (test infrastructure: only tests use it).

Restates webgpu-dna_b200/csrc/surrogate.cu in numpy: a 64 -> 128 -> 128 ->
128 -> 80 network with exact-erf GELU, bf16 weights and bf16 layer inputs
(round to nearest even, as the tensor-core operands), products summed in
float64 here (f32 on the GPU), mean-squared-error loss over the batch and the
80 outputs.  ``exact=True`` drops every bf16 rounding, for finite-difference
checks of the gradient formulas.
"""
import math

import numpy as np

IN, HID, OUT = 64, 128, 80
SHAPES = [(HID, IN), (HID, HID), (HID, HID), (OUT, HID)]


def offsets():
    off, o = [], 0
    for (n_out, n_in) in SHAPES:
        off.append((o, o + n_out * n_in))
        o += n_out * n_in + n_out
    return off, o


OFFS, NPARAM = offsets()


def bf16(x):
    """Round float32 values to bfloat16 (nearest even), returned as float32."""
    a = np.ascontiguousarray(x, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).reshape(a.shape)


_erf = np.vectorize(math.erf)


def gelu(z):
    return 0.5 * z * (1.0 + _erf(z / math.sqrt(2.0)))


def gelu_d(z):
    return 0.5 * (1.0 + _erf(z / math.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / math.sqrt(2.0 * math.pi)


def unpack(p):
    Ws, bs = [], []
    for (n_out, n_in), (w0, b0) in zip(SHAPES, OFFS):
        Ws.append(np.asarray(p[w0:w0 + n_out * n_in], np.float64).reshape(n_out, n_in))
        bs.append(np.asarray(p[b0:b0 + n_out], np.float64))
    return Ws, bs


def forward(p, X, exact=False):
    """X: standardised inputs (n x 64).  Returns Y and the saved layer state."""
    rnd = (lambda a: np.asarray(a, np.float64)) if exact else (lambda a: bf16(a).astype(np.float64))
    Ws, bs = unpack(p)
    Wq = [rnd(W.astype(np.float32)) if not exact else W for W in Ws]
    H = [rnd(np.asarray(X, np.float32))]
    Z = []
    for l in range(4):
        z = H[-1] @ Wq[l].T + bs[l]
        if l < 3:
            z = z.astype(np.float32).astype(np.float64) if not exact else z
            Z.append(z)
            H.append(rnd(gelu(z).astype(np.float32)) if not exact else gelu(z))
        else:
            Y = z
    return Y, {"H": H, "Z": Z, "W": Wq}


def loss_and_grad(p, X, T, exact=False):
    """Mean squared error and its gradient with respect to the parameters."""
    n = X.shape[0]
    Y, s = forward(p, X, exact)
    diff = Y - np.asarray(T, np.float64)
    loss = float((diff ** 2).sum() / (n * OUT))
    D = 2.0 * diff / (n * OUT)
    g = np.zeros(NPARAM)
    rnd = (lambda a: a) if exact else (lambda a: bf16(a.astype(np.float32)).astype(np.float64))
    for l in range(3, -1, -1):
        (w0, b0), (n_out, n_in) = OFFS[l], SHAPES[l]
        Dq = rnd(D)
        g[w0:w0 + n_out * n_in] = (Dq.T @ s["H"][l]).reshape(-1)
        g[b0:b0 + n_out] = D.sum(axis=0)
        if l > 0:
            dH = Dq @ s["W"][l]
            D = dH * gelu_d(s["Z"][l - 1])
    return loss, g


def init(seed):
    """Glorot-uniform weights, zero biases (the same distribution as the device init)."""
    rng = np.random.default_rng(seed)
    p = np.zeros(NPARAM, np.float32)
    for (n_out, n_in), (w0, _) in zip(SHAPES, OFFS):
        a = math.sqrt(6.0 / (n_in + n_out))
        p[w0:w0 + n_out * n_in] = rng.uniform(-a, a, n_out * n_in)
    return p
