"""NumPy restatement of the learned troubled-cell predictor (test infrastructure only).

The predictor has no counterpart in the reference (jpalafou/FVHOE flags
troubled cells only with the a-posteriori check, `fvhoe/solver.py:653-732`);
this module is the CPU definition the CUDA kernels are checked against:

* features of a cell: for each of (rho, v_X, v_Y, P) and each offset (a, b)
  in [-2, 2]^2, d = w(x+a, y+b) - w(x, y) and
  f = sign(d) log1p(|d| / (eps R)) / log1p(1 / eps), eps = 1e-5, with R the
  variable's range over the stage's 3-ghost box (the global NAD extrema of
  `fvhoe/slope_limiting.py:118-140`);
* network 100 -> 64 -> 64 -> 1 with GELU in its tanh form, parameters packed as
  W1[64][100], b1, W2[64][64], b2, w3[64], b3 (FP32);
* loss: binary cross-entropy with logits, positives weighted by pos_weight,
  averaged over the batch.

`gradients(..., bf16=True)` rounds the tensor-core operands (features,
weights, hidden activations and the backpropagated dz) to BF16 where the
CUDA kernels do, so the comparison isolates accumulation order; with
`bf16=False` it is the exact FP64 gradient, checked by finite differences.
"""

import math

import numpy as np

N_IN = 100
N_ROW = 112
N_HID = 64
EPS = 1e-5

W1 = 0
B1 = W1 + N_HID * N_IN
W2 = B1 + N_HID
B2 = W2 + N_HID * N_HID
W3 = B2 + N_HID
B3 = W3 + N_HID
N_PARAMS = B3 + 1

__all__ = ["N_PARAMS", "N_IN", "N_ROW", "bf16", "bf16_bits", "from_bf16_bits", "unpack", "features", "forward",
           "loss", "gradients"]


def bf16(x):
    """Round to the nearest BF16 value (ties to even), returned as float32."""
    return from_bf16_bits(bf16_bits(x))


def bf16_bits(x):
    a = np.ascontiguousarray(np.asarray(x, dtype=np.float32))
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16).astype(np.uint16)
    return r


def from_bf16_bits(b):
    b = np.asarray(b, dtype=np.uint16)
    return (b.astype(np.uint32) << 16).view(np.float32)


def unpack(p):
    p = np.asarray(p)
    return (p[W1:B1].reshape(N_HID, N_IN), p[B1:W2], p[W2:B2].reshape(N_HID, N_HID), p[B2:W3], p[W3:B3],
            p[B3])


def features(w, vid, ranges, ghosts):
    """Feature rows (nx*ny, 100) of a 2D primitive array w (nvars, nx+2g, ny+2g), g >= 2."""
    g = ghosts
    nx, ny = w.shape[1] - 2 * g, w.shape[2] - 2 * g
    norm = 1.0 / math.log1p(1.0 / EPS)
    out = np.empty((nx, ny, N_IN), dtype=np.float64)
    for v, var in enumerate(vid):
        r = ranges[v] if ranges[v] > 0 else 1.0
        inv_s = 1.0 / (EPS * r)
        c = w[var, g:g + nx, g:g + ny]
        for a in range(-2, 3):
            for b in range(-2, 3):
                d = w[var, g + a:g + a + nx, g + b:g + b + ny] - c
                out[:, :, v * 25 + (a + 2) * 5 + (b + 2)] = np.sign(d) * np.log1p(np.abs(d) * inv_s) * norm
    return out.reshape(nx * ny, N_IN)


_C = math.sqrt(2.0 / math.pi)
_A = 0.044715


def _gelu(x):
    """GELU, tanh form (Hendrycks & Gimpel 2016)."""
    return 0.5 * x * (1.0 + np.tanh(_C * (x + _A * x ** 3)))


def _gelu_grad(x):
    t = np.tanh(_C * (x + _A * x ** 3))
    return 0.5 * (1.0 + t) + 0.5 * x * (1.0 - t * t) * _C * (1.0 + 3.0 * _A * x * x)


def _round(x, on):
    return bf16(x).astype(np.float64) if on else x


def _forward(p, X, rb):
    w1, b1, w2, b2, w3, b3 = (np.asarray(t, dtype=np.float64) for t in unpack(p))
    X = _round(np.asarray(X, dtype=np.float64)[:, :N_IN], rb)
    z1 = X @ _round(w1, rb).T + b1
    a1 = _round(_gelu(z1), rb)
    z2 = a1 @ _round(w2, rb).T + b2
    a2 = _gelu(z2)
    return X, z1, a1, z2, a2, a2 @ w3 + b3


def forward(p, X, bf16_operands=True):
    """Logits of the rows of X (n, >= 100)."""
    return _forward(p, X, bf16_operands)[-1]


def loss(p, X, y, pos_weight, bf16_operands=False):
    x = forward(p, X, bf16_operands)
    y = np.asarray(y, dtype=np.float64)
    sp = np.log1p(np.exp(-np.abs(x))) + np.maximum(-x, 0.0)  # softplus(-x)
    return float(np.mean((1.0 - y) * x + (1.0 + (pos_weight - 1.0) * y) * sp))


def gradients(p, X, y, pos_weight, bf16_operands=True):
    """Gradient of the mean loss with respect to the packed parameters, and the loss."""
    rb = bf16_operands
    w1, b1, w2, b2, w3, b3 = (np.asarray(t, dtype=np.float64) for t in unpack(p))
    X, z1, a1, z2, a2, x = _forward(p, X, rb)
    y = np.asarray(y, dtype=np.float64)
    n = X.shape[0]
    sig = 1.0 / (1.0 + np.exp(-x))
    dlogit = (sig * (pos_weight * y + 1.0 - y) - pos_weight * y) / n
    g = np.zeros(N_PARAMS, dtype=np.float64)
    g[W3:B3] = a2.T @ dlogit
    g[B3] = dlogit.sum()
    dz2 = _round(dlogit[:, None] * w3[None, :] * _gelu_grad(z2), rb)
    g[W2:B2] = (dz2.T @ a1).ravel()
    g[B2:W3] = dz2.sum(axis=0)
    dz1 = _round((dz2 @ _round(w2, rb)) * _gelu_grad(z1), rb)
    g[W1:B1] = (dz1.T @ X).ravel()
    g[B1:W2] = dz1.sum(axis=0)
    sp = np.log1p(np.exp(-np.abs(x))) + np.maximum(-x, 0.0)
    return g, float(np.mean((1.0 - y) * x + (1.0 + (pos_weight - 1.0) * y) * sp))
