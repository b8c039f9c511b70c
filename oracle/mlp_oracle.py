"""TEST INFRASTRUCTURE -- not part of the product.

FP64 numpy restatement of the warm-start MLP (fully connected layers, exact
GELU between them, mean-squared-error loss) used by tests/ as the checker of
the GPU's BF16 forward and backward kernels.  Parameters are a flat FP32
vector in the library's order: W0[out][in], b0, W1, b1, ...
"""
import numpy as np
from scipy.special import erf


def bf16(x):
    """Round to bfloat16 (nearest even) and back, as the GPU GEMM operands."""
    a = np.ascontiguousarray(x, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(params, dims):
    out, o = [], 0
    for i in range(len(dims) - 1):
        nw = dims[i] * dims[i + 1]
        w = params[o:o + nw].reshape(dims[i + 1], dims[i]).astype(np.float64)
        o += nw
        b = params[o:o + dims[i + 1]].astype(np.float64)
        o += dims[i + 1]
        out.append((w, b))
    return out


def gelu(z):
    return 0.5 * z * (1.0 + erf(z / np.sqrt(2.0)))


def gelu_d(z):
    return 0.5 * (1.0 + erf(z / np.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / np.sqrt(2.0 * np.pi)


def forward(params, dims, x, round_bf16=True):
    """Returns (output, [(input_l, z_l)]) ; GEMM operands rounded to bf16 like
    the GPU when round_bf16."""
    r = bf16 if round_bf16 else (lambda v: np.asarray(v, dtype=np.float64))
    layers = unpack(params, dims)
    a = r(x)
    cache = []
    for i, (w, b) in enumerate(layers):
        z = a @ r(w).T + b
        cache.append((a, z))
        a = r(gelu(z)) if i + 1 < len(layers) else z
    return a, cache


def loss_and_grad(params, dims, x, t, round_bf16=True):
    """MSE loss and its gradient (flat, library order)."""
    r = bf16 if round_bf16 else (lambda v: np.asarray(v, dtype=np.float64))
    layers = unpack(params, dims)
    y, cache = forward(params, dims, x, round_bf16)
    n = y.size
    loss = float(np.sum((y - t) ** 2) / n)
    dz = 2.0 * (y - t) / n
    grads = [None] * len(layers)
    for i in range(len(layers) - 1, -1, -1):
        a, _ = cache[i]
        w, _ = layers[i]
        grads[i] = (dz.T @ a, dz.sum(axis=0))
        if i > 0:
            dz = (dz @ r(w)) * gelu_d(cache[i - 1][1])
    flat = np.concatenate([np.concatenate([gw.ravel(), gb]) for gw, gb in grads])
    return loss, flat
