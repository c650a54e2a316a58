"""FP64 numpy reference of the learned ionic step's network -- TEST
INFRASTRUCTURE ONLY (the checker of the GPU trainer and of the tensor-core
inference kernel; the product never imports it).

Network: dims[0] -> dims[1] -> ... -> dims[L], tanh on hidden layers, linear
output; parameters flattened as W1 (dims[1] x dims[0], row-major), b1, W2,
b2, ...  Loss: mean over rows of sum_j w_j (f(x)_j - y_j)^2.
"""
import numpy as np


def unflatten(p, dims):
    out, off = [], 0
    for l in range(len(dims) - 1):
        nw = dims[l + 1] * dims[l]
        W = p[off:off + nw].reshape(dims[l + 1], dims[l]); off += nw
        b = p[off:off + dims[l + 1]]; off += dims[l + 1]
        out.append((W.astype(np.float64), b.astype(np.float64)))
    return out


def forward(p, dims, X, bf16=False):
    """Outputs (and hidden activations).  bf16=True emulates the deployed
    kernel: BF16 weights and BF16 activations between layers, FP32-exact
    accumulation of the products."""
    layers = unflatten(p, dims)
    h = np.asarray(X, dtype=np.float64)
    acts = [h]
    for l, (W, b) in enumerate(layers):
        if bf16:
            W = to_bf16(W)
            h = to_bf16(h)
        z = h @ W.T + b
        h = np.tanh(z) if l < len(layers) - 1 else z
        acts.append(h)
    return h, acts


def loss_grad(p, dims, X, Y, w=None):
    layers = unflatten(p, dims)
    B = X.shape[0]
    out, acts = forward(p, dims, X)
    w = np.ones(out.shape[1]) if w is None else np.asarray(w, dtype=np.float64)
    d = out - Y
    loss = float(np.sum(w * d * d) / B)
    delta = 2.0 * w * d / B
    grads = []
    for l in range(len(layers) - 1, -1, -1):
        W, _ = layers[l]
        hprev = acts[l]
        gW = delta.T @ hprev
        gb = delta.sum(axis=0)
        grads.append((gW, gb))
        if l > 0:
            delta = (delta @ W) * (1.0 - hprev * hprev)
    grads.reverse()
    flat = np.concatenate([np.concatenate([gW.ravel(), gb]) for gW, gb in grads])
    return loss, flat


def to_bf16(a):
    """Round to the nearest bfloat16 (ties to even), returned as float64."""
    a = np.asarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = (u + 0x7FFF + ((u >> 16) & 1)) >> 16
    return (r.astype(np.uint32) << 16).view(np.float32).astype(np.float64)
