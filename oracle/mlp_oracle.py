"""CPU oracle of the warm-start MLP (test infrastructure only: imported by tests/
and never by the library).

The network of filsim_b200's fs_mlp.cu: x -> 3 x [Linear + SiLU] -> Linear, mean
square loss over the valid rows and targets. With bf16=True the oracle rounds
at the points where the GPU kernels hold BF16 values (round to nearest even):
the normalised inputs, the weights used by the GEMMs, the hidden activations,
the output gradient and the hidden-layer gradients; sums are taken in float64.
With bf16=False everything is float64, for checking the backward pass against
finite differences.
"""
import numpy as np


def bf16(x):
    """Round float32 values to the nearest BF16 (ties to even), returned as float32."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32)
    r = ((u >> 16) & 1) + np.uint32(0x7FFF)
    return ((u + r) & np.uint32(0xFFFF0000)).astype(np.uint32).view(np.float32)


def unflatten(flat, dims):
    """[W1 b1 W2 b2 W3 b3 W4 b4] -> [(W, b)], W row-major [out x in]."""
    out, o = [], 0
    for l in range(4):
        n_out, n_in = dims[l + 1], dims[l]
        W = flat[o:o + n_out * n_in].reshape(n_out, n_in)
        o += n_out * n_in
        b = flat[o:o + n_out]
        o += n_out
        out.append((W, b))
    return out


def flatten(grads):
    return np.concatenate([np.concatenate([gW.ravel(), gb.ravel()]) for gW, gb in grads])


def _silu_parts(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return z * s, s * (1.0 + z * (1.0 - s))


def forward(layers, x, use_bf16=True):
    """x: normalised inputs [n x k_in]. Returns (y, cache)."""
    rnd = bf16 if use_bf16 else (lambda a: np.asarray(a, dtype=np.float64))
    h = rnd(x).astype(np.float64)
    cache = {"h": [h], "z": []}
    for l in range(3):
        W, b = layers[l]
        z = h @ rnd(W).astype(np.float64).T + b
        if use_bf16:
            z = z.astype(np.float32).astype(np.float64)
        a, _ = _silu_parts(z)
        h = rnd(a).astype(np.float64)
        cache["z"].append(z)
        cache["h"].append(h)
    W, b = layers[3]
    y = h @ rnd(W).astype(np.float64).T + b
    return y, cache


def loss_and_gradients(layers, x, t, n, ntgt, use_bf16=True):
    """Mean square loss over rows < n and targets < ntgt, and its gradients."""
    rnd = bf16 if use_bf16 else (lambda a: np.asarray(a, dtype=np.float64))
    y, cache = forward(layers, x, use_bf16)
    d = np.zeros_like(y)
    d[:n, :ntgt] = y[:n, :ntgt] - t[:n, :ntgt]
    scale = 1.0 / (n * ntgt)
    loss = float((d ** 2).sum() * scale)
    g = rnd(2.0 * d * scale).astype(np.float64)
    grads = [None] * 4
    for l in (3, 2, 1, 0):
        W, _ = layers[l]
        h_in = cache["h"][l]
        grads[l] = (g.T @ h_in, g.sum(axis=0))
        if l > 0:
            gh = g @ rnd(W).astype(np.float64)
            _, dsilu = _silu_parts(cache["z"][l - 1])
            g = rnd(gh * dsilu).astype(np.float64)
    return loss, grads
