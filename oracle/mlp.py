"""FP64 reference of the surrogate MLP (TEST INFRASTRUCTURE ONLY).

The network has no counterpart in the reference; this file states its
mathematics -- the checker for the GPU forward and backward kernels
(hackathon_b200/csrc/mlp.cu): 65 -> 256 -> 256 -> 256 -> 256 -> 5,
h = GELU(W x + b) with GELU(z) = z Phi(z) (the erf form), a linear output
layer, and the loss mean((o - y)^2) over the batch and the 5 outputs.
Parameters use the library's flat layout: per layer W [out][in] row-major,
then b [out].
"""
import numpy as np
from scipy.special import erf

DIMS = [(65, 256), (256, 256), (256, 256), (256, 256), (256, 5)]


def unflatten(flat):
    out, off = [], 0
    for i, o in DIMS:
        W = flat[off:off + o * i].reshape(o, i)
        off += o * i
        b = flat[off:off + o]
        off += o
        out.append((W.astype(np.float64), b.astype(np.float64)))
    assert off == flat.size
    return out


def flatten(layers):
    return np.concatenate([np.concatenate([W.ravel(), b]) for W, b in layers])


def gelu(z):
    return 0.5 * z * (1 + erf(z / np.sqrt(2)))


def gelu_grad(z):
    return 0.5 * (1 + erf(z / np.sqrt(2))) + z * np.exp(-0.5 * z * z) / np.sqrt(2 * np.pi)


def forward(flat, x, keep=False):
    layers = unflatten(flat)
    h = np.asarray(x, np.float64)
    acts = [h]
    zs = []
    for li, (W, b) in enumerate(layers):
        z = h @ W.T + b
        zs.append(z)
        h = gelu(z) if li < len(layers) - 1 else z
        acts.append(h)
    return (h, acts, zs) if keep else h


def loss_and_grads(flat, x, y):
    o, acts, zs = forward(flat, x, keep=True)
    layers = unflatten(flat)
    n = x.shape[0]
    d = o - y
    loss = float((d * d).sum() / (n * 5))
    g = 2 * d / (n * 5)
    grads = [None] * len(layers)
    for li in range(len(layers) - 1, -1, -1):
        W, _ = layers[li]
        grads[li] = (g.T @ acts[li], g.sum(0))
        if li:
            g = (g @ W) * gelu_grad(zs[li - 1])
    return loss, flatten(grads)
