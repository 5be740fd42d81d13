"""CPU oracle of the learned-correction MLP (TEST INFRASTRUCTURE ONLY).

Restates in NumPy the forward pass, the loss and the hand-written backward
pass of gaukuk_b200/csrc/gk_mlp.cu: 16 -> 64 -> 64 -> 4 with the tanh form of
GELU, mean over samples of the squared error summed over the 4 outputs.  With
bf16=True the values are rounded to BF16 at the same points as the device
kernels (inputs, weights, hidden activations, dY, dZ2, dZ1), and everything
else is computed in float64, so the device gradient should match to FP32
accumulation error.  Only tests use this module.
"""
import numpy as np

NI, NH, NO = 16, 64, 4
A, B = 0.7978845608028654, 0.044715


def bf16(x):
    """Round float64 values to the nearest BF16 (ties to even), returned as float64."""
    f = np.asarray(x, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(blob):
    o = 0
    w1 = blob[o:o + NH * NI].reshape(NH, NI); o += NH * NI
    b1 = blob[o:o + NH]; o += NH
    w2 = blob[o:o + NH * NH].reshape(NH, NH); o += NH * NH
    b2 = blob[o:o + NH]; o += NH
    w3 = blob[o:o + NO * NH].reshape(NO, NH); o += NO * NH
    b3 = blob[o:o + NO]
    return [np.asarray(v, np.float64) for v in (w1, b1, w2, b2, w3, b3)]


def gelu(x):
    th = np.tanh(A * (x + B * x ** 3))
    return 0.5 * x * (1 + th), 0.5 * (1 + th) + 0.5 * x * (1 - th ** 2) * A * (1 + 3 * B * x * x)


def forward_backward(blob, X, T, rounding=True, pair_w=None):
    """Loss and the batch-summed gradient (NPARAM).  pair_w None: the sum of
    squared errors.  Otherwise samples (2m, 2m + 1) are pairs and each pair
    contributes (1 - w)(e0^2 + e1^2) + w (e1 - e0)^2 per output
    (gaukuk_b200/csrc/gk_mlp.cu, k_mlp_grad)."""
    r = bf16 if rounding else (lambda v: np.asarray(v, np.float64))
    w1, b1, w2, b2, w3, b3 = unpack(blob)
    w1r, w2r, w3r = r(w1), r(w2), r(w3)
    x = r(X)
    z1 = x @ w1r.T + b1
    h1, d1 = gelu(z1)
    h1 = r(h1)
    z2 = h1 @ w2r.T + b2
    h2, d2 = gelu(z2)
    h2 = r(h2)
    y = h2 @ w3r.T + b3
    res = y - T
    n = len(X)
    if pair_w is None:
        loss = float(np.sum(res * res))
        dres = res
    else:
        w = float(pair_w)
        e0, e1 = res[0::2], res[1::2]
        d = e1 - e0
        loss = float(np.sum((1 - w) * (e0 * e0 + e1 * e1) + w * d * d))
        dres = np.empty_like(res)
        dres[0::2] = (1 - w) * e0 - w * d
        dres[1::2] = (1 - w) * e1 + w * d
    dy = r(2.0 / n * dres)
    dh2 = dy @ w3r
    dz2 = r(dh2 * d2)
    dh1 = dz2 @ w2r
    dz1 = r(dh1 * d1)
    g = [dz1.T @ x, dz1.sum(0), dz2.T @ h1, dz2.sum(0), dy.T @ h2, dy.sum(0)]
    return loss, np.concatenate([v.ravel() for v in g]), y
