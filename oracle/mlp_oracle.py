"""CPU restatement of the learned return map's network (test infrastructure only).

Only tests/ import this module, as the checker of the device MLP kernels: the forward pass and the
gradient of the weighted mean squared error that the device trains with. It follows the layout of
the parameter vector of mpm_surrogate (include/mpm_b200.h): W1 [64][16], b1 [64], W2 [64][64],
b2 [64], W3 [8][64], b3 [8], weights W[out][in], ReLU after layers 1 and 2.

There is no reference counterpart (the reference has no learned return map), so this restatement
is pinned by central finite differences of its own loss (tests/test_surrogate.py).

emulate_bf16=True rounds every tensor-core operand to BF16 (round to nearest even) exactly where
the device kernels round: inputs, weights, the activations fed to the next layer, the output
gradient and the pre-activation gradients fed to the backward GEMMs. Accumulation stays FP64, so
the device must agree to FP32 accumulation order and rare BF16 tie flips.
"""
import numpy as np

H = 64
SIZES = dict(W1=(H, 16), b1=(H,), W2=(H, H), b2=(H,), W3=(8, H), b3=(8,))
ORDER = ("W1", "b1", "W2", "b2", "W3", "b3")
NPARAMS = sum(int(np.prod(s)) for s in SIZES.values())  # 5768


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    out, k = {}, 0
    for name in ORDER:
        n = int(np.prod(SIZES[name]))
        out[name] = p[k:k + n].reshape(SIZES[name])
        k += n
    return out


def pack(d):
    return np.concatenate([np.asarray(d[name], dtype=np.float64).ravel() for name in ORDER])


def bf16(x):
    """Round to the nearest BF16 value (ties to even), returned as float64."""
    a = np.asarray(x, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def forward(p, X, emulate_bf16=False):
    """Outputs (n, 8) and the cache for backward. X is (n, 8)."""
    r = bf16 if emulate_bf16 else (lambda a: np.asarray(a, dtype=np.float64))
    w = unpack(p)
    Xp = np.zeros((X.shape[0], 16))
    Xp[:, :8] = X
    Xr = r(Xp)
    z1 = Xr @ r(w["W1"]).T + w["b1"]
    h1 = np.maximum(z1, 0)
    h1r = r(h1)
    z2 = h1r @ r(w["W2"]).T + w["b2"]
    h2 = np.maximum(z2, 0)
    h2r = r(h2)
    y = h2r @ r(w["W3"]).T + w["b3"]
    return y, dict(Xr=Xr, h1=h1, h1r=h1r, h2=h2, h2r=h2r, w=w, r=r)


def loss_grad(p, X, Y, out_weight=None, emulate_bf16=False):
    """Weighted mean squared error over the 7 outputs and its gradient (flat, like p). Column 7 of
    a target row is that sample's weight (the device trains on plastic states only: weight 1)."""
    n = X.shape[0]
    wo = np.ones(8) if out_weight is None else np.asarray(out_weight, dtype=np.float64).copy()
    wo[7] = 0.0
    ws = np.asarray(Y, dtype=np.float64)[:, 7:8]
    y, c = forward(p, X, emulate_bf16)
    r, w = c["r"], c["w"]
    e = y - Y
    loss = float(np.sum(ws * wo * e * e) / n)
    dy = 2.0 * ws * wo * e / n
    dyr = r(dy)
    d2 = (dyr @ r(w["W3"])) * (c["h2"] > 0)
    d2r = r(d2)
    d1 = (d2r @ r(w["W2"])) * (c["h1"] > 0)
    d1r = r(d1)
    g = dict(W3=dyr.T @ c["h2r"], b3=dy.sum(0), W2=d2r.T @ c["h1r"], b2=d2.sum(0),
             W1=d1r.T @ c["Xr"], b1=d1.sum(0))
    g["W1"][:, 8:] = 0.0
    g["W3"][7, :] = 0.0
    g["b3"][7] = 0.0
    return loss, pack(g)
