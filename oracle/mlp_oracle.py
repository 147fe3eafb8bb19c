"""CPU ORACLE -- test infrastructure only.  Never imported by the product.

numpy restatement of the learned-preconditioner network of the engine (no counterpart in the
reference, so parity is pinned by finite differences of this restatement, not by reference
vectors): features, forward pass with the engine's BF16 rounding points (weights of all layers,
activations entering layers 2 and 3), the loss mean(wgt (t (1 + R tanh m) - tgt)^2), R = 0.25, with
t = -r/u (0 when |u| <= 1e-6), and its gradient by back-propagation with the rounding treated as
identity (straight-through), which is what the GPU trainer computes.
"""
import numpy as np

NIN, NH = 35, 64
RANGE = 0.25  # factor = 1 + RANGE * tanh(m)
OFF_W1 = 0
OFF_B1 = OFF_W1 + NH * NIN
OFF_W2 = OFF_B1 + NH
OFF_B2 = OFF_W2 + NH * NH
OFF_W3 = OFF_B2 + NH
OFF_B3 = OFF_W3 + NH * NH
OFF_W4 = OFF_B3 + NH
OFF_B4 = OFF_W4 + NH
NW = OFF_B4 + 1


def bf16(x):
    """Round float32 values to the nearest BF16 (ties to even), returned as float32."""
    a = np.ascontiguousarray(x, dtype=np.float32)
    b = a.view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    return b.astype(np.uint32).view(np.float32).reshape(a.shape)


def unpack(w):
    w = np.asarray(w)
    return (w[OFF_W1:OFF_B1].reshape(NH, NIN), w[OFF_B1:OFF_W2], w[OFF_W2:OFF_B2].reshape(NH, NH), w[OFF_B2:OFF_W3],
            w[OFF_W3:OFF_B3].reshape(NH, NH), w[OFF_B3:OFF_W4], w[OFF_W4:OFF_B4], w[OFF_B4])


def features(ea, eb, u, r):
    e = np.asarray(ea, dtype=np.uint64) | (np.asarray(eb, dtype=np.uint64) << np.uint64(16))
    X = np.zeros((len(e), NIN), dtype=np.float32)
    for i in range(32):
        X[:, i] = ((e >> np.uint64(i)) & np.uint64(1)).astype(np.float32)
    u = np.asarray(u, dtype=np.float32)
    au = np.abs(u)
    X[:, 32] = u / (np.float32(1) + au)
    X[:, 33] = np.float32(0.05) / (np.float32(0.05) + au)
    X[:, 34] = np.log2(np.abs(np.asarray(r, dtype=np.float32)) + np.float32(2.0 ** -30)) / np.float32(30) + np.float32(1)
    return X


def forward(w, X, rounding=True, dtype=np.float32):
    W1, b1, W2, b2, W3, b3, w4, b4 = unpack(np.asarray(w, dtype=dtype))
    rd = bf16 if rounding else (lambda a: a)
    W1r, W2r, W3r, w4r = rd(W1).astype(dtype), rd(W2).astype(dtype), rd(W3).astype(dtype), rd(w4).astype(dtype)
    X = X.astype(dtype)
    z1 = X @ W1r.T + b1
    h1 = rd(np.maximum(z1, 0)).astype(dtype)
    z2 = h1 @ W2r.T + b2
    h2 = rd(np.maximum(z2, 0)).astype(dtype)
    z3 = h2 @ W3r.T + b3
    h3 = np.maximum(z3, 0)
    m = h3 @ w4r + b4
    return {"h1": h1, "h2": h2, "h3": h3, "m": m, "W2r": W2r, "W3r": W3r, "w4r": w4r, "X": X}


def factor(w, ea, eb, u, r, rounding=True):
    return 1.0 + RANGE * np.tanh(forward(w, features(ea, eb, u, r), rounding)["m"])


def loss_grad(w, ea, eb, u, r, tgt, rounding=True, dtype=np.float32, wgt=None):
    """Weighted mean-squared loss and its gradient with respect to the master weights."""
    X = features(ea, eb, u, r)
    F = forward(w, X, rounding, dtype)
    u = np.asarray(u, dtype=np.float64)
    r = np.asarray(r, dtype=np.float64)
    t = np.where(np.abs(u) > 1e-6, -r / np.where(np.abs(u) > 1e-6, u, 1.0), 0.0)
    th = np.tanh(F["m"].astype(np.float64))
    diff = t * (1.0 + RANGE * th) - np.asarray(tgt, dtype=np.float64)
    n = len(u)
    ws = np.ones(n) if wgt is None else np.asarray(wgt, dtype=np.float64)
    loss = float(np.sum(ws * diff * diff) / n)
    dm = 2.0 * ws * diff * t * RANGE * (1.0 - th * th) / n
    h1, h2, h3 = (F[k].astype(np.float64) for k in ("h1", "h2", "h3"))
    g = np.zeros(NW)
    g[OFF_W4:OFF_B4] = dm @ h3
    g[OFF_B4] = dm.sum()
    d3 = np.outer(dm, F["w4r"].astype(np.float64)) * (h3 > 0)
    g[OFF_W3:OFF_B3] = (d3.T @ h2).ravel()
    g[OFF_B3:OFF_W4] = d3.sum(0)
    d2 = (d3 @ F["W3r"].astype(np.float64)) * (h2 > 0)
    g[OFF_W2:OFF_B2] = (d2.T @ h1).ravel()
    g[OFF_B2:OFF_W3] = d2.sum(0)
    d1 = (d2 @ F["W2r"].astype(np.float64)) * (h1 > 0)
    g[OFF_W1:OFF_B1] = (d1.T @ F["X"].astype(np.float64)).ravel()
    g[OFF_B1:OFF_W2] = d1.sum(0)
    return loss, g


def random_weights(seed, output_scale=0.3):
    rng = np.random.default_rng(seed)
    w = np.zeros(NW, dtype=np.float32)
    for off, fi, fo in ((OFF_W1, NIN, NH), (OFF_W2, NH, NH), (OFF_W3, NH, NH)):
        a = np.sqrt(6.0 / (fi + fo))
        w[off:off + fi * fo] = rng.uniform(-a, a, fi * fo)
    w[OFF_B1:OFF_W2] = rng.normal(0, 0.1, NH)
    w[OFF_B2:OFF_W3] = rng.normal(0, 0.1, NH)
    w[OFF_B3:OFF_W4] = rng.normal(0, 0.1, NH)
    w[OFF_W4:OFF_B4] = rng.normal(0, output_scale, NH)
    w[OFF_B4] = 0.05
    return w


def random_samples(n, seed):
    rng = np.random.default_rng(seed)
    ea = rng.integers(0, 1 << 16, n).astype(np.uint32) & rng.integers(0, 1 << 16, n).astype(np.uint32)
    eb = rng.integers(0, 1 << 16, n).astype(np.uint32) & rng.integers(0, 1 << 16, n).astype(np.uint32)
    u = rng.uniform(0.05, 6.0, n) * rng.choice([-1.0, 1.0, 1.0, 1.0, 1.0], n)
    u = u.astype(np.float32)
    r = (rng.normal(0, 1, n) * 10.0 ** rng.uniform(-6, 0, n)).astype(np.float32)
    t = np.where(np.abs(u) > 1e-6, -r / u, 0.0)
    tgt = (t * (1.0 + 0.3 * np.sin(3 * u)) + 0.01 * rng.normal(0, 1, n) * np.abs(r)).astype(np.float32)
    wgt = rng.uniform(0.5, 2.0, n).astype(np.float32)
    return {"ea": ea, "eb": eb, "u": u, "r": r, "tgt": tgt, "wgt": wgt}
