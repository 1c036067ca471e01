"""FP64 CPU restatement of the tile-scoring MLP (64 -> 128 -> 128 -> 1, ReLU,
mean squared error) used to check the device forward and backward passes.
Parameter layout as in include/dtwj.h: W1 [128][64], b1, W2 [128][128], b2,
w3, b3."""
import numpy as np

IN, HID = 64, 128
SIZES = (("W1", HID * IN), ("b1", HID), ("W2", HID * HID), ("b2", HID), ("w3", HID), ("b3", 1))


def unpack(p):
    out, o = {}, 0
    for name, size in SIZES:
        out[name] = np.asarray(p[o:o + size], dtype=np.float64)
        o += size
    out["W1"] = out["W1"].reshape(HID, IN)
    out["W2"] = out["W2"].reshape(HID, HID)
    return out


def blocks(g):
    """The gradient split into its parameter blocks (flat)."""
    out, o = {}, 0
    for name, size in SIZES:
        out[name] = np.asarray(g[o:o + size], dtype=np.float64)
        o += size
    return out


def forward(p, x):
    q = unpack(p)
    x = np.asarray(x, dtype=np.float64)
    h1 = np.maximum(x @ q["W1"].T + q["b1"], 0.0)
    h2 = np.maximum(h1 @ q["W2"].T + q["b2"], 0.0)
    return h2 @ q["w3"] + q["b3"][0], h1, h2


def bf16(a):
    """Round to bfloat16 (nearest, ties to even) and back, as float64."""
    u = np.asarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def grad(p, x, y, bf16_operands=False):
    """(gradient in the parameter layout, loss) of mean((y_hat - y)^2).  With
    bf16_operands every GEMM operand is rounded to bfloat16 where the device
    rounds it (X, W1, H1, W2 in the forward; dH2, H1, W2, dH1, X in the
    backward), all arithmetic staying FP64."""
    r = bf16 if bf16_operands else (lambda a: np.asarray(a, dtype=np.float64))
    q = unpack(p)
    x = np.asarray(x, dtype=np.float64)
    y = np.asarray(y, dtype=np.float64)
    h1 = np.maximum(r(x) @ r(q["W1"]).T + q["b1"], 0.0)
    h2 = np.maximum(r(h1) @ r(q["W2"]).T + q["b2"], 0.0)
    yh = h2 @ q["w3"] + q["b3"][0]
    e = yh - y
    n = x.shape[0]
    dy = 2.0 * e / n
    dw3 = h2.T @ dy
    db3 = np.array([dy.sum()])
    dh2 = np.outer(dy, q["w3"]) * (h2 > 0)
    dW2 = r(dh2).T @ r(h1)
    db2 = dh2.sum(0)
    dh1 = (r(dh2) @ r(q["W2"])) * (h1 > 0)
    dW1 = r(dh1).T @ r(x)
    db1 = dh1.sum(0)
    g = np.concatenate([dW1.ravel(), db1, dW2.ravel(), db2, dw3, db3])
    return g, float(np.mean(e * e))
