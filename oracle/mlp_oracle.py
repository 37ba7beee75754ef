"""FP64 reference of the warm-start MLP (numpy).

TEST INFRASTRUCTURE ONLY: the checker for the product's BF16 tensor-core
forward and backward kernels (climatenet_b200/csrc/mlp.cu).  Network
10 -> 64 -> 64 -> 3 with ReLU; parameters packed as
W1[64][10] b1[64] W2[64][64] b2[64] W3[3][64] b3[3]; loss = mean over samples
of the squared error summed over the 3 outputs.  It has no counterpart in the
reference, whose contact solver has no learned component.
"""
import numpy as np

IN, H, OUT = 10, 64, 3
SHAPES = [("W1", (H, IN)), ("b1", (H,)), ("W2", (H, H)), ("b2", (H,)), ("W3", (OUT, H)), ("b3", (OUT,))]
N_PARAMS = sum(int(np.prod(s)) for _, s in SHAPES)


def unpack(w):
    w = np.asarray(w, dtype=np.float64)
    out, o = {}, 0
    for name, shp in SHAPES:
        n = int(np.prod(shp))
        out[name] = w[o:o + n].reshape(shp)
        o += n
    return out


def pack(d):
    return np.concatenate([np.asarray(d[name], dtype=np.float64).ravel() for name, _ in SHAPES])


def forward(w, X):
    p = unpack(w)
    X = np.asarray(X, dtype=np.float64)
    z1 = X @ p["W1"].T + p["b1"]
    h1 = np.maximum(z1, 0.0)
    z2 = h1 @ p["W2"].T + p["b2"]
    h2 = np.maximum(z2, 0.0)
    return h2 @ p["W3"].T + p["b3"]


def loss_and_grad(w, X, T):
    """Loss and its gradient by backpropagation, all in FP64."""
    p = unpack(w)
    X = np.asarray(X, dtype=np.float64)
    T = np.asarray(T, dtype=np.float64)
    n = X.shape[0]
    z1 = X @ p["W1"].T + p["b1"]
    h1 = np.maximum(z1, 0.0)
    z2 = h1 @ p["W2"].T + p["b2"]
    h2 = np.maximum(z2, 0.0)
    y = h2 @ p["W3"].T + p["b3"]
    e = y - T
    loss = float((e * e).sum() / n)
    dy = 2.0 * e / n
    g = {"W3": dy.T @ h2, "b3": dy.sum(0)}
    dz2 = (dy @ p["W3"]) * (z2 > 0)
    g["W2"] = dz2.T @ h1
    g["b2"] = dz2.sum(0)
    dz1 = (dz2 @ p["W2"]) * (z1 > 0)
    g["W1"] = dz1.T @ X
    g["b1"] = dz1.sum(0)
    return loss, pack(g)
