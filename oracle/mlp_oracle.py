"""CPU restatement of the learned con2prim network's forward and backward
passes, for checking the tensor-core kernels (astrofd_b200/csrc/mlp.cu).

TEST INFRASTRUCTURE ONLY.  It follows the kernels' arithmetic contract:
operands rounded to bfloat16 where the kernels store them in shared memory
(input features, weights, hidden activations, ReLU derivatives, the output
gradients dZ), products accumulated in high precision (float64 here, float32
on the tensor cores), biases and the loss in float32/float64.  The hidden
layers use ReLU, which the kernels apply inside the bfloat16 rounding of the
activations (the same value: rounding commutes with max(., 0)).
"""
import numpy as np


def bf16(a):
    """Round-to-nearest-even to bfloat16, returned as float64."""
    a = np.ascontiguousarray(np.asarray(a, dtype=np.float32))
    u = a.view(np.uint32)
    r = ((u >> 16) & 1) + np.uint32(0x7FFF)
    return ((u + r) & np.uint32(0xFFFF0000)).view(np.float32).astype(np.float64)


def relu(z):
    return np.maximum(z, 0.0)


def relu_grad(z):
    return (z > 0.0).astype(np.float64)


def forward(P, X):
    """P: dict of parameter arrays (W[out][in]); X: raw features [n, 5].
    Returns outputs in normalised target units and the cached activations."""
    xn = (X.astype(np.float32) - P["xmu"]) / P["xsd"]
    h0 = bf16(xn)
    Ws = [bf16(P[k]) for k in ("W1", "W2", "W3", "W4")]
    bs = [P[k].astype(np.float64) for k in ("b1", "b2", "b3", "b4")]
    hs, ds = [h0], []
    h = h0
    for l in range(3):
        z = h @ Ws[l].T + bs[l]
        ds.append(relu_grad(z))
        h = bf16(relu(z))
        hs.append(h)
    y = h @ Ws[3].T + bs[3]
    return y, hs, ds, Ws


def loss_and_grads(P, X, T):
    """Mean squared error in normalised target units and its gradient with
    respect to W1 b1 W2 b2 W3 b3 W4 b4."""
    n = X.shape[0]
    y, hs, ds, Ws = forward(P, X)
    t = (T.astype(np.float32) - P["ymu"]) / P["ysd"]
    e = y - t
    loss = float(np.mean(e * e))
    dz = bf16(2.0 * e / (n * y.shape[1]))
    g = {}
    for l in (3, 2, 1, 0):
        g[f"W{l + 1}"] = dz.T @ hs[l]
        g[f"b{l + 1}"] = dz.sum(0)
        if l > 0:
            dz = bf16((dz @ Ws[l]) * ds[l - 1])
    return loss, g
