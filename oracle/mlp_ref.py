"""FP64 numpy reference of the closure network's forward and backward pass.

TEST INFRASTRUCTURE ONLY (the checker for the tensor-core kernels).  GEMM
operands are rounded to BF16 exactly where the device rounds them (inputs,
hidden activations, output-layer and hidden gradients, weights); everything
else is FP64, so differences against the device are accumulation order and
the device's FP32 arithmetic.
"""
import numpy as np

NFEAT, KIN, HID, NOUT = 12, 16, 64, 16


def bf16(x):
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16).astype(np.uint32) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def hswish(z):
    """Hidden activation: hard-swish z * clip(z/6 + 1/2, 0, 1) (the device
    computes it in FP32 as z * sat(fma(z, 1/6, 1/2)))."""
    z32 = np.asarray(z, dtype=np.float32)
    t = np.clip(z32 * np.float32(1.0 / 6.0) + np.float32(0.5), 0.0, 1.0)
    return (z32 * t).astype(np.float64)


def hswish_grad(z):
    return np.where(z <= -3.0, 0.0, np.where(z >= 3.0, 1.0, z / 3.0 + 0.5))


def sigm(z):
    return 1.0 / (1.0 + np.exp(-z))


def softplus(z):
    return np.where(z > 20, z, np.log1p(np.exp(np.minimum(z, 20))))


def normalise(Xraw, meta):
    X = np.zeros((len(Xraw), KIN))
    X[:, :NFEAT] = (Xraw.astype(np.float32) - meta[:NFEAT]) * meta[NFEAT:2 * NFEAT]
    return bf16(X.astype(np.float32))


def forward(P, X):
    """X: normalised, bf16-rounded (n x 16).  Returns caches and outputs."""
    W = {k: bf16(P[k]) for k in ("W1", "W2", "W3", "W4")}
    b = {k: P[k].astype(np.float64) for k in ("b1", "b2", "b3", "b4")}
    Z1 = X @ W["W1"].T + b["b1"]
    A1 = bf16(hswish(Z1).astype(np.float32))
    Z2 = A1 @ W["W2"].T + b["b2"]
    A2 = bf16(hswish(Z2).astype(np.float32))
    Z3 = A2 @ W["W3"].T + b["b3"]
    A3 = bf16(hswish(Z3).astype(np.float32))
    Z4 = A3 @ W["W4"].T + b["b4"]
    return dict(X=X, W=W, Z1=Z1, A1=A1, Z2=Z2, A2=A2, Z3=Z3, A3=A3, Z4=Z4, out=softplus(Z4[:, :2]))


def backward(c, Y):
    B = len(Y)
    Z4 = c["Z4"][:, :2]
    r = softplus(Z4) - Y
    loss = float(np.sum(r * r) / B)
    dZ4 = np.zeros((B, NOUT))
    dZ4[:, :2] = 2.0 * r * sigm(Z4) / B
    g = {"b4": dZ4.sum(0)}
    dZ4b = bf16(dZ4.astype(np.float32))
    g["W4"] = dZ4b.T @ c["A3"]
    dA = dZ4b @ c["W"]["W4"]
    for l, Aprev in ((3, c["A2"]), (2, c["A1"]), (1, c["X"])):
        z = c[f"Z{l}"]
        dZ = dA * hswish_grad(z)
        g[f"b{l}"] = dZ.sum(0)
        dZb = bf16(dZ.astype(np.float32))
        g[f"W{l}"] = dZb.T @ Aprev
        if l > 1:
            dA = dZb @ c["W"][f"W{l}"]
    return g, loss
