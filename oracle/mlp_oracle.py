"""FP64 numpy restatement of the warm-start MLP -- TEST INFRASTRUCTURE ONLY.

The checker for the CUDA training kernels (warpvbd_b200/csrc/vbd_warmstart.cu):
forward pass, mean-squared-error loss and the analytic gradients with respect
to every parameter, in the parameter layout of include/vbd_b200.h
(W1[64][22] b1[64] W2[64][64] b2[64] W3[3][64] b3[3]).  Not part of the
reference, which has no learned component.
"""
import numpy as np

N_IN, N_HID, N_OUT = 22, 64, 3
SIZES = [("W1", (N_HID, N_IN)), ("b1", (N_HID,)), ("W2", (N_HID, N_HID)), ("b2", (N_HID,)),
         ("W3", (N_OUT, N_HID)), ("b3", (N_OUT,))]
N_PARAMS = sum(int(np.prod(s)) for _, s in SIZES)


def unpack(p):
    out, o = {}, 0
    for name, shape in SIZES:
        n = int(np.prod(shape))
        out[name] = np.asarray(p[o:o + n], dtype=np.float64).reshape(shape)
        o += n
    return out


def pack(d):
    return np.concatenate([np.asarray(d[name], np.float64).reshape(-1) for name, _ in SIZES])


def silu(a):
    return a / (1.0 + np.exp(-a))


def silu_grad(a):
    s = 1.0 / (1.0 + np.exp(-a))
    return s * (1.0 + a * (1.0 - s))


def forward(p, X):
    """X [B, >=21] -> (out [B, 3], cache)."""
    w = unpack(p)
    x = np.asarray(X, np.float64)[:, :N_IN]
    a1 = x @ w["W1"].T + w["b1"]
    h1 = silu(a1)
    a2 = h1 @ w["W2"].T + w["b2"]
    h2 = silu(a2)
    out = h2 @ w["W3"].T + w["b3"]
    return out, (x, a1, h1, a2, h2)


def loss_and_grad(p, X, Y):
    """mean over B*3 outputs of the squared error, and its gradient."""
    w = unpack(p)
    out, (x, a1, h1, a2, h2) = forward(p, X)
    B = x.shape[0]
    d = out - np.asarray(Y, np.float64)
    loss = float((d * d).sum() / (3 * B))
    dout = 2.0 * d / (3 * B)
    g = {"W3": dout.T @ h2, "b3": dout.sum(0)}
    d2 = (dout @ w["W3"]) * silu_grad(a2)
    g["W2"] = d2.T @ h1
    g["b2"] = d2.sum(0)
    d1 = (d2 @ w["W2"]) * silu_grad(a1)
    g["W1"] = d1.T @ x
    g["b1"] = d1.sum(0)
    return loss, pack(g), float((d * d).sum())
