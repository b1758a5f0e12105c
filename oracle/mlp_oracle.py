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


def vertex_constants(X, tets, E, nu, rho):
    """Per-vertex warm-start constants (h, log10(E/(rho h^2)), nu, valence/20)
    and the valence, from incident-tet means: h is the mean of cbrt(6 V_t),
    log E, rho and nu are plain means over the incident tets."""
    X = np.asarray(X, np.float64)
    T = np.asarray(tets, np.int64).reshape(-1, 4)
    n = X.shape[0]
    D = np.stack([X[T[:, i]] - X[T[:, 3]] for i in range(3)], axis=2)
    vol = np.abs(np.linalg.det(D)) / 6.0
    k = np.bincount(T.reshape(-1), minlength=n).astype(np.float64)

    def vmean(per_tet):
        s = np.zeros(n)
        for i in range(4):
            np.add.at(s, T[:, i], per_tet)
        return np.divide(s, k, out=np.zeros(n), where=k > 0)
    h = vmean(np.cbrt(6.0 * vol))
    logE, r, v = vmean(np.log10(E)), vmean(rho), vmean(nu)
    with np.errstate(divide="ignore", invalid="ignore"):
        w1 = np.where(k > 0, logE - np.log10(r * h * h), 0.0)
    return np.stack([np.where(k > 0, h, 1.0), w1, v, k / 20.0], 1), k.astype(np.int64)


def features(X, tets, E, nu, rho, active, x, v, dt, g, x_prev=None, v_prev=None):
    """Feature rows [n, 24] of the coming step of length dt at state (x, v)
    (positions, velocities); x_prev, v_prev: the state the previous step
    started from (None before the first step: no history).  Rows of vertices
    that are not solved (fixed or without tets) are zero.  Row layout:
    0-2 inertia displacement v dt + g dt^2, 3-5 v dt, 6-8 1-ring mean of the
    neighbours' v dt minus the vertex's own, 9-11 the same for the
    displacement from rest, 12-14 the previous step's correction
    x - (x_prev + v_prev dt + g dt^2), 15-17 g dt^2 -- all divided by h and
    then by s, the RMS of the 18 -- then log10(E dt^2/(rho h^2)), nu,
    valence/20, log10 s, s, 1.  Neighbours count once per incident tet."""
    X = np.asarray(X, np.float64)
    T = np.asarray(tets, np.int64).reshape(-1, 4)
    n = X.shape[0]
    ws, k = vertex_constants(X, T, E, nu, rho)
    u = np.asarray(x, np.float64) - X
    vel = np.asarray(v, np.float64)
    g2 = np.asarray(g, np.float64) * dt * dt
    su, sv = np.zeros((n, 3)), np.zeros((n, 3))
    for a in range(4):
        for b in range(4):
            if a != b:
                np.add.at(su, T[:, a], u[T[:, b]] - u[T[:, a]])
                np.add.at(sv, T[:, a], vel[T[:, b]] - vel[T[:, a]])
    solved = np.asarray(active, bool) & (k > 0)
    cnt = np.maximum(3 * k, 1)[:, None]
    ih = 1.0 / ws[:, :1]
    if x_prev is not None:
        target = np.asarray(x_prev, np.float64) - X + np.asarray(v_prev, np.float64) * dt + g2
        up = u - target
    else:
        up = np.zeros((n, 3))
    d = np.concatenate([(vel * dt + g2) * ih, vel * dt * ih, sv / cnt * dt * ih, su / cnt * ih,
                        up * ih, np.broadcast_to(g2, (n, 3)) * ih], 1)
    s = np.sqrt((d * d).mean(1)) + 1e-30
    out = np.zeros((n, 24))
    out[:, :18] = d / s[:, None]
    out[:, 18] = ws[:, 1] + 2.0 * np.log10(dt)
    out[:, 19] = ws[:, 2]
    out[:, 20] = ws[:, 3]
    out[:, 21] = np.log10(s)
    out[:, 22] = s
    out[:, 23] = 1.0
    out[~solved] = 0.0
    return out
