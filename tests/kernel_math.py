"""numpy restatement of the CUDA kernel's per-slot closed form (slot_accumulate in
warpvbd_b200/csrc/vbd_kernels.cu), so its algebra can be checked against the
oracle's literal matrix formulation on the CPU.  Test helper only."""
import numpy as np


def shape_gradients(X4):
    """b_q (rows of Dm^-1, b_3 = -sum) for rest positions X4 [4,3]."""
    Dm = np.stack([X4[0] - X4[3], X4[1] - X4[3], X4[2] - X4[3]], axis=1)
    inv = np.linalg.inv(Dm)
    b = np.zeros((4, 3))
    b[:3] = inv
    b[3] = -inv.sum(axis=0)
    return b, abs(np.linalg.det(Dm)) / 6.0


def material_coeffs(material, mu, lam, vol):
    if material == "snh":
        mu2, lam2 = 4.0 * mu / 3.0, lam + 5.0 * mu / 6.0
        return vol * mu2, vol * lam2
    return vol * mu, vol * lam


def slot_grad_hess(material, X4, x4, a, mu, lam):
    """Elastic gradient / Hessian of vertex a of one tet, kernel closed form."""
    b_all, vol = shape_gradients(X4)
    p0, p1 = material_coeffs(material, mu, lam, vol)
    u = x4 - X4
    others = [q for q in range(4) if q != a]
    G = sum(np.outer(u[n] - u[a], b_all[n]) for n in others)
    b = -sum(b_all[n] for n in others)
    Fb = b + G @ b
    t = np.trace(G)
    if material == "snh":
        cofG = np.array([[G[1, 1] * G[2, 2] - G[1, 2] * G[2, 1], G[1, 2] * G[2, 0] - G[1, 0] * G[2, 2],
                          G[1, 0] * G[2, 1] - G[1, 1] * G[2, 0]],
                         [G[2, 1] * G[0, 2] - G[2, 2] * G[0, 1], G[2, 2] * G[0, 0] - G[2, 0] * G[0, 2],
                          G[2, 0] * G[0, 1] - G[2, 1] * G[0, 0]],
                         [G[0, 1] * G[1, 2] - G[0, 2] * G[1, 1], G[0, 2] * G[1, 0] - G[0, 0] * G[1, 2],
                          G[0, 0] * G[1, 1] - G[0, 1] * G[1, 0]]])
        detG = G[0] @ cofG[0]
        Jm1 = t + 0.5 * (t * t - np.trace(G @ G)) + detG
        Icm3 = 2 * t + (G * G).sum()
        inv = 1.0 / (Icm3 + 4.0)
        Cb = (1 + t) * b - G.T @ b + cofG @ b
        g = 0.25 * p0 * Icm3 * inv * Fb + 0.75 * p0 * (G @ b + G.T @ b - t * b - cofG @ b) \
            + p1 * Jm1 * Cb
        H = 2 * p0 * inv * inv * np.outer(Fb, Fb) + p0 * (Icm3 + 3) * inv * (b @ b) * np.eye(3) \
            + p1 * np.outer(Cb, Cb)
        return g, H
    E = 0.5 * (G + G.T + G.T @ G)
    trE = np.trace(E)
    F = np.eye(3) + G
    g = 2 * p0 * F @ (E @ b) + p1 * trE * Fb
    H = (p1 + p0) * np.outer(Fb, Fb) + p0 * (b @ b) * (F @ F.T) \
        + (p1 * trE * (b @ b) + 2 * p0 * (b @ E @ b)) * np.eye(3)
    return g, H


def slot_psi(material, X4, x4, a, mu, lam):
    """Strain energy of one tet seen from its vertex a, kernel closed form
    (slot_psi in warpvbd_b200/csrc/vbd_device.cuh; the kernel evaluates it from
    each tet's owner slot, its solved vertex of lowest id):
    SNH  p0/2 (Ic - 3 - ln(1 + (Ic - 3)/4)) + p1/2 (J - 1 - 3/4 p0/p1)^2, i.e.
         the reference's mu'/2 (Ic - 3) - mu'/2 ln(Ic + 1) + lambda'/2 (J - alpha)^2
         up to the constant mu'/2 ln 4, with J - 1 and Ic - 3 from G = F - I;
    StVK p0 E:E + p1/2 tr(E)^2."""
    b_all, vol = shape_gradients(X4)
    p0, p1 = material_coeffs(material, mu, lam, vol)
    u = x4 - X4
    others = [q for q in range(4) if q != a]
    G = sum(np.outer(u[n] - u[a], b_all[n]) for n in others)
    t = np.trace(G)
    if material == "snh":
        Jm1 = t + 0.5 * (t * t - np.trace(G @ G)) + np.linalg.det(G)
        Icm3 = 2.0 * t + np.sum(G * G)
        r = Jm1 - 0.75 * p0 / p1
        return 0.5 * p0 * (Icm3 - np.log1p(0.25 * Icm3)) + 0.5 * p1 * r * r
    E = 0.5 * (G + G.T + G.T @ G)
    return p0 * np.sum(E * E) + 0.5 * p1 * np.trace(E) ** 2
