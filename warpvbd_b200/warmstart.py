"""Learned warm start for VBD (not part of the reference).

A per-vertex MLP (22 inputs -> 64 SiLU -> 64 SiLU -> 3) predicts the
correction each time step converges to, relative to the inertia guess and
in units of the vertex's own motion scale (so the regression is scale-free).  The
solver starts a step from the prediction when it lowers the incremental
potential and from the inertia guess otherwise, then runs its sweeps to the
same tolerance, so plain VBD still decides the result.  Features, inference
(bf16 weights), training (fp32 forward, backward and Adam) and the energy
test all run as CUDA kernels of libvbd_b200.so; this module only
orchestrates them, with torch tensors as device buffers.

    data = rollout_dataset(seed=1)               # plain-VBD rollouts on the GPU
    model, info = train_warmstart(*data)         # trained by the CUDA kernels
    solver.set_warmstart(model)                  # VBDSolver or BatchedVBDSolver

The network acts on normalised features and predicts normalised targets; a
model is the pair (parameters, normalisation), the normalisation being the
inputs' mean[22] and 1/std[22] then the targets' std[3] and mean[3].  The
inference kernel applies it in fp32 around bf16 weights (folding it into the
weights would put large cancellations into bf16).
"""
import ctypes
import os

import numpy as np

from . import _lib, scenes

N_IN, N_HID, N_OUT = 22, 64, 3
N_PARAMS = N_HID * N_IN + N_HID + N_HID * N_HID + N_HID + N_OUT * N_HID + N_OUT  # 5827
FEAT_WIDTH = 24
DEFAULT_WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data",
                               "warmstart_mlp.npz")
# parameter slices, in the order of include/vbd_b200.h
_W1 = slice(0, N_HID * N_IN)
_B1 = slice(_W1.stop, _W1.stop + N_HID)
_W2 = slice(_B1.stop, _B1.stop + N_HID * N_HID)
_B2 = slice(_W2.stop, _W2.stop + N_HID)
_W3 = slice(_B2.stop, _B2.stop + N_OUT * N_HID)
_B3 = slice(_W3.stop, _W3.stop + N_OUT)


def _torch():
    import torch
    return torch


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def init_params(seed=0):
    """Glorot-uniform weights, zero biases (fp32)."""
    rng = np.random.default_rng(seed)
    p = np.zeros(N_PARAMS, np.float32)
    for sl, (fo, fi) in ((_W1, (N_HID, N_IN)), (_W2, (N_HID, N_HID)), (_W3, (N_OUT, N_HID))):
        a = np.sqrt(6.0 / (fi + fo))
        p[sl] = rng.uniform(-a, a, size=fo * fi).astype(np.float32)
    return p


def fold_normalization(p, mu_x, sd_x, mu_y, sd_y):
    """Parameters trained on (x - mu_x)/sd_x -> (y - mu_y)/sd_y, rewritten to
    act on raw features and produce raw targets."""
    p = np.asarray(p, np.float64).copy()
    W1 = p[_W1].reshape(N_HID, N_IN) / sd_x[None, :]
    p[_B1] = p[_B1] - W1 @ mu_x
    p[_W1] = W1.reshape(-1)
    W3 = p[_W3].reshape(N_OUT, N_HID) * sd_y[:, None]
    p[_B3] = p[_B3] * sd_y + mu_y
    p[_W3] = W3.reshape(-1)
    return p.astype(np.float32)


class MLPTrainer:
    """Adam on the CUDA training kernels (vbd_mlp_train_batch, vbd_mlp_adam)."""

    def __init__(self, params, device="cuda", max_batch=8192):
        torch = _torch()
        self.torch = torch
        self.device = torch.device(device)
        self.P = torch.tensor(np.asarray(params, np.float32), device=self.device)
        self.G = torch.zeros_like(self.P)
        self.M = torch.zeros_like(self.P)
        self.V = torch.zeros_like(self.P)
        self.max_batch = max_batch
        self.scratch = torch.empty(_lib.load().vbd_mlp_train_scratch_floats(max_batch),
                                   device=self.device)
        self.loss = torch.zeros(1, dtype=torch.float64, device=self.device)
        self.t = 0
        self.stream = torch.cuda.current_stream(self.device).cuda_stream

    def gradient(self, X, Y, idx=None, batch=None):
        """Loss gradient (and sum of squared errors) of one minibatch."""
        L = _lib.load()
        batch = int(batch if batch is not None else (idx.numel() if idx is not None else X.shape[0]))
        if batch > self.max_batch:
            raise ValueError("batch larger than the trainer's scratch")
        self.loss.zero_()
        _lib.check(L.vbd_mlp_train_batch(_ptr(X), _ptr(Y), _ptr(idx), batch, _ptr(self.P),
                                         _ptr(self.G), _ptr(self.scratch), _ptr(self.loss),
                                         ctypes.c_void_p(self.stream)), "vbd_mlp_train_batch")
        return self.G, self.loss

    def step(self, lr, beta1=0.9, beta2=0.999, eps=1e-8):
        self.t += 1
        _lib.check(_lib.load().vbd_mlp_adam(_ptr(self.P), _ptr(self.G), _ptr(self.M),
                                            _ptr(self.V), N_PARAMS, float(lr), float(beta1),
                                            float(beta2), float(eps), self.t,
                                            ctypes.c_void_p(self.stream)), "vbd_mlp_adam")

    def forward(self, X):
        torch = self.torch
        n = X.shape[0]
        out = torch.empty((n, N_OUT), device=self.device)
        _lib.check(_lib.load().vbd_mlp_forward(_ptr(X), n, _ptr(self.P), _ptr(out),
                                               None, ctypes.c_void_p(self.stream)),
                   "vbd_mlp_forward")
        return out

    def fit(self, X, Y, epochs=10, batch=4096, lr=2e-3, lr_end=1e-4, seed=0):
        """Minibatch Adam with a cosine learning-rate decay; returns the mean
        squared error of every epoch."""
        torch = self.torch
        n = X.shape[0]
        gen = torch.Generator(device=self.device)
        gen.manual_seed(seed)
        steps_per_epoch = max(1, n // batch)
        total = epochs * steps_per_epoch
        history = []
        for ep in range(epochs):
            perm = torch.randperm(n, generator=gen, device=self.device).to(torch.int32)
            acc = torch.zeros(1, dtype=torch.float64, device=self.device)
            for k in range(steps_per_epoch):
                idx = perm[k * batch:(k + 1) * batch]
                _, loss = self.gradient(X, Y, idx, batch)
                acc += loss
                frac = (ep * steps_per_epoch + k) / max(1, total - 1)
                cur = lr_end + 0.5 * (lr - lr_end) * (1.0 + np.cos(np.pi * frac))
                self.step(cur)
            history.append(float(acc.item()) / (steps_per_epoch * batch * N_OUT))
        return history

    def params(self):
        return self.P.detach().cpu().numpy().copy()


def training_envs(seed, n_env, fine=False, cube=(5, 12), column=(3, 24)):
    """Seeded cantilever and mass-spring environments with random materials
    (E log-uniform in [1e5, 1e7] Pa, nu uniform in [0.30, 0.48]).  Cantilevers
    have 5 cm voxels (10-30 voxels long); with `fine`, every other one is a
    1 m beam of 40 or 80 voxels (2.5 / 1.25 cm) instead, so that beams of the
    benchmark's resolutions are in the data too.  Mass-springs: cube edge and
    column length uniform integers in `cube` and `column` (inclusive)."""
    rng = np.random.default_rng(seed)
    envs = []
    for i in range(n_env):
        E = float(np.exp(rng.uniform(np.log(1e5), np.log(1e7))))
        nu = float(rng.uniform(0.30, 0.48))
        if i % 3 == 0 and fine and i % 6 == 0:
            n = int(rng.choice([40, 80]))
            envs.append(scenes.cantilever(n, youngs=E, poisson=nu))
        elif i % 3 == 0:
            n = int(rng.choice([10, 20, 30]))
            envs.append(scenes.cantilever(n, max(1, n // 10), max(1, n // 10), length=n * 0.01 * 5,
                                          youngs=E, poisson=nu))
        else:
            envs.append(scenes.mass_spring(int(rng.integers(cube[0], cube[1] + 1)),
                                           int(rng.integers(column[0], column[1] + 1)),
                                           youngs=E, poisson=nu))
    return envs


def rollout_dataset(seed=1, n_batches=6, envs_per_batch=24, steps=100, record_every=5,
                    dt=1e-3, tol=1e-7, max_iter=1000, velocity_noise=0.1, device="cuda",
                    fine=False, target_tol=None, target_max_iter=20000, cube=(5, 12),
                    column=(3, 24)):
    """Plain-VBD rollouts on the GPU: every `record_every` steps the features
    at the step start and the correction the step converged to.  Each batch
    has its own random gravity direction; every active vertex starts with
    N(0, velocity_noise^2) velocity.  Returns (X [N, 24], Y [N, 3]) torch
    tensors on the device.

    `target_tol`: the recorded steps are first solved to this tighter
    tolerance (at most `target_max_iter` sweeps) for their targets -- the
    step's converged solution rather than where VBD at `tol` stops -- and
    then, from the same state, at `tol` to continue the rollout, so the
    inputs follow the trajectories the solver runs at inference."""
    torch = _torch()
    from .batched import BatchedVBDSolver
    rng = np.random.default_rng(seed)
    Xs, Ys = [], []
    for b in range(n_batches):
        envs = training_envs(int(rng.integers(1 << 31)), envs_per_batch, fine=fine, cube=cube,
                             column=column)
        # batch 0 falls along -z; the others along a random direction
        d = np.array([0.0, 0.0, -1.0]) if b == 0 else rng.normal(size=3)
        g = 9.81 * d / np.linalg.norm(d)
        sol = BatchedVBDSolver(envs, gravity=g, dx_tol=tol, max_iter=max_iter, device=device)
        act = np.concatenate([e.active for e in envs])
        # velocity-noise level cycles through 0, 0.1 sigma, sigma: the features
        # are scale-free, but the mix covers motions dominated by gravity as
        # well as by the initial velocity
        sigma = velocity_noise * (0.0, 0.1, 1.0)[b % 3]
        v0 = rng.normal(scale=sigma, size=(act.size, 3)) * act[:, None]
        sol.set_state(velocities=v0)
        n = sol.n_vertices
        feat = torch.empty((n, FEAT_WIDTH), device=device)
        tgt = torch.empty((n, N_OUT), device=device)
        for k in range(steps):
            if k % record_every == 0:
                sol.ws_features(dt, feat)
                if target_tol is not None:
                    x0, v0 = sol.positions(), sol.velocities()
                    sol.step(dt, dx_tol=target_tol, max_iter=target_max_iter)
                    sol.ws_targets(feat, tgt)
                    sol.set_state(positions=x0, velocities=v0)
                    sol.step(dt)
                else:
                    sol.step(dt)
                    sol.ws_targets(feat, tgt)
                mask = feat[:, 23] > 0
                Xs.append(feat[mask].clone())
                Ys.append(tgt[mask].clone())
            else:
                sol.step(dt)
        sol.close()
    return torch.cat(Xs), torch.cat(Ys)


def train_warmstart(X, Y, epochs=12, batch=4096, lr=2e-3, seed=0, device="cuda"):
    """Train on raw features / targets; returns (model, info): model =
    (parameters of the normalised network, normalisation vector [50])."""
    torch = _torch()
    mu_x = X[:, :N_IN].double().mean(0)
    sd_x = X[:, :N_IN].double().std(0).clamp_min(1e-6)
    mu_y = Y.double().mean(0)
    sd_y = Y.double().std(0).clamp_min(1e-9)
    Xn = X.clone()
    Xn[:, :N_IN] = ((X[:, :N_IN].double() - mu_x) / sd_x).float()
    Yn = ((Y.double() - mu_y) / sd_y).float().contiguous()
    trainer = MLPTrainer(init_params(seed), device=device, max_batch=batch)
    hist = trainer.fit(Xn.contiguous(), Yn, epochs=epochs, batch=batch, lr=lr, seed=seed)
    norm = np.concatenate([mu_x.cpu().numpy(), 1.0 / sd_x.cpu().numpy(), sd_y.cpu().numpy(),
                           mu_y.cpu().numpy()]).astype(np.float32)
    # fraction of the target variance the network explains (normalised space)
    with torch.no_grad():
        pred = trainer.forward(Xn.contiguous())
        r2 = 1.0 - float(((pred - Yn) ** 2).mean() / (Yn ** 2).mean())
    info = {"loss": hist, "r2": r2, "samples": int(X.shape[0])}
    return (trainer.params(), norm), info


def save(path, model, info=None):
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    params, norm = model
    extra = {} if info is None else {k: np.asarray(v) for k, v in info.items()}
    np.savez(path, params=np.asarray(params, np.float32), norm=np.asarray(norm, np.float32),
             **extra)


def load(path=DEFAULT_WEIGHTS):
    """(parameters, normalisation) of a saved model."""
    with np.load(path) as d:
        p = d["params"].astype(np.float32)
        n = d["norm"].astype(np.float32)
    if p.size != N_PARAMS or n.size != 2 * N_IN + 2 * N_OUT:
        raise ValueError(f"{path}: unexpected model sizes {p.size}, {n.size}")
    return p, n
