"""JSON-lines metrics of a simulation loop: one line per step.

    log = StepLog("run.jsonl", n_solved=sol_info_vertices, dt=1e-3)
    for k in range(steps):
        t0 = time.perf_counter()
        sweeps = solver.step(1e-3)
        log.record(sweeps, time.perf_counter() - t0)
    log.close()

Each line holds the step index, the sweep count (the mean, max and min over
environments of a batch, or the single count), the step's wall time, the
simulated-seconds per wall-second of the step and of the run so far (per
environment for a batch: environment-seconds), and the vertex updates per
second (solved vertices x sweeps / wall time).
"""
import json

import numpy as np


class StepLog:
    def __init__(self, path_or_file, n_solved, dt, n_env=1):
        """`n_solved`: solved vertices of every environment (an int for one
        mesh, or a sequence per environment); `dt`: the step length."""
        self._own = isinstance(path_or_file, str)
        self.f = open(path_or_file, "w") if self._own else path_or_file
        self.n_solved = np.atleast_1d(np.asarray(n_solved, np.float64))
        self.dt = float(dt)
        self.n_env = max(int(n_env), len(self.n_solved))
        self.step = 0
        self.wall = 0.0

    def record(self, sweeps, wall_s, **extra):
        it = np.atleast_1d(np.asarray(sweeps, np.float64))
        wall_s = float(wall_s)
        self.step += 1
        self.wall += wall_s
        solved = self.n_solved if self.n_solved.size == it.size else np.full(it.size,
                                                                              self.n_solved.sum())
        line = {"step": self.step, "sweeps_mean": float(it.mean()), "sweeps_max": int(it.max()),
                "sweeps_min": int(it.min()), "wall_ms": 1e3 * wall_s,
                "sim_s_per_wall_s": self.n_env * self.dt / wall_s if wall_s > 0 else None,
                "run_sim_s_per_wall_s": self.n_env * self.dt * self.step / self.wall
                if self.wall > 0 else None,
                "vertex_updates_per_s": float((solved * it).sum()) / wall_s if wall_s > 0
                else None}
        line.update(extra)
        self.f.write(json.dumps(line) + "\n")
        return line

    def close(self):
        if self._own:
            self.f.close()


def read(path):
    """The lines of a StepLog file as dicts."""
    with open(path) as f:
        return [json.loads(s) for s in f if s.strip()]


__all__ = ["StepLog", "read"]
