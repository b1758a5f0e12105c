"""Persistent mode (one cooperative launch per step; colours separated by
neighbour-scoped readiness, or by grid barriers) against the per-colour graph
mode and the FP64 oracle (GPU tests, through the C ABI)."""
import numpy as np
import pytest

from oracle import oracle
from warpvbd_b200 import scenes

pytestmark = pytest.mark.gpu


def _solver(s, mode, precision="mixed", **kw):
    from warpvbd_b200 import VBDSolver
    return VBDSolver(**s.solver_kwargs(), damping_coefficient=0.0, dx_tol=1e-7, max_iter=1000,
                     precision=precision, mode=mode, **kw)


def _diag(X):
    return float(np.linalg.norm(X.max(0) - X.min(0)))


@pytest.mark.parametrize("n,tpv,threads,precision,bound", [
    (20, 4, 256, "mixed", 1e-8), (40, 4, 256, "mixed", 1e-8), (80, 4, 256, "mixed", 1e-8),
    (80, 8, 512, "mixed", 1e-8), (160, 4, 256, "mixed", 1e-8), (160, 2, 512, "mixed", 1e-8),
    (40, 4, 256, "fp64", 1e-13), (80, 8, 512, "fp64", 1e-13)])
def test_persist_matches_graph_mode(n, tpv, threads, precision, bound):
    """Within a colour every vertex update reads only other colours, so the
    two schedules do the same arithmetic: sweep counts must agree exactly and
    positions to rounding.  The two kernels are compiled separately and the
    compiler may contract a multiply-add differently: one fp32 rounding of a
    position update is ~1e-11 m here, and 40 steps carry it to ~3e-10 of the
    diagonal (measured); in fp64 the same is ~1e-16."""
    s = scenes.cantilever(n)
    steps = 20 if n >= 160 else 40
    g = _solver(s, "graph", tpv=tpv, precision=precision)
    p = _solver(s, "persist", tpv=tpv, block_threads=threads, precision=precision)
    assert p.info()["mode"] == 0x400
    D = _diag(s.vertices)
    worst = 0.0
    for _ in range(steps):
        xg = g.step(g.old_positions, 1e-3).numpy()
        xp = p.step(p.old_positions, 1e-3).numpy()
        assert g.last_iterations == p.last_iterations
        worst = max(worst, np.abs(xg - xp).max() / D)
    print(f"persist vs graph, cantilever {n}, tpv {tpv}, {precision}: max diff {worst:.3e} "
          "of the diagonal")
    assert worst < bound, worst


@pytest.mark.parametrize("n,tpv,threads,order_index", [
    (40, 4, 128, False), (80, 16, 128, False), (160, 4, 128, True), (160, 8, 256, False)])
def test_neighbour_readiness_matches_grid_barriers(n, tpv, threads, order_index):
    """Waiting only for the neighbouring blocks between colours changes the
    schedule, not the arithmetic: every vertex still reads the latest values
    of lower colours and the previous sweep's of higher ones, so positions and
    sweep counts are bit-identical to the grid-barrier schedule."""
    s = scenes.cantilever(n)
    a = _solver(s, "persist", precision="fp64", tpv=tpv, block_threads=threads,
                order_index=order_index)
    b = _solver(s, "persist", precision="fp64", tpv=tpv, block_threads=threads,
                order_index=order_index, persist_sync="grid")
    assert a.info()["n_blocks"] > 1
    for _ in range(20 if n >= 160 else 40):
        xa = a.step(a.old_positions, 1e-3).numpy()
        xb = b.step(b.old_positions, 1e-3).numpy()
        assert a.last_iterations == b.last_iterations
        assert np.array_equal(xa, xb)


@pytest.mark.parametrize("n", [40, 80])
def test_persist_fp64_matches_oracle(n):
    s = scenes.cantilever(n)
    p = _solver(s, "persist", precision="fp64")
    orc = oracle.OracleSolver(**s.solver_kwargs(), damping_coefficient=0.0, dx_tol=1e-7,
                              max_iter=1000, guarded=True)
    D = _diag(s.vertices)
    for _ in range(15):
        xp = p.step(p.old_positions, 1e-3).numpy()
        xo = orc.step(None, 1e-3)
        assert p.last_iterations == orc.last_iterations
        assert np.abs(xp - xo).max() / D < 1e-9


def test_persist_mass_spring_matches_oracle():
    s = scenes.mass_spring(11, 20)
    p = _solver(s, "persist")
    orc = oracle.OracleSolver(**s.solver_kwargs(), damping_coefficient=0.0, dx_tol=1e-7,
                              max_iter=1000, guarded=True)
    D = _diag(s.vertices)
    for _ in range(60):
        xp = p.step(p.old_positions, 1e-3).numpy()
        xo = orc.step(None, 1e-3)
    assert np.abs(xp - xo).max() / D < 1e-5


def test_persist_max_iter_and_warning(capsys):
    s = scenes.cantilever(40)
    p = _solver(s, "persist")
    p.step(p.old_positions, 1e-3, max_iter=3)
    assert p.last_iterations == 3
    assert "did not converge" in capsys.readouterr().out


def test_expired_barrier_wait_reports_timeout_and_the_solver_recovers():
    """Every grid-barrier wait is bounded.  With a limit of zero polls the
    first block to arrive at a barrier gives up at once: the step must fail
    with VBD_ERR_TIMEOUT (no hang), and after restoring the limits and the
    state the solver must step exactly like a fresh one."""
    from warpvbd_b200 import _lib
    s = scenes.cantilever(80)
    p = _solver(s, "persist")
    L = _lib.load()
    assert L.vbd_set_wait_limits(p._h, 0, 0) == 0
    with pytest.raises(_lib.VBDError) as ei:
        for _ in range(3):
            p.step(p.old_positions, 1e-3)
    assert ei.value.status == _lib.ERR_TIMEOUT
    assert L.vbd_set_wait_limits(p._h, 1 << 26, 2_000_000_000) == 0
    p.reset()
    q = _solver(s, "persist")
    for _ in range(5):
        xp = p.step(p.old_positions, 1e-3).numpy()
        xq = q.step(q.old_positions, 1e-3).numpy()
        assert np.array_equal(xp, xq)
