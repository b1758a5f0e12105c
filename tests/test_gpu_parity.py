"""CUDA solver against the FP64 oracle (GPU tests, through the C ABI).

Tolerances (fp32 solver vs FP64 oracle, same mesh / material / steps):
  * every vertex position within 1e-5 of the bounding-box diagonal;
  * tip-face mean displacement within 1e-5 relative (1e-4 for the shorter
    StVK / damping / batched runs is not needed: the same 1e-5 is used);
  * the FP64 device build within 1e-9 of the diagonal.
"""
import numpy as np
import pytest

from oracle import oracle
from warpvbd_b200 import scenes

pytestmark = pytest.mark.gpu

POS_TOL = 1e-5     # x bbox diagonal
TIP_TOL = 1e-5     # relative


def _diag(X):
    return float(np.linalg.norm(X.max(0) - X.min(0)))


def _tip_disp(x, s):
    return (x[s.tip] - s.vertices[s.tip]).mean(axis=0)


def run_pair(s, steps, material="snh", kd=0.0, precision="mixed", mode="auto", tol=1e-7,
             max_iter=1000, dt=1e-3, **kw):
    from warpvbd_b200 import VBDSolver
    gpu = VBDSolver(**s.solver_kwargs(), damping_coefficient=kd, dx_tol=tol, max_iter=max_iter,
                    material=material, precision=precision, mode=mode, **kw)
    orc = oracle.OracleSolver(**s.solver_kwargs(), damping_coefficient=kd, dx_tol=tol,
                              max_iter=max_iter, material=material, guarded=True)
    its_g, its_o, worst = [], [], 0.0
    D = _diag(s.vertices)
    for k in range(steps):
        xg = gpu.step(gpu.old_positions, dt).numpy()
        xo = orc.step(None, dt)
        its_g.append(gpu.last_iterations)
        its_o.append(orc.last_iterations)
        worst = max(worst, np.abs(xg - xo).max() / D)
    return gpu, orc, xg, xo, np.array(its_g), np.array(its_o), worst


@pytest.mark.parametrize("mode", ["block", "graph", "hostloop", "persist"])
def test_cantilever_20x2x2_300_steps(mode):
    s = scenes.cantilever(20)
    steps = 300 if mode != "hostloop" else 60
    gpu, orc, xg, xo, ig, io, worst = run_pair(s, steps, mode=mode)
    assert gpu.info()["mode"] == {"block": 0x100, "graph": 0x200, "hostloop": 0x300,
                                  "persist": 0x400}[mode]
    assert worst < POS_TOL, worst
    dg, do = _tip_disp(xg, s), _tip_disp(xo, s)
    rel = np.linalg.norm(dg - do) / np.linalg.norm(do)
    assert rel < TIP_TOL, (rel, dg, do)
    assert np.abs(ig - io).max() <= 2, (ig, io)
    assert np.array_equal(xg[~s.active], s.vertices[~s.active])


def test_pure_fp32_state_drift_is_bounded():
    """All-fp32 state: the displacement's own rounding (ulp 6e-8 m at 0.5 m)
    feeds the Newton step, so the trajectory drifts further from FP64 than the
    default mixed mode; bounded at 1e-4 of the diagonal over 300 steps."""
    s = scenes.cantilever(20)
    gpu, orc, xg, xo, ig, io, worst = run_pair(s, 300, precision="fp32", mode="block")
    assert worst < 1e-4, worst


def test_fp64_device_build_matches_oracle_tightly():
    s = scenes.cantilever(20)
    gpu, orc, xg, xo, ig, io, worst = run_pair(s, 100, precision="fp64", mode="block")
    assert worst < 1e-9, worst
    assert np.array_equal(ig, io)


def test_fp64_graph_mode():
    s = scenes.cantilever(40)
    gpu, orc, xg, xo, ig, io, worst = run_pair(s, 20, precision="fp64", mode="graph")
    assert worst < 1e-9, worst
    assert np.array_equal(ig, io)


@pytest.mark.parametrize("mode", ["block", "persist", "graph"])
def test_stvk_cantilever(mode):
    s = scenes.cantilever(20)
    gpu, orc, xg, xo, ig, io, worst = run_pair(s, 100, material="stvk", mode=mode)
    assert worst < POS_TOL, worst
    assert orc.guard_hits == 0
    assert np.abs(ig - io).max() <= 2


@pytest.mark.parametrize("mode", ["block", "persist", "graph"])
def test_reference_default_damping(mode):
    s = scenes.cantilever(20)
    gpu, orc, xg, xo, ig, io, worst = run_pair(s, 100, kd=1.0, mode=mode)
    assert worst < POS_TOL, worst


def test_mass_spring_11_20():
    s = scenes.mass_spring(11, 20)
    gpu, orc, xg, xo, ig, io, worst = run_pair(s, 100, mode="block")
    assert worst < POS_TOL, worst
    dg, do = _tip_disp(xg, s), _tip_disp(xo, s)
    assert np.linalg.norm(dg - do) / np.linalg.norm(do) < TIP_TOL


def test_cantilever_40_graph_vs_block_vs_oracle():
    s = scenes.cantilever(40)
    _, _, xg, xo, ig, io, worst = run_pair(s, 30, mode="graph")
    assert worst < POS_TOL, worst
    _, _, xb, _, ib, _, worst_b = run_pair(s, 30, mode="block")
    assert worst_b < POS_TOL, worst_b


def test_batched_uneven_envs_match_per_env_oracle():
    from warpvbd_b200 import BatchedVBDSolver
    envs = scenes.env_batch(5, seed=11)
    b = BatchedVBDSolver(envs, dx_tol=1e-7, max_iter=1000)
    orcs = [oracle.OracleSolver(**e.solver_kwargs(), damping_coefficient=0.0, dx_tol=1e-7,
                                max_iter=1000, guarded=True) for e in envs]
    for k in range(30):
        its = b.step(1e-3)
        x = b.positions()
        for e, (env, o) in enumerate(zip(envs, orcs)):
            xo = o.step(None, 1e-3)
            xe = x[b.env_slice(e)]
            assert np.abs(xe - xo).max() / _diag(env.vertices) < POS_TOL
            assert abs(int(its[e]) - o.last_iterations) <= 2
    assert len(set(its.tolist())) >= 1


def test_batched_fp64_matches_oracle_tightly():
    """The FP64 build of the batched (tiered) solver against the FP64 oracle,
    environment by environment: within 1e-9 of the diagonal, same sweeps."""
    from warpvbd_b200 import BatchedVBDSolver
    envs = scenes.env_batch(6, seed=13)
    b = BatchedVBDSolver(envs, dx_tol=1e-7, max_iter=1000, precision="fp64", cluster=4,
                         tiered=True)
    orcs = [oracle.OracleSolver(**e.solver_kwargs(), damping_coefficient=0.0, dx_tol=1e-7,
                                max_iter=1000, guarded=True) for e in envs]
    for k in range(15):
        its = b.step(1e-3)
        x = b.positions()
        for e, (env, o) in enumerate(zip(envs, orcs)):
            xo = o.step(None, 1e-3)
            assert np.abs(x[b.env_slice(e)] - xo).max() / _diag(env.vertices) < 1e-9, (k, e)
            assert int(its[e]) == o.last_iterations, (k, e)


@pytest.mark.parametrize("cluster", [2, 3, 4, 5, 6, 8])
def test_single_env_split_over_a_cluster(cluster):
    """Block mode with the mesh replicated in every block of a cluster: each
    block updates its share of a colour and broadcasts it through distributed
    shared memory."""
    s = scenes.cantilever(40)
    gpu, orc, xg, xo, ig, io, worst = run_pair(s, 30, mode="block", cluster=cluster)
    inf = gpu.info()
    assert inf["cluster"] == cluster and inf["n_blocks"] == cluster
    assert worst < POS_TOL, worst
    assert np.abs(ig - io).max() <= 2, (ig, io)


def test_cluster_size_above_16_is_refused():
    """The Python front ends refuse a cluster size outside 0..16 before
    shifting it into the flags; the C ABI refuses 17..31 in the 5-bit field
    and any flag bit above it (a size of 32 or more, or a negative one)."""
    import ctypes
    from warpvbd_b200 import BatchedVBDSolver, _lib
    from warpvbd_b200._lib import VBDError
    envs = scenes.env_batch(2, seed=1)
    for c in (17, 32, 48, -1):
        with pytest.raises(ValueError, match="cluster must be"):
            BatchedVBDSolver(envs, cluster=c)
    s = envs[0]
    L = _lib.load()
    X, tets = _lib.f64(s.vertices), _lib.i32(s.tets)
    rho, E, nu = _lib.f64(s.density), _lib.f64(s.youngs), _lib.f64(s.poisson)
    base = _lib.MATERIAL_SNH | _lib.PRECISION_FP64 | _lib.MODE_BLOCK
    for bits in (17 << _lib.CLUSTER_SHIFT, 32 << _lib.CLUSTER_SHIFT, 1 << 28):
        h = ctypes.c_void_p()
        st = L.vbd_create(_lib.ptr(X, "d"), X.shape[0], _lib.ptr(tets, "i"), tets.shape[0],
                          _lib.ptr(rho, "d"), _lib.ptr(E, "d"), _lib.ptr(nu, "d"), None, 0.0,
                          None, None, base | bits, 0, 0, 0, ctypes.byref(h))
        assert st == _lib.ERR_INVALID_ARG, (bits, st)
        assert b"cluster size" in L.vbd_last_error_message()


def test_batched_heavy_environment_split():
    """A large soft environment among small stiff ones: after the first step
    the planner gives it a whole cluster; results match the oracle per
    environment and the unsplit run."""
    from warpvbd_b200 import BatchedVBDSolver
    envs = [scenes.mass_spring(15, 30, youngs=1e5, poisson=0.45)]
    envs += [scenes.mass_spring(7, 5, youngs=1e6) for _ in range(7)]
    split = BatchedVBDSolver(envs, dx_tol=1e-7, max_iter=1000, cluster=4)
    plain = BatchedVBDSolver(envs, dx_tol=1e-7, max_iter=1000, cluster=1)
    orcs = [oracle.OracleSolver(**e.solver_kwargs(), damping_coefficient=0.0, dx_tol=1e-7,
                                max_iter=1000, guarded=True) for e in envs]
    for k in range(15):
        its = split.step(1e-3)
        its_plain = plain.step(1e-3)
        x, xp = split.positions(), plain.positions()
        for e, (env, o) in enumerate(zip(envs, orcs)):
            xo = o.step(None, 1e-3)
            sl = split.env_slice(e)
            assert np.abs(x[sl] - xo).max() / _diag(env.vertices) < POS_TOL, (k, e)
            assert abs(int(its[e]) - o.last_iterations) <= 2
        assert np.abs(x - xp).max() < 1e-9
        assert np.array_equal(its, its_plain)
    assert split.info()["n_blocks"] > len(envs)   # the heavy environment was split


def test_step_api_semantics():
    from warpvbd_b200 import VBDSolver
    s = scenes.cantilever(20)
    sol = VBDSolver(**s.solver_kwargs(), damping_coefficient=0.0, dx_tol=1e-7, max_iter=1000)
    x1 = sol.step(sol.old_positions, 1e-3)
    a1 = x1.numpy()
    v1 = sol.old_velocities.numpy()
    assert np.allclose(v1, (a1 - s.vertices) / 1e-3, atol=1e-6)
    x2 = sol.step(sol.old_positions, 1e-3)
    with pytest.raises(RuntimeError):
        x1.numpy()                         # overwritten by the second step
    # stepping from an explicit host array uploads it
    sol.reset()
    assert np.allclose(sol.old_positions.numpy(), s.vertices)
    x = sol.step(a1, 1e-3).numpy()
    assert np.isfinite(x).all()
    # colour table in the reference layout
    col = oracle.graph_coloring(s.tets)
    table = sol.color_groups
    for c in range(table.shape[0]):
        assert np.array_equal(table[c][table[c] >= 0], np.nonzero(col == c)[0])
    assert sol.adj_v2e.shape == (189, 20)


def test_nonconvergence_warning_and_nonfinite(capsys):
    from warpvbd_b200 import VBDSolver
    s = scenes.cantilever(20)
    sol = VBDSolver(**s.solver_kwargs(), damping_coefficient=0.0, dx_tol=1e-7, max_iter=2)
    sol.step(sol.old_positions, 1e-3)
    assert sol.last_iterations == 2
    assert "did not converge" in capsys.readouterr().out
    bad = s.vertices.copy()
    bad[50] = np.nan
    with pytest.raises(FloatingPointError):
        sol.step(bad, 1e-3)


@pytest.mark.parametrize("cluster,threads", [(4, 256), (8, 128), (2, 512), (5, 512), (6, 256)])
def test_tiered_launch_is_bit_identical_to_one_launch(cluster, threads):
    """Heavy environments on clusters in one launch, the rest one block each
    in a concurrent second launch: every environment's arithmetic is the
    same as in the single launch, so positions and sweep counts must agree
    exactly, step after step (the plan is re-made from the sweep counts after
    every step, so environments move between the tiers)."""
    from warpvbd_b200 import BatchedVBDSolver
    envs = scenes.env_batch(24, seed=4)
    one = BatchedVBDSolver(envs, dx_tol=1e-7, max_iter=1000, cluster=cluster,
                           block_threads=threads)
    two = BatchedVBDSolver(envs, dx_tol=1e-7, max_iter=1000, cluster=cluster,
                           block_threads=threads, tiered=True)
    for _ in range(12):
        a = one.step(1e-3)
        b = two.step(1e-3)
        assert np.array_equal(a, b)
    assert np.array_equal(one.positions(), two.positions())
    assert np.array_equal(one.velocities(), two.velocities())


def test_step_timeline():
    """The traced tiered step computes the same as the untraced one, and its
    timeline holds every block once: each environment with its sweep count,
    split environments on `cluster` blocks of the split launch or on
    2 x `cluster` blocks of the wide tier."""
    from warpvbd_b200 import BatchedVBDSolver
    envs = scenes.env_batch(24, seed=4)
    kw = dict(dx_tol=1e-7, max_iter=1000, cluster=4, block_threads=256, tiered=True)
    ref, traced = BatchedVBDSolver(envs, **kw), BatchedVBDSolver(envs, **kw)
    traced.set_trace(True)
    for _ in range(4):
        a = ref.step(1e-3)
        b = traced.step(1e-3)
        assert np.array_equal(a, b)
        tl = traced.timeline()
        assert np.all(tl["end_ns"] >= tl["start_ns"]) and tl["start_ns"].min() == 0
        assert sorted(set(tl["env"].tolist())) == list(range(len(envs)))
        for e in range(len(envs)):
            rows = tl["env"] == e
            assert np.all(tl["sweeps"][rows] == b[e])
            n = int(rows.sum())
            assert (n, set(tl["launch"][rows].tolist())) in ((1, {1}), (4, {0}), (8, {2}))
            assert sorted(tl["rank"][rows].tolist()) == list(range(n))
    assert np.array_equal(ref.positions(), traced.positions())
    traced.set_trace(False)
    traced.step(1e-3)
    assert len(traced.timeline()["env"]) == 0


@pytest.mark.parametrize("precision,tol", [("mixed", 1e-4), ("fp64", 1e-9)])
def test_incremental_potential_matches_oracle(precision, tol):
    """The potential the learned warm start compares (each tet's strain energy
    once from the tet list, plus the solved vertices' inertia energy), as
    differences between two candidate states, against the FP64 oracle's
    incremental potential: the two differ only by constants (the SNH
    energy's constant per tet and the inertia form's x-independent terms).
    Relative tolerance on the difference: 1e-4 with fp32 strain energies,
    1e-9 in FP64."""
    from warpvbd_b200 import BatchedVBDSolver
    envs = scenes.env_batch(3, seed=7)
    b = BatchedVBDSolver(envs, dx_tol=1e-7, max_iter=1000, precision=precision)
    for _ in range(3):
        b.step(1e-3)
    x, v = b.positions(), b.velocities()
    act = np.concatenate([e.active for e in envs])[:, None]
    rng = np.random.default_rng(1)
    xa = x + 2e-4 * rng.normal(size=x.shape) * act
    xb = x + 2e-4 * rng.normal(size=x.shape) * act
    ea, eb = b.incremental_potential(xa), b.incremental_potential(xb)
    for e, env in enumerate(envs):
        o = oracle.OracleSolver(**env.solver_kwargs(), damping_coefficient=0.0, dx_tol=1e-7,
                                max_iter=1000)
        sl = b.env_slice(e)
        o.set_state(x[sl], v[sl])
        d_o = o.incremental_potential(xa[sl], 1e-3) - o.incremental_potential(xb[sl], 1e-3)
        d_k = ea[e] - eb[e]
        print(f"{precision} env {e}: difference {d_k:.9e} vs oracle {d_o:.9e}")
        assert abs(d_k - d_o) <= tol * abs(d_o), (e, d_k, d_o)


@pytest.mark.parametrize("tiered,warm", [(False, False), (True, False), (True, True)])
def test_step_into_host_array(tiered, warm):
    """step(out=...) leaves the same positions as step() + positions():
    written by the step kernels into a page-locked array, copied after the
    step into a pageable one; sweep counts identical."""
    import torch
    from warpvbd_b200 import BatchedVBDSolver, warmstart
    envs = scenes.env_batch(10, seed=6)
    kw = dict(dx_tol=1e-7, max_iter=1000, cluster=4, tiered=tiered)
    a, b = BatchedVBDSolver(envs, **kw), BatchedVBDSolver(envs, **kw)
    if warm:
        model = warmstart.load()
        a.set_warmstart(model)
        b.set_warmstart(model)
    n = a.n_vertices
    pinned = torch.empty((n, 3), dtype=torch.float64, pin_memory=True).numpy()
    pageable = np.empty((n, 3))
    for k in range(6):
        ia = a.step(1e-3)
        xa = a.positions()
        out = pinned if k % 2 == 0 else pageable
        out[:] = np.nan
        ib = b.step(1e-3, out=out)
        assert np.array_equal(ia, ib)
        assert np.array_equal(xa, out), k
    assert np.array_equal(a.velocities(), b.velocities())


def test_checkpoint_resume(tmp_path):
    """A run saved after 5 steps (io.save_state) and restored into a fresh
    solver continues as the uninterrupted run: the state is (x, v).  The
    checkpoint holds absolute positions, and the solver keeps displacements
    from rest, so the restored state differs by the rounding of x - X
    (~1e-18 m here), which the iteration carries along: same sweep counts,
    positions within 1e-9 m (measured 1.3e-11), far below the 1e-7 update
    tolerance."""
    from warpvbd_b200 import BatchedVBDSolver, io
    envs = scenes.env_batch(6, seed=8)
    a = BatchedVBDSolver(envs, dx_tol=1e-7, max_iter=1000)
    for _ in range(5):
        a.step(1e-3)
    io.save_state(tmp_path / "ck.npz", a.positions(), a.velocities(), step=5)
    b = BatchedVBDSolver(envs, dx_tol=1e-7, max_iter=1000)
    x, v, extra = io.load_state(tmp_path / "ck.npz")
    b.set_state(positions=x, velocities=v)
    assert int(extra["step"]) == 5
    for _ in range(5):
        assert np.array_equal(a.step(1e-3), b.step(1e-3))
    assert np.abs(a.positions() - b.positions()).max() < 1e-9


def test_checkpoint_resume_warm_started_batch(tmp_path):
    """The learned warm start also reads the previous step's inertia target,
    which a checkpoint of (x, v) does not hold: a warm-started batch restored
    into a fresh solver continues within the solver's tolerance of the
    uninterrupted run, not bit for bit (io.save_state's docstring)."""
    from warpvbd_b200 import BatchedVBDSolver, io, warmstart
    envs = scenes.env_batch(6, seed=8)
    model = warmstart.load()
    a = BatchedVBDSolver(envs, dx_tol=1e-7, max_iter=1000)
    a.set_warmstart(model)
    for _ in range(5):
        a.step(1e-3)
    io.save_state(tmp_path / "ck.npz", a.positions(), a.velocities(), step=5)
    b = BatchedVBDSolver(envs, dx_tol=1e-7, max_iter=1000)
    b.set_warmstart(model)
    x, v, _ = io.load_state(tmp_path / "ck.npz")
    b.set_state(positions=x, velocities=v)
    for _ in range(5):
        a.step(1e-3)
        b.step(1e-3)
    xa, xb = a.positions(), b.positions()
    worst = max(np.abs(xa[a.env_slice(e)] - xb[a.env_slice(e)]).max() / _diag(envs[e].vertices)
                for e in range(len(envs)))
    print(f"warm-started resume: largest difference {worst:.2e} of the diagonal")
    assert worst < 1e-4


def test_downloads_into_caller_arrays():
    """positions(out=...) / DeviceArray.numpy(out=...) fill a caller array
    (e.g. page-locked) with exactly what a fresh download returns."""
    import torch
    from warpvbd_b200 import BatchedVBDSolver, VBDSolver
    envs = scenes.env_batch(3, seed=2)
    b = BatchedVBDSolver(envs, dx_tol=1e-7, max_iter=1000)
    b.step(1e-3)
    n = b.n_vertices
    pinned = torch.empty((n, 3), dtype=torch.float64, pin_memory=True).numpy()
    assert b.positions(out=pinned) is pinned
    assert np.array_equal(pinned, b.positions())
    b.set_state(positions=pinned)
    assert np.array_equal(b.positions(), pinned)
    s = scenes.cantilever(20)
    v = VBDSolver(**s.solver_kwargs(), damping_coefficient=0.0, dx_tol=1e-7, max_iter=1000)
    x = torch.empty((s.n_vertices, 3), dtype=torch.float64, pin_memory=True).numpy()
    v.step(v.old_positions, 1e-3).numpy(out=x)
    assert np.array_equal(x, v.old_positions.numpy())
    with pytest.raises(ValueError):
        v.old_positions.numpy(out=np.empty((3, 3)))


def test_random_voxel_shapes_match_oracle():
    """Property test: random voxel shapes (up to 6 x 4 x 4, the x = 0 face
    fixed), random stiffness; the block-mode solver against the FP64 oracle
    for 20 steps, same per-vertex tolerance as the cantilever."""
    from hypothesis import HealthCheck, given, settings
    from hypothesis import strategies as st

    from warpvbd_b200 import VBDSolver, mesh

    @settings(max_examples=8, deadline=None, suppress_health_check=[HealthCheck.too_slow])
    @given(st.integers(2, 6), st.integers(1, 4), st.integers(1, 4),
           st.lists(st.booleans(), min_size=96, max_size=96), st.floats(1e5, 1e6))
    def check(nx, ny, nz, bits, youngs):
        vox = np.array(bits[:nx * ny * nz], bool).reshape(nx, ny, nz)
        vox[0] = True  # the fixed face and something attached to it
        vox[:, 0, 0] = True
        h = 0.02
        X, hexes = mesh.voxel2hex(vox, h, h, h)
        T = np.asarray(mesh.hex2tets(hexes), np.int32).reshape(-1, 4)
        n_t = T.shape[0]
        kw = dict(initial_positions=X, elements=T, densities=np.full(n_t, 1000.0),
                  youngs_modulus=np.full(n_t, youngs), poissons_ratio=np.full(n_t, 0.4),
                  active_mask=X[:, 0] > 1e-9)
        gpu = VBDSolver(**kw, damping_coefficient=0.0, dx_tol=1e-7, max_iter=1000, mode="block")
        orc = oracle.OracleSolver(**kw, damping_coefficient=0.0, dx_tol=1e-7, max_iter=1000,
                                  guarded=True)
        D = _diag(X)
        for _ in range(20):
            xg = gpu.step(gpu.old_positions, 1e-3).numpy()
            xo = orc.step(None, 1e-3)
            assert np.abs(xg - xo).max() / D < POS_TOL
            assert abs(gpu.last_iterations - orc.last_iterations) <= 2

    check()
