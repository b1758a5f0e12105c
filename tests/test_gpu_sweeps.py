"""The accuracy / scaling sweeps (warpvbd_b200.sweeps) on small cases (GPU):
every row runs the FP64 solver and the mixed-precision one side by side, and
the identical-systems batch keeps its throughput as the count grows."""
import pytest

from warpvbd_b200 import sweeps

pytestmark = pytest.mark.gpu


def test_resolution_rows_time_both_precisions():
    res = sweeps.resolution(sizes=(20,), materials=("snh", "stvk"), steps=20)
    for key, r in res.items():
        assert r["fp64_sim_s_per_wall_s"] > 0 and r["sim_s_per_wall_s"] > 0, key
        assert r["fp64_mode"] == r["mode"] == "block", key
        assert r["max_vertex_error_of_diag"] < 1e-5, (key, r["max_vertex_error_of_diag"])


def test_identical_systems_scale():
    """16 copies of the mass-spring system take about as long per step as 4
    (the device is far from full); the planner once put all 16 on clusters
    of 8 that could not all be resident, which doubled the step."""
    res = sweeps.nsim(counts=(4, 16), steps=10, warmup=3)
    r4, r16 = res["4"], res["16"]
    print(f"4 systems {r4['ms_per_step']:.3f} ms, 16 systems {r16['ms_per_step']:.3f} ms")
    assert r16["ms_per_step"] < 1.6 * r4["ms_per_step"]
