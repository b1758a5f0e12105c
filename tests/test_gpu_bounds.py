"""The bounds-checked build (libvbd_b200_check.so: every slot's neighbour and
record ids checked against its environment before use, an id out of range
reported as VBD_ERR_BOUNDS) runs the same steps as the regular build: same
positions bit for bit, same sweep counts, no bounds error -- in block mode
(tiered batch, with the learned warm start), persistent mode and graph mode.
Stands in for compute-sanitizer, which is not available here.  The checked
library runs in a child process (WARPVBD_B200_LIB selects it)."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CHECK_LIB = os.path.join(ROOT, "warpvbd_b200", "libvbd_b200_check.so")

SCRIPT = r"""
import json, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
from warpvbd_b200 import BatchedVBDSolver, VBDSolver, scenes, warmstart
out = {}
envs = scenes.env_batch(12, seed=3)
b = BatchedVBDSolver(envs, dx_tol=1e-7, max_iter=1000, cluster=4, tiered=True)
its = [b.step(1e-3).tolist() for _ in range(4)]
b.set_warmstart(warmstart.load())
its += [b.step(1e-3).tolist() for _ in range(3)]
out["batch"] = {"iters": its, "x": b.positions().tolist(), "status": b.last_status}
for mode in ("persist", "graph"):
    s = scenes.cantilever(40)
    v = VBDSolver(**s.solver_kwargs(), damping_coefficient=0.0, dx_tol=1e-7, max_iter=1000,
                  mode=mode)
    it = []
    for _ in range(4):
        x = v.step(v.old_positions, 1e-3).numpy()
        it.append(int(v.last_iterations))
    out[mode] = {"iters": it, "x": x.tolist(), "status": v.last_status}
print(json.dumps(out))
"""


def _run(lib):
    env = dict(os.environ)
    if lib:
        env["WARPVBD_B200_LIB"] = lib
    else:
        env.pop("WARPVBD_B200_LIB", None)
    r = subprocess.run([sys.executable, "-c", SCRIPT, ROOT], env=env, capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    return json.loads(r.stdout.strip().splitlines()[-1])


def test_checked_build_matches_regular_build():
    if not os.path.exists(CHECK_LIB):
        pytest.fail(f"bounds-checked library missing: {CHECK_LIB} (make -C warpvbd_b200/csrc check)")
    ref, chk = _run(None), _run(CHECK_LIB)
    for key in ("batch", "persist", "graph"):
        assert chk[key]["status"] == 0, (key, chk[key]["status"])
        assert chk[key]["iters"] == ref[key]["iters"], key
        assert np.array_equal(np.array(chk[key]["x"]), np.array(ref[key]["x"])), key
