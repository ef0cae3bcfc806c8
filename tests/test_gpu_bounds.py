"""The bounds-checked debug build (libmfree_checked.so, -DMFREE_BOUNDS_CHECK):
every index the kernels compute from data -- sort destinations, cell ranges,
the pair kernel's cell starts, halo staging ranges, target and candidate
records, the contact triangle ranges --
is tested against its array and counted when outside, instead of being used.
Small cases of every kernel variant (and a dense scene whose tiles read their
records from global memory) run through it in a process of their own
(the library is loaded once per process): no index may fall outside, and the
physics must still match the FP64 oracle.  This stands in for a memory checker,
which is not available on the GPU machines."""
import json
import os
import subprocess
import sys

import pytest

from helpers import TOL

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SCRIPT = r"""
import json, os, sys
sys.path.insert(0, os.environ["MFREE_ROOT"])
sys.path.insert(0, os.path.join(os.environ["MFREE_ROOT"], "tests"))
import oracle
from iwf_mfree_gpu_3d_b200 import api, build, scenes
from helpers import compare, gpu_state, oracle_state
L = api.lib(build.LIB_CHECKED)
out = {"checked": int(L.mfree_bounds_checked()), "cases": {}}
cases = {
    "brookshaw_8k": (scenes.small_scene(), {}),
    "cspm_pse_precision": (scenes.orthogonal_cutting(30, 15, 12, cspm=True, conduction=2), {"precision": 1}),
    "exhaustive_contact": (scenes.orthogonal_cutting(24, 12, 10, algorithm=1), {}),
    "full_stencil_32_lanes": (scenes.orthogonal_cutting(24, 12, 10), {"full_stencil": 1, "lanes_per_particle": 32}),
}
for name, (sc, opt) in cases.items():
    sim = api.Simulation.from_scene(sc, **opt)
    orc = oracle.Oracle(sc, prec=64)
    for _ in range(30):
        sim.step()
        orc.step()
    err = compare(gpu_state(sim, f64=bool(opt.get("precision"))), oracle_state(orc), sc)
    out["cases"][name] = {"bounds_errors": sim.counters()["bounds_errors"],
                          "err": {k: float(err[k]) for k in ("POS", "VEL", "S", "T", "RHO")},
                          "blank_mismatch": int(err["blank_mismatch"])}
    sim.close()
b = api.Batch()
sims = [api.Simulation.from_scene(scenes.mixed_scene(sp)) for sp in scenes.mixed_specs(3, seed=5, n_lo=2000, n_hi=6000)]
for s in sims:
    b.admit(s)
b.step(10)
b.sync()
out["cases"]["batch"] = {"bounds_errors": sum(s.counters()["bounds_errors"] for s in sims)}
b.close()
# a dense scene (h = 2.2 dx): tiles read their records from global memory
# and targets overflow their neighbour queue
sim = api.Simulation.from_scene(scenes.orthogonal_cutting(30, 20, 16, hdx=2.2, cspm=True, conduction=2))
for _ in range(3):
    sim.step()
out["cases"]["dense_global_records"] = {"bounds_errors": sim.counters()["bounds_errors"]}
sim.close()
print(json.dumps(out))
"""


def test_bounds_checked_build_finds_no_index_outside_its_array():
    lib = os.path.join(ROOT, "iwf_mfree_gpu_3d_b200", "libmfree_checked.so")
    assert os.path.exists(lib), "build libmfree_checked.so first (python -m iwf_mfree_gpu_3d_b200.build --checked)"
    env = dict(os.environ, MFREE_ROOT=ROOT)
    r = subprocess.run([sys.executable, "-c", SCRIPT], env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    out = json.loads(r.stdout.strip().splitlines()[-1])
    print(json.dumps(out, indent=1))
    assert out["checked"] == 1
    for name, case in out["cases"].items():
        assert case["bounds_errors"] == 0, (name, case)
        if "err" in case:
            assert case["blank_mismatch"] == 0, (name, case)
            for k, v in case["err"].items():
                assert v < TOL["bounds_30"][k], (name, k, case)
