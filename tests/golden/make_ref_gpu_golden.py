"""Generate tests/golden/ref_gpu_step.npz from the reference's own GPU step.

The states come from baseline/_ref/ref_step_<variant>, the reference's
leap_frog::step (src/leap_frog.cu:121-195) built for sm_100a from its sources
by baseline/build_ref_gpu.sh, run on small seeded scenes (scenes.py):

  brookshaw  orthogonal_cutting(16, 8, 6): Brookshaw conduction, no CSPM
  cspm_pse   orthogonal_cutting(16, 8, 6, cspm=True, conduction=2)

For each scene the file holds the particle state after 1 step and after 20
steps from rest, and after 1 step from a loaded state (loaded(): a random
deviatoric stress of the order of the yield stress, random velocities,
temperatures and densities (tests/helpers.py), so that one step exercises
every term, the artificial stress and the Jaumann and CSPM algebra included),
in creation
order (fields in the reference's per-field layout, float32), with the tool
force of the last step.  Needs a GPU and the built comparator:
  python tests/golden/make_ref_gpu_golden.py [out.npz]
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

sys.path.insert(0, os.path.dirname(HERE))

from baseline import refgpu  # noqa: E402
from helpers import loaded  # noqa: E402
from iwf_mfree_gpu_3d_b200 import scenes  # noqa: E402

FIELDS = ("POS", "VEL", "S", "RHO", "T", "EPS_PL", "BLANKED", "FC", "FT", "POS_T", "VEL_T", "S_T", "RHO_T", "T_T",
          "R")
STEPS = (1, 20)


def golden_scenes():
    return {"brookshaw": scenes.orthogonal_cutting(16, 8, 6),
            "cspm_pse": scenes.orthogonal_cutting(16, 8, 6, cspm=True, conduction=2)}


def main():
    out = sys.argv[1] if len(sys.argv) > 1 else os.path.join(HERE, "ref_gpu_step.npz")
    data = {}
    runs = [(name, str(steps), sc, steps) for name, sc in golden_scenes().items() for steps in STEPS]
    runs += [(name, "loaded", loaded(sc), 1) for name, sc in golden_scenes().items()]
    for name, tag, sc, steps in runs:
        st = refgpu.run(sc, 0, steps, state=True)["state"]
        order = np.argsort(st["ID"], kind="stable")
        assert np.array_equal(st["ID"][order], np.arange(sc.n))
        for f in FIELDS:
            data[f"{name}_{tag}_{f}"] = st[f][order].astype(np.float32)
        data[f"{name}_{tag}_TOOL_FORCES"] = st["TOOL_FORCES"].astype(np.float32)
    np.savez_compressed(out, **data)
    print("wrote", out, sum(v.nbytes for v in data.values()), "bytes of arrays")


if __name__ == "__main__":
    main()
