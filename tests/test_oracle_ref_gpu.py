"""The oracle against the reference's own GPU step (golden states).

tests/golden/ref_gpu_step.npz holds particle states written by the reference's
leap_frog::step (src/leap_frog.cu:121-195), built for sm_100a from its sources
(baseline/build_ref_gpu.sh) and run on small seeded scenes
(tests/golden/make_ref_gpu_golden.py): after 1 and 20 steps from rest and after
1 step from a loaded state (tests/helpers.py ``loaded``: random stress,
velocities, temperatures and densities, so that every term of the step, the
artificial-stress rotation, the Jaumann rate and the CSPM correction included,
is exercised).  The oracle runs on the CPU here.

* Its FP32 form restates the reference's FP32 build: from rest the first step
  (contact forces of the initial configuration) is bitwise equal, and after one
  loaded step or 20 steps every field agrees to the last bits that the
  reference's compiler changes by fusing multiply-adds (relative L2 <= 1e-5).
* Its FP64 form is within FP32 rounding of the reference's FP32 state.

Tolerances are relative L2 per field (positions as displacements, temperature
as T - T0), about three times the measured values (floor 1e-7).
"""
import os
import sys

import numpy as np
import pytest

import oracle

from helpers import compare, loaded, oracle_state

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import make_ref_gpu_golden as G  # noqa: E402

GOLD = os.path.join(HERE, "golden", "ref_gpu_step.npz")
NAMES = [f for f in G.FIELDS if f != "BLANKED"]

ALL0 = {f: 0.0 for f in NAMES}
TOL = {
    # (tag, precision): per-field bound, "force" for the summed tool force
    ("1", 32): dict(ALL0, force=1e-6),
    ("1", 64): dict(ALL0, FC=3e-5, force=3e-5),
    ("20", 32): dict(POS=4.5e-6, VEL=3.3e-6, S=4.2e-6, RHO=3.3e-8, T=2.8e-6, EPS_PL=1e-6, FC=1e-7, FT=3.4e-6,
                     POS_T=2.8e-6, VEL_T=2.6e-6, S_T=7.2e-6, RHO_T=6.3e-6, T_T=1e-5, R=4e-6, force=1e-3),
    ("20", 64): dict(POS=9e-5, VEL=9e-5, S=4.5e-5, RHO=4e-7, T=6e-5, EPS_PL=2.3e-5, FC=1.8e-4, FT=5.1e-3,
                     POS_T=6.3e-5, VEL_T=6e-5, S_T=1.6e-4, RHO_T=1.4e-4, T_T=1.2e-4, R=1.7e-4, force=4e-4),
    ("loaded", 32): dict({f: 1e-6 for f in NAMES}, force=1e-6),
    ("loaded", 64): dict({f: 2e-6 for f in NAMES}, POS=1.5e-3, FC=3.3e-5, force=3e-5),
}


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLD)


@pytest.mark.parametrize("prec", [32, 64])
@pytest.mark.parametrize("tag", ["1", "20", "loaded"])
@pytest.mark.parametrize("name", ["brookshaw", "cspm_pse"])
def test_oracle_matches_the_reference_gpu_step(oracle_lib, gold, name, tag, prec):
    sc = G.golden_scenes()[name]
    if tag == "loaded":
        sc = loaded(sc)
    steps = 20 if tag == "20" else 1
    orc = oracle.Oracle(sc, prec=prec)
    if tag == "loaded":
        orc.set_field("S", sc.S0)
    for k in range(steps):
        orc.step(record=(k == steps - 1))
    ref = {f: gold[f"{name}_{tag}_{f}"].astype(np.float64) for f in G.FIELDS}
    err = compare(oracle_state(orc, NAMES), ref, sc, NAMES)
    assert err["blank_mismatch"] == 0, err
    tol = TOL[(tag, prec)]
    for f in NAMES:
        assert err[f] <= tol[f], (name, tag, prec, f, err[f], tol[f])
    fr = gold[f"{name}_{tag}_TOOL_FORCES"].astype(np.float64)
    fo = orc.tool_forces().astype(np.float64)
    assert np.linalg.norm(fo - fr) <= tol["force"] * np.linalg.norm(fr), (fo, fr)
