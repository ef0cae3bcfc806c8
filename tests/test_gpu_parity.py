"""Parity of the CUDA step (through the C ABI) with the CPU oracle.

Bit-exact: cell ids, the stable sort permutation, cell ranges and neighbour
counts, every step.  Floating point: per-field relative L2 against the FP64
oracle (positions as displacements, temperature as T - T0) with the
tolerances written in each test.
"""
import numpy as np
import pytest

import oracle
from iwf_mfree_gpu_3d_b200 import api, scenes

from helpers import by_id, grain_checks, check, compare, gpu_state, oracle_state

pytestmark = pytest.mark.gpu


def _sim(scene, **opt):
    return api.Simulation.from_scene(scene, **opt)


def test_integer_pipeline_bit_exact_every_step():
    sc = scenes.small_scene()
    sim = _sim(sc, diagnostics=1)
    (nx, ny, nz), bbmin, dx = sim.grid()
    ncell = nx * ny * nz
    for step in range(30):
        pos_before = sim.get("POS")
        sim.step()
        idx = sim.get("IDX")
        hsh = sim.get("HASH")
        blanked_after = sim.get("BLANKED")
        n_act, n_init = sim.counts()
        blanked_at_hash = np.empty_like(blanked_after)
        blanked_at_hash[idx] = blanked_after
        h_ref = oracle.hash_fp32(pos_before, blanked_at_hash, np.array(bbmin, np.float32), dx, (nx, ny, nz))
        idx_ref, sh_ref, cs_ref, ce_ref = oracle.sort_cells(h_ref, n_act, ncell)
        assert n_act == int((h_ref != np.iinfo(np.int32).max).sum())
        np.testing.assert_array_equal(idx, idx_ref)
        np.testing.assert_array_equal(hsh, sh_ref)
        cs, ce = sim.cells()
        np.testing.assert_array_equal(cs, cs_ref)
        np.testing.assert_array_equal(ce, ce_ref)
        nnb_ref = oracle.neighbor_counts_fp32(sim.get("POS_HALF"), sim.get("H"), hsh, cs, ce, n_act, (nx, ny, nz))
        np.testing.assert_array_equal(sim.get("NUM_NBH")[:n_act], nnb_ref)
    sim.close()


def test_integer_pipeline_bit_exact_full_size_1m():
    """The 1,000,000-particle configuration (CSPM + PSE): cell ids, the stable
    sort, cell ranges and neighbour counts bit-exact with the oracle's FP32
    pipeline for 3 steps, at full size."""
    sc = scenes.million_scene()
    sim = _sim(sc, diagnostics=1)
    (nx, ny, nz), bbmin, dx = sim.grid()
    ncell = nx * ny * nz
    for step in range(3):
        pos_before = sim.get("POS")
        sim.step()
        idx = sim.get("IDX")
        n_act, n_init = sim.counts()
        blanked_after = sim.get("BLANKED")
        blanked_at_hash = np.empty_like(blanked_after)
        blanked_at_hash[idx] = blanked_after
        h_ref = oracle.hash_fp32(pos_before, blanked_at_hash, np.array(bbmin, np.float32), dx, (nx, ny, nz))
        idx_ref, sh_ref, cs_ref, ce_ref = oracle.sort_cells(h_ref, n_act, ncell)
        np.testing.assert_array_equal(idx, idx_ref)
        hsh = sim.get("HASH")
        np.testing.assert_array_equal(hsh, sh_ref)
        cs, ce = sim.cells()
        np.testing.assert_array_equal(cs, cs_ref)
        np.testing.assert_array_equal(ce, ce_ref)
        nnb_ref = oracle.neighbor_counts_fp32(sim.get("POS_HALF"), sim.get("H"), hsh, cs, ce, n_act, (nx, ny, nz))
        np.testing.assert_array_equal(sim.get("NUM_NBH")[:n_act], nnb_ref)
    sim.close()


def test_three_steps_against_fp64_oracle_full_size_1m():
    """The 1,000,000-particle configuration against the FP64 oracle (OpenMP on
    the host cores) after 3 steps, with the tolerances of the 100-step test."""
    sc = scenes.million_scene()
    sim = _sim(sc)
    orc = oracle.Oracle(sc, prec=64)
    for _ in range(3):
        sim.step()
        orc.step()
    err = compare(gpu_state(sim), oracle_state(orc), sc)
    print("1M, 3-step relative L2 (FP32 CUDA vs FP64 oracle):", err)
    check(err, "1m_3")
    sim.close()


def test_100_steps_against_fp64_oracle_full_size_1m_plain_and_precision():
    """The 1,000,000-particle configuration (CSPM, artificial stress, PSE)
    after 100 steps, run once in plain FP32 and once in the precision form
    (compensated hi/lo positions and velocities), each against one FP64
    oracle run: the per-field relative L2 error of both is printed, both stay
    within its tolerances, and the precision form's displacement error is at
    most a tenth of plain FP32's (measured: 0.019)."""
    sc = scenes.million_scene()
    plain = _sim(sc)
    prec = _sim(sc, precision=1)
    orc = oracle.Oracle(sc, prec=64)
    for _ in range(100):
        plain.step()
        prec.step()
        orc.step()
    o = oracle_state(orc)
    e_plain = compare(gpu_state(plain), o, sc)
    e_prec = compare(gpu_state(prec, f64=True), o, sc)
    for name, err in (("plain FP32", e_plain), ("precision form", e_prec)):
        print(f"1M, 100-step relative L2 vs FP64 oracle, {name}: " +
              ", ".join(f"{k} {v:.3e}" for k, v in err.items()))
    check(e_plain, "1m_100")
    check(e_prec, "1m_100_prec")
    assert e_prec["POS"] <= 0.1 * e_plain["POS"]
    plain.close()
    prec.close()


def test_single_grain_full_size_against_fp64_oracle():
    """The single-grain configuration at full size: a 400 x 160 x 64 block
    (4,096,000 particles) plus the grain's diamond tool particles, cut by the
    1,280-triangle truncated icosphere at 30 m/s from the first step, 10 steps.
    The compensated form (the configuration's form) against the FP64 oracle:
    its per-field report is printed and is no larger than the reference's own
    GPU step's; the plain FP32 form against the reference's GPU step."""
    sc = scenes.single_grain()
    sim = _sim(sc)
    orc = oracle.Oracle(sc, prec=64)
    for _ in range(10):
        sim.step()
        orc.step()
    o = oracle_state(orc)
    err = compare(gpu_state(sim, f64=True), o, sc)
    sim.close()
    print("single grain, 4.1M particles, 10-step relative L2 vs FP64 oracle: " +
          ", ".join(f"{k} {v:.3e}" for k, v in err.items()))
    sc0 = scenes.single_grain(precision=0)
    plain = _sim(sc0)
    for _ in range(10):
        plain.step()
    grain_checks(sc0, plain, err, o, 10, "grain_40")
    plain.close()


def test_one_step_against_fp32_oracle():
    """One step from the same input: the CUDA path against the oracle in the
    reference's FP32 semantics.  Differences come from summation order,
    FMA contraction and device math functions only."""
    sc = scenes.small_scene()
    sim = _sim(sc)
    orc = oracle.Oracle(sc, prec=32)
    sim.step()
    orc.step()
    err = compare(gpu_state(sim), oracle_state(orc), sc)
    assert err["blank_mismatch"] == 0
    for k in ("POS", "VEL", "RHO", "VEL_T", "POS_T", "RHO_T"):
        assert err[k] < 2e-5, (k, err)
    sim.close()


def test_100_steps_against_fp64_oracle_8k():
    """8,000 particles, Brookshaw, artificial stress, Johnson-Cook, contact:
    per-field relative L2 after 100 steps against the FP64 oracle."""
    sc = scenes.small_scene()
    sim = _sim(sc)
    orc = oracle.Oracle(sc, prec=64)
    for k in range(100):
        sim.step()
        orc.step()
    err = compare(gpu_state(sim), oracle_state(orc), sc)
    print("100-step relative L2 (FP32 CUDA vs FP64 oracle):", err)
    check(err, "8k_100")
    sim.close()


def test_1000_steps_small_configuration():
    """The small configuration as stated: 1000 steps of the 8,000-particle
    scene against the FP64 oracle.  Over that many steps of contact every FP32
    trajectory parts from FP64 about as far as the reference's own GPU step
    does, and how far depends on last bits (a rounding-level change of the
    pair arithmetic moved the velocity error between 3.2e-3 and 4.7e-3, the
    reference's being 3.1e-3), so where that build is at hand the CUDA path's
    error may be at most twice the reference's, field by field; elsewhere the
    bounds of 8k_1000."""
    sc = scenes.small_scene()
    sim = _sim(sc)
    orc = oracle.Oracle(sc, prec=64)
    for _ in range(1000):
        sim.step()
        orc.step()
    o = oracle_state(orc)
    err = compare(gpu_state(sim), o, sc)
    sim.close()
    print("1000-step relative L2 (FP32 CUDA vs FP64 oracle):", {k: f"{v:.2e}" for k, v in err.items()})
    assert err["blank_mismatch"] == 0
    from baseline import refgpu
    if not refgpu.available(refgpu.variant_of(sc)):
        check(err, "8k_1000")
        return
    names = ["POS", "VEL", "S", "EPS_PL", "T", "RHO"]
    st = refgpu.run(sc, 0, 1000, state=True)["state"]
    r = {n: by_id(st["ID"], st[n].astype(np.float64)) for n in names + ["BLANKED"]}
    e_ref = compare(r, o, sc, names)
    print("reference GPU step vs FP64 oracle:", {k: f"{v:.2e}" for k, v in e_ref.items()})
    for f in names:
        assert err[f] <= 2.0 * e_ref[f] + 1e-7, (f, err[f], e_ref[f])


def test_graph_replay_equals_eager_steps():
    sc = scenes.small_scene()
    a = _sim(sc)
    b = _sim(sc)
    for _ in range(12):
        a.step()
    b.advance(12, use_graph=True)
    b.sync()
    for name in ("POS", "VEL", "S", "T", "EPS_PL", "ID"):
        np.testing.assert_array_equal(a.get(name), b.get(name))
    assert a.time() == b.time()
    a.close()
    b.close()


@pytest.mark.parametrize("lpp", [8, 16, 32])
def test_lanes_per_particle_variants_agree(lpp):
    sc = scenes.small_scene()
    ref = _sim(sc, lanes_per_particle=8)
    sim = _sim(sc, lanes_per_particle=lpp)
    for _ in range(5):
        ref.step()
        sim.step()
    ga, gb = gpu_state(sim), gpu_state(ref)
    err = compare(ga, gb, sc)
    for k in ("POS", "VEL", "S", "T"):
        assert err[k] < 1e-4, (k, err)
    ref.close()
    sim.close()


def test_tool_setup_matches_oracle_fp32():
    sc = scenes.small_scene()
    sim = _sim(sc)
    orc = oracle.Oracle(sc, prec=32)
    gi, oi = sim.tool_info(0), orc.tool_info(0)
    assert gi["n3"] == oi["n3"] and gi["num_boxed"] == oi["num_boxed"] and gi["num_tris"] == oi["num_tris"]
    np.testing.assert_array_equal(np.float32(gi["bbmin"]), np.float32(oi["bbmin"]))
    np.testing.assert_array_equal(np.float32(gi["dx"]), np.float32(oi["dx"]))
    np.testing.assert_array_equal(sim.tool_normals(0), orc.tool_normals(0).astype(np.float32))
    gc, gs = sim.tool_cells(0)
    oc, os_ = orc.tool_cells(0)
    np.testing.assert_array_equal(gc, oc)
    np.testing.assert_array_equal(gs, os_)
    sim.close()
