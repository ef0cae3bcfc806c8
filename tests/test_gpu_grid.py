"""The unlocked cell grid (grid_gpu_green(max_cell, N), update_geometry's
unlocked branch, grid_gpu_base.cu:185-233): before every step the grid box
becomes the bounding box of the active particles and the cell edge their
largest h.  The grid of each step must be the reference's FP32 arithmetic on
the positions at the start of the step, the integer pipeline must stay
bit-exact on it, and the physics must match the FP64 oracle."""
import numpy as np
import pytest

import oracle
from iwf_mfree_gpu_3d_b200 import api, scenes

from helpers import check, compare, gpu_state, oracle_state, unlocked_grid

pytestmark = pytest.mark.gpu


def _scene(max_cell=400000):
    sc = scenes.small_scene()
    sc.grid_max_cell = max_cell
    return sc


def test_unlocked_grid_integer_pipeline_bit_exact_every_step():
    sc = _scene()
    sim = api.Simulation.from_scene(sc, diagnostics=1)
    for step in range(30):
        pos_before = sim.get("POS")
        h_before = sim.get("H")
        n_prev = sim.counts()[0]
        sim.step()
        (nx, ny, nz), bbmin, dx = sim.grid()
        n3, lo, edge = unlocked_grid(pos_before, h_before, n_prev)
        assert (nx, ny, nz) == n3, step
        np.testing.assert_array_equal(np.array(bbmin, np.float32), lo)
        assert np.float32(dx) == edge
        idx = sim.get("IDX")
        hsh = sim.get("HASH")
        blanked_after = sim.get("BLANKED")
        n_act, _ = sim.counts()
        blanked_at_hash = np.empty_like(blanked_after)
        blanked_at_hash[idx] = blanked_after
        h_ref = oracle.hash_fp32(pos_before, blanked_at_hash, lo, edge, n3)
        idx_ref, sh_ref, cs_ref, ce_ref = oracle.sort_cells(h_ref, n_act, nx * ny * nz)
        np.testing.assert_array_equal(idx, idx_ref)
        np.testing.assert_array_equal(hsh, sh_ref)
        cs, ce = sim.cells()
        np.testing.assert_array_equal(cs, cs_ref)
        np.testing.assert_array_equal(ce, ce_ref)
        nnb_ref = oracle.neighbor_counts_fp32(sim.get("POS_HALF"), sim.get("H"), hsh, cs, ce, n_act, n3)
        np.testing.assert_array_equal(sim.get("NUM_NBH")[:n_act], nnb_ref)
    sim.close()


def test_unlocked_grid_100_steps_against_fp64_oracle():
    sc = _scene()
    sim = api.Simulation.from_scene(sc)
    orc = oracle.Oracle(sc, prec=64)
    for _ in range(100):
        sim.step()
        orc.step()
    err = compare(gpu_state(sim), oracle_state(orc), sc)
    print("unlocked grid, 100-step relative L2 (FP32 CUDA vs FP64 oracle):", err)
    check(err, "8k_100")
    sim.close()


def test_unlocked_grid_advance_equals_single_steps():
    """mfree_advance on an unlocked grid (graph requested) steps eagerly and
    gives the same bits as single steps."""
    sc = _scene()
    a = api.Simulation.from_scene(sc)
    b = api.Simulation.from_scene(sc)
    a.advance(12, record_every=1, use_graph=True)
    for _ in range(12):
        b.step(record_forces=True)
    for name in ("POS", "VEL", "S", "T", "EPS_PL", "ID"):
        np.testing.assert_array_equal(a.get(name), b.get(name), err_msg=name)
    assert a.grid() == b.grid()
    a.close()
    b.close()


def test_unlocked_grid_beyond_max_cell_is_an_error():
    sim = api.Simulation.from_scene(_scene(max_cell=1000))
    with pytest.raises(api.MfreeError) as e:
        sim.step()
    assert e.value.status == api.ERR_ARG
    sim.close()


def test_unlocked_grid_context_steps_alone():
    b = api.Batch()
    sim = api.Simulation.from_scene(_scene())
    with pytest.raises(api.MfreeError):
        b.admit(sim)
    b.close()
    sim.close()
