"""Batches (mfree_batch_*): many scenes stepped with one launch per kernel.

A single scene (mfree_step / mfree_advance) runs the same batched kernels over
a table of one scene, so a scene's results in a batch must be identical --
bit for bit, tolerance 0 -- to the same scene stepped alone with the same
pair-loop tiling, whatever else is in the batch and whenever it joined.  The tests also cover the life cycle
(step counts, retirement, the memory budget, the variant check), graph replay
against eager launches, and the autotuner (which must leave the scenes'
state untouched).
"""
import numpy as np
import pytest

from iwf_mfree_gpu_3d_b200 import api, scenes

from helpers import by_id

pytestmark = pytest.mark.gpu

NAMES = ("POS", "VEL", "S", "T", "EPS_PL", "RHO", "FC", "FT")


def _specs():
    return scenes.mixed_specs(4, seed=7, n_lo=1500, n_hi=9000)


def _scene(k):
    return scenes.mixed_scene(_specs()[k])


def _state(sim):
    ids = sim.get("ID")
    out = {n: by_id(ids, sim.get(n)) for n in NAMES}
    out["forces"] = sim.tool_forces().copy()
    out["time"] = sim.time()
    return out


def _assert_same(a, b, what):
    for n in a:
        np.testing.assert_array_equal(np.asarray(a[n]), np.asarray(b[n]), err_msg=f"{what}: {n}")


def _alone(k, steps, **opt):
    sim = api.Simulation.from_scene(_scene(k), **opt)
    sim.advance(steps, record_every=1, use_graph=True)
    st = _state(sim)
    sim.close()
    return st


@pytest.mark.parametrize("use_graph", [True, False])
def test_scene_alone_equals_scene_in_a_changing_batch(use_graph):
    # slots 0, 1 start together; 2 joins after 6 steps (the others are then at
    # another state parity); 1 stops at 10, 2 at 6 + 9, 0 at 20, 3 runs on
    targets = {0: 20, 1: 10, 2: 9, 3: 0}
    b = api.Batch()
    sims = {k: api.Simulation.from_scene(_scene(k)) for k in range(4)}
    slot = {k: b.admit(sims[k], targets[k]) for k in (0, 1, 3)}
    b.step(6, record_every=1, use_graph=use_graph)
    slot[2] = b.admit(sims[2], targets[2])
    b.step(14, record_every=1, use_graph=use_graph)
    for k in (0, 1, 2):
        done, target, status = b.query(slot[k])
        assert (done, target, status) == (targets[k], targets[k], b.DONE), k
    done3, _, status3 = b.query(slot[3])
    assert (done3, status3) == (20, b.RUNNING)
    for k, steps in ((0, 20), (1, 10), (2, 9), (3, 20)):
        _assert_same(_state(sims[k]), _alone(k, steps), f"scene {k}")
    b.close()


def test_retired_scene_steps_alone_again_and_matches():
    b = api.Batch()
    s0 = api.Simulation.from_scene(_scene(0))
    s1 = api.Simulation.from_scene(_scene(1))
    k0 = b.admit(s0)
    b.admit(s1)
    b.step(5, record_every=1)
    with pytest.raises(api.MfreeError):
        s0.step()  # the batch owns it
    s0 = b.retire(k0, keep=True)
    s0.advance(4, record_every=1)  # back on its own stream
    _assert_same(_state(s0), _alone(0, 9), "retired scene")
    s0.close()
    b.close()


def test_memory_budget_and_variant_check():
    s0 = api.Simulation.from_scene(_scene(0))
    s1 = api.Simulation.from_scene(_scene(1))
    s0.step()  # allocates the grid-sized scratch
    b = api.Batch(hbm_budget=s0.device_bytes() + 4096)
    assert b.admit(s0) is not None
    assert b.admit(s1) is None  # does not fit: stays with the caller
    info = b.info()
    assert info["scenes"] == 1 and info["bytes"] == s0.device_bytes() and info["budget"] > 0
    s1.advance(2)  # still usable alone
    b.close()
    s1.close()
    b2 = api.Batch()
    b2.admit(api.Simulation.from_scene(_scene(2)))
    cspm = api.Simulation.from_scene(scenes.orthogonal_cutting(12, 6, 6, cspm=True, precision=1))
    with pytest.raises(api.MfreeError):
        b2.admit(cspm)
    cspm.close()
    b2.close()


def test_scene_bytes_estimate_matches_the_allocation():
    sc = _scene(1)
    sc.tools = []
    sim = api.Simulation.from_scene(sc)
    sim.step()
    (nx, ny, nz), _, _ = sim.grid()
    assert sim.device_bytes() == api.scene_bytes(sc.pos.shape[0], nx * ny * nz)
    sim.close()


def test_autotune_leaves_the_scenes_untouched_and_its_tiling_is_used():
    b = api.Batch()
    sims = [api.Simulation.from_scene(_scene(k)) for k in (0, 1)]
    for s in sims:
        b.admit(s)
    b.step(3, record_every=1)
    before = [_state(s) for s in sims]
    lpp, depth, ms = b.autotune(trial_steps=2)
    assert lpp in (8, 16, 32) and 4 <= depth <= 8 and ms > 0
    assert b.tiling() == (lpp, depth)
    for s, st in zip(sims, before):
        _assert_same(_state(s), st, "after autotune")
    # the tuned tiling differs from the default only in rounding; a scene
    # stepped alone with it from the same state is identical
    b.step(4, record_every=1)
    ref = api.Simulation.from_scene(_scene(0))
    ref.advance(3, record_every=1)
    ref.set_options(**dict(_scene(0).options, lanes_per_particle=lpp, tile_depth=depth))
    ref.advance(4, record_every=1)
    _assert_same(_state(sims[0]), _state(ref), "tuned tiling")
    ref.close()
    b.close()
