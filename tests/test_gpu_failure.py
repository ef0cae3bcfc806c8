"""Failure detection on the GPU without a fault: the pair kernel's staging
waits are bounded (~0.5 s); mfree_inject_fault makes them wait for bytes that
never come, so every wait runs out.  The kernel counts it and leaves, the next
call reports MFREE_ERR_TIMEOUT, the counter shows it, and the CUDA context
stays usable (a fresh context steps normally afterwards)."""
import numpy as np
import pytest

from iwf_mfree_gpu_3d_b200 import api, scenes

pytestmark = pytest.mark.gpu


def test_staging_wait_that_runs_out_is_reported():
    sim = api.Simulation.from_scene(scenes.small_scene())
    sim.step()
    sim.step()
    assert sim.counters()["staging_timeouts"] == 0
    sim.inject_fault(1)
    sim.step()  # every block's first staging wait runs out (~0.5 s), then it leaves
    with pytest.raises(api.MfreeError) as err:
        sim.sync()  # the status of the last step (the next step would report it too)
    assert err.value.status == api.ERR_TIMEOUT
    assert sim.counters()["staging_timeouts"] > 0
    sim.inject_fault(0)
    sim.close()
    # the device is still usable: a new context steps and matches a reference run
    a = api.Simulation.from_scene(scenes.small_scene())
    b = api.Simulation.from_scene(scenes.small_scene())
    a.advance(3)
    b.advance(3, use_graph=False)
    np.testing.assert_array_equal(a.get("POS"), b.get("POS"))
    assert a.counters()["staging_timeouts"] == 0
    a.close()
    b.close()
