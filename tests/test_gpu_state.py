"""Checkpoint and resume (mfree_export_state / mfree_import_state): a context
rebuilt from an exported record steps on bit for bit as the exported one,
graph replay and tool-force recording included; damaged records are refused."""
import numpy as np
import pytest

from iwf_mfree_gpu_3d_b200 import api, scenes

pytestmark = pytest.mark.gpu

NAMES = ("POS", "VEL", "S", "T", "EPS_PL", "RHO", "FC", "FT", "BLANKED", "ID")


def _state(sim):
    out = {n: sim.get(n) for n in NAMES}
    out["forces"] = sim.tool_forces()
    out["time"] = np.array(sim.time())
    out["counters"] = np.array(list(sim.counters().values()))
    return out


def test_imported_context_continues_bitwise():
    sc = scenes.small_scene(precision=1)
    a = api.Simulation.from_scene(sc)
    for _ in range(7):
        a.step(record_forces=True)
    rec = a.export_state()
    b = api.Simulation.import_state(rec)
    assert (b.n_init, b.num_tools) == (a.n_init, 1)
    for sim in (a, b):
        sim.advance(6, record_every=2, use_graph=True)
        sim.step(record_forces=True)
    sa, sb = _state(a), _state(b)
    for k in sa:
        np.testing.assert_array_equal(sa[k], sb[k], err_msg=k)
    a.close()
    b.close()


def test_damaged_records_are_refused():
    sim = api.Simulation.from_scene(scenes.small_scene())
    sim.step()
    rec = sim.export_state()
    sim.close()
    with pytest.raises(api.MfreeError):
        api.Simulation.import_state(rec[:-16])  # truncated
    bad = bytearray(rec)
    bad[0:8] = b"NOTMFREE"
    with pytest.raises(api.MfreeError):
        api.Simulation.import_state(bytes(bad))
