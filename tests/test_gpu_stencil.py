"""Stencil pruning of the pair loop: the pair kernel skips the cells of the
5x5x5 stencil that lie wholly beyond the target's support radius.  Only
out-of-support candidates are skipped, in the same order, so every field must
equal the full-stencil run bit for bit; a step whose predictor moves a
particle too far for the pruning's margin falls back to the full stencil and
is counted.  With PSE conduction, which sums every candidate of the stencil,
only tiles whose PSE sums are exactly zero (every staged temperature equal)
are pruned, and their PSE terms skipped -- again bit for bit."""
import numpy as np
import pytest

from iwf_mfree_gpu_3d_b200 import api, scenes

pytestmark = pytest.mark.gpu

FIELDS = ["POS", "VEL", "S", "EPS_PL", "T", "RHO", "POS_T", "VEL_T", "S_T", "RHO_T", "T_T", "FC", "FT", "ID",
          "HASH", "NUM_NBH", "BLANKED"]


def _pair(sc, steps, setup=None, **opt):
    runs = []
    for full in (0, 1):
        sim = api.Simulation.from_scene(sc, diagnostics=1, full_stencil=full, **opt)
        if setup is not None:
            setup(sim)
        for _ in range(steps):
            sim.step()
        runs.append(({n: sim.get(n).copy() for n in FIELDS}, sim.counters()))
        sim.close()
    return runs


def _assert_identical(a, b):
    for n in FIELDS:
        np.testing.assert_array_equal(a[n], b[n], err_msg=n)


@pytest.mark.parametrize("cspm,conduction", [(False, 1), (True, 1), (False, 0), (True, 0)])
def test_pruned_stencil_equals_full_stencil(cspm, conduction):
    sc = scenes.orthogonal_cutting(30, 15, 12, cspm=cspm, conduction=conduction)
    (fa, ca), (fb, cb) = _pair(sc, 40)
    _assert_identical(fa, fb)
    assert ca["full_stencil_steps"] == 0
    assert cb["full_stencil_steps"] == 0


@pytest.mark.parametrize("cspm", [True, False])
def test_zero_pse_tiles_equal_the_full_evaluation(cspm):
    """PSE conduction from a uniform temperature: every tile starts with
    exactly-zero PSE sums and is run without them on the pruned stencil;
    plastic work and friction heat the particles at the tool, whose tiles then
    evaluate the PSE terms.  60 steps, bit for bit against the full
    evaluation, with both kinds of tile counted."""
    sc = scenes.orthogonal_cutting(30, 15, 12, cspm=cspm, conduction=2)
    (fa, ca), (fb, cb) = _pair(sc, 60)
    _assert_identical(fa, fb)
    n = sc.n
    assert cb["pse_zero_targets"] == 0
    assert ca["pse_zero_targets"] >= n  # the first step: every tile
    assert ca["pse_zero_targets"] < 60 * n  # heated tiles evaluated the PSE terms
    assert not np.all(fa["T"] == fa["T"][0])


def test_zero_pse_skip_leaves_nonuniform_temperatures_alone():
    """A random temperature field: no tile has a zero PSE sum, and the fields
    equal the full evaluation."""
    sc = scenes.orthogonal_cutting(30, 15, 12, cspm=True, conduction=2)
    sc.T = (300.0 + np.random.default_rng(3).uniform(0.0, 50.0, sc.n)).astype(np.float32)
    (fa, ca), (fb, _) = _pair(sc, 5)
    _assert_identical(fa, fb)
    assert ca["pse_zero_targets"] == 0


def _kick(speed):
    def kick(sim):
        v = sim.get("VEL").reshape(-1, 4).copy()
        v[:: 997, 0] = speed  # cm/us
        sim.set("VEL", v)
    return kick


def test_fast_particles_widen_the_pruning_margin():
    """A few particles at 3000 m/s move ~5 % of a cell in the predictor's half
    step: the margin grows with the step's largest move and the fields stay
    those of the full stencil."""
    sc = scenes.orthogonal_cutting(30, 15, 12)
    (fa, ca), (fb, _) = _pair(sc, 3, setup=_kick(0.3))
    _assert_identical(fa, fb)
    assert ca["full_stencil_steps"] == 0


def test_very_fast_particles_switch_the_step_to_the_full_stencil():
    """Particles at 30 km/s move about half a cell in the half step, beyond
    the largest margin the pruning takes: those steps use the full stencil
    and are counted."""
    sc = scenes.orthogonal_cutting(30, 15, 12)
    (fa, ca), (fb, _) = _pair(sc, 3, setup=_kick(3.0))
    _assert_identical(fa, fb)
    assert ca["full_stencil_steps"] >= 1


def test_pruned_stencil_in_a_batch_equals_full_stencil():
    """Scenes of a batch prune with their own grid origins and give the same
    fields as the same batch run with the full stencil."""
    specs = [scenes.orthogonal_cutting(24, 12, 10, conduction=1), scenes.orthogonal_cutting(28, 14, 9, conduction=1)]
    out = {}
    for full in (0, 1):
        b = api.Batch()
        sims = [api.Simulation.from_scene(sc, diagnostics=1, full_stencil=full) for sc in specs]
        for s in sims:
            assert b.admit(s) is not None
        b.step(25)
        b.sync()
        out[full] = [{n: s.get(n).copy() for n in FIELDS} for s in sims]
        b.close()
    for a, c in zip(out[0], out[1]):
        _assert_identical(a, c)
