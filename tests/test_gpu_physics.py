"""Parity of the CUDA step with the FP64 oracle for the other switches of the
reference (CSPM + PSE, the compensated precision form, exhaustive contact,
tool particles with conduction) and the failure paths (NaN blanking, secant
iteration limit), all through the C ABI."""
import numpy as np
import pytest

import oracle
from iwf_mfree_gpu_3d_b200 import api, scenes

from helpers import grain_checks, check, compare, gpu_state, oracle_state

pytestmark = pytest.mark.gpu


def _run(sc, steps, **opt):
    sim = api.Simulation.from_scene(sc, **opt)
    orc = oracle.Oracle(sc, prec=64)
    for _ in range(steps):
        sim.step()
        orc.step()
    return sim, orc


def test_cspm_pse_100_steps():
    """CSPM correction + PSE conduction (the 1M configuration's switches) on a
    30 x 15 x 12 block: per-field relative L2 after 100 steps."""
    sc = scenes.orthogonal_cutting(30, 15, 12, cspm=True, conduction=2)
    sim, orc = _run(sc, 100)
    err = compare(gpu_state(sim), oracle_state(orc), sc)
    print("CSPM+PSE 100-step relative L2:", err)
    check(err, "cspm_pse_100")
    sim.close()


def test_precision_form_tracks_fp64_closer():
    """Compensated hi/lo positions and velocities: the displacement error
    against the FP64 oracle is at most a fifth of plain FP32's (measured:
    0.17) after 60 steps, and position and velocity stay within three times
    their measured errors (1.5e-5, 5.2e-5).  The velocity error of this small
    scene is set by a few particles at the tool, whose friction switches
    between stick and slip at the Coulomb cap on last-bit differences of the
    normal force; plain FP32 measures 2.2e-5."""
    sc = scenes.small_scene()
    plain, orc = _run(sc, 60)
    prec = api.Simulation.from_scene(sc, precision=1)
    for _ in range(60):
        prec.step()
    o = oracle_state(orc)
    e_plain = compare(gpu_state(plain), o, sc)
    e_prec = compare(gpu_state(prec, f64=True), o, sc)
    print("plain:", e_plain["POS"], e_plain["VEL"], "precision form:", e_prec["POS"], e_prec["VEL"])
    assert e_prec["POS"] < 4.5e-5 and e_prec["VEL"] < 1.6e-4
    assert e_prec["POS"] <= 0.2 * e_plain["POS"]
    plain.close()
    prec.close()


def test_exhaustive_contact_algorithm():
    sc = scenes.small_scene(algorithm=api.CONTACT_EXHAUSTIVE)
    sim, orc = _run(sc, 30)
    err = compare(gpu_state(sim), oracle_state(orc), sc)
    print("exhaustive contact 30-step relative L2:", err)
    check(err, "exhaustive_30")
    sim.close()


def _force_series(sc, steps):
    """Tool forces recorded on every step (tool_forces::get_forces_host,
    tool_3d_gpu.cu:30-69) by the CUDA path and the FP64 oracle."""
    sim = api.Simulation.from_scene(sc)
    orc = oracle.Oracle(sc, prec=64)
    fg, fo = [], []
    for _ in range(steps):
        sim.step(record_forces=True)
        orc.step(record=True)
        fg.append(sim.tool_forces().astype(np.float64).copy())
        fo.append(orc.tool_forces().astype(np.float64).copy())
    return sim, orc, np.array(fg), np.array(fo)


def test_tool_forces_match_oracle_over_100_steps():
    """The summed tool force of every step against the FP64 oracle's over 100
    steps: the force series (relative L2 over steps and components), the
    impulse (the sum over steps) and the steps on which the tool touches."""
    sc = scenes.small_scene()
    sim, orc, fg, fo = _force_series(sc, 100)
    touch_g, touch_o = np.abs(fg).sum(axis=2) > 0, np.abs(fo).sum(axis=2) > 0
    e_series = np.linalg.norm(fg - fo) / np.linalg.norm(fo)
    e_impulse = np.linalg.norm(fg.sum(0) - fo.sum(0)) / np.linalg.norm(fo.sum(0))
    print(f"tool forces over 100 steps: series rel L2 {e_series:.3e}, impulse {e_impulse:.3e}, "
          f"contact steps {touch_g.sum()} (oracle {touch_o.sum()})")
    assert touch_o.sum() > 20
    # contact starts and ends where a particle crosses the tool surface: a
    # last-bit difference may move one such step
    assert int((touch_g != touch_o).sum()) <= 2
    # measured: series 2.8e-5, impulse 8.6e-6
    assert e_series < 1e-4 and e_impulse < 3e-5
    sim.close()


def test_two_tools_against_fp64_oracle():
    """Two wedges at different depths cutting one block side by side (the
    reference's multi-tool stepping, tools processed in order): every field
    after 100 steps and each tool's force series against the FP64 oracle."""
    sc = scenes.two_tool_scene()
    sim, orc, fg, fo = _force_series(sc, 100)
    err = compare(gpu_state(sim), oracle_state(orc), sc)
    print("two tools 100-step relative L2:", err)
    check(err, "two_tools_100")
    for k in range(2):
        assert (np.abs(fo[:, k]).sum(axis=1) > 0).sum() > 5, k  # both tools touch the block
        e_series = np.linalg.norm(fg[:, k] - fo[:, k]) / np.linalg.norm(fo[:, k])
        print(f"tool {k}: force series rel L2 {e_series:.3e}")
        assert e_series < 1e-4, (k, e_series)  # measured 2.7e-5 and 4.5e-6


def test_five_grains_against_fp64_oracle_and_the_reference_step():
    """Five grains in the reference's five-tool arrangement (a centre grain,
    two leading beside it, two trailing behind): the first step's contact
    force of every tool against the FP64 oracle (the leading row in contact,
    the trailing row not yet), then 40 steps checked as the single-grain
    scenes are (against the reference's own GPU step where built)."""
    sc = scenes.five_grain_scene()
    sim, orc, fg, fo = _force_series(sc, 1)
    for k in range(5):
        ng, no = np.linalg.norm(fg[0, k]), np.linalg.norm(fo[0, k])
        if k < 3:
            assert no > 0, k  # the leading row touches the block from the first step
            assert np.linalg.norm(fg[0, k] - fo[0, k]) < 1e-5 * no, (k, fg[0, k], fo[0, k])
        else:
            assert ng == 0 and no == 0, (k, ng, no)
    for _ in range(39):
        sim.step()
        orc.step()
    o = oracle_state(orc)
    err = compare(gpu_state(sim), o, sc)
    print("five grains, 40-step relative L2 vs FP64 oracle:", {k: f"{v:.2e}" for k, v in err.items()})
    grain_checks(sc, sim, err, o, 40, "grain_40")
    sim.close()
    sim.close()


def test_tool_particles_conduct_heat():
    """Tool particles (tool_p = 1) exchange heat by Brookshaw conduction, skip
    the mechanics and translate with the tool (actions_gpu.cu:55-68)."""
    sc = scenes.small_scene()
    n = sc.n
    # make the 200 particles with the largest x tool particles at 600 K
    sel = np.argsort(sc.pos[:, 0])[-200:]
    sc.tool_p[sel] = 1.0
    sc.T[sel] = 600.0
    sc.fixed[sel] = 0.0
    sc.trml_tool = dict(cp=5.2e-6, tq=0.0, k=2.2e-10, alpha=2.2e-10 / (3.5 * 5.2e-6), T_init=300.0, eta=0.0)
    sim, orc = _run(sc, 40)
    g, o = gpu_state(sim), oracle_state(orc)
    err = compare(g, o, sc)
    print("tool particles 40-step relative L2:", err)
    check(err, "tool_particles_40")
    # tool particles moved rigidly with the tool velocity
    ids = sim.get("ID")
    pos = np.empty((n, 4), np.float32)
    pos[ids] = sim.get("POS")
    dxt = pos[sel, 0] - sc.pos[sel, 0]
    assert np.allclose(dxt, dxt.mean(), atol=1e-9) and dxt.mean() < 0
    sim.close()


def test_single_grain_with_tool_particles_against_oracle():
    """The single-grain configuration at small size: a truncated-icosphere
    grain (1,280 triangles, radius 6 dx) cutting a 40 x 20 x 12 block from the
    first step, its volume sampled into diamond tool particles (thermal
    contact the reference way), 40 steps.  The compensated form's error
    against the FP64 oracle is no larger than the reference's own GPU step's,
    and the plain FP32 form follows the reference's GPU step to ~1e-6 (the
    grain's contact parts FP32 from FP64 within a few steps, see grain_40 in
    helpers.py)."""
    make = lambda precision: scenes.single_grain(40, 20, 12, radius=6.0, depth=4.0, v_tool=3.0e-3,  # noqa: E731
                                                 precision=precision)
    sc = make(1)
    assert (sc.tool_p == 1.0).sum() > 300
    sim, orc = _run(sc, 40)
    o = oracle_state(orc)
    err = compare(gpu_state(sim, f64=True), o, sc)
    print("single grain 40-step relative L2:", {k: f"{v:.2e}" for k, v in err.items()})
    sim.close()
    sc0 = make(0)
    plain = api.Simulation.from_scene(sc0)
    for _ in range(40):
        plain.step()
    grain_checks(sc0, plain, err, o, 40, "grain_40")
    plain.close()


def test_nan_rate_spreads_and_is_blanked():
    """A NaN rate is not blanked by itself (do_blanking only refuses to
    unblank, actions_gpu.cu:506-529): it spreads through the pair loop, the
    contaminated positions leave the box and those particles are blanked and
    kept blanked.  The reference multiplies NaN neighbours outside the support
    by a zero kernel gradient, so its NaN front covers the whole 5x5x5 stencil;
    the CUDA path skips those pairs, so its blanked set is a subset of the
    oracle's."""
    sc = scenes.small_scene()
    sim = api.Simulation.from_scene(sc)
    orc = oracle.Oracle(sc, prec=64)
    vt = np.zeros((sc.n, 3), np.float32)
    vt[1234, 0] = np.nan
    sim.set("VEL_T", vt)
    orc.set_field("VEL_T", vt.astype(np.float64))
    for _ in range(4):
        sim.step()
        orc.step()
    g_ids = set(sim.get("ID")[sim.get("BLANKED") == 1].tolist())
    o_ids = set(orc.field("ID")[orc.field("BLANKED") == 1].astype(int).tolist())
    assert 1234 in g_ids and len(g_ids) > 1
    assert g_ids <= o_ids
    n_act, n_init = sim.counts()
    assert n_act == n_init - len(g_ids)
    assert set(sim.get("ID")[n_act:].tolist()) == g_ids  # blanked particles sort to the tail
    assert sim.counters()["nan_blanked"] >= 1
    act = sim.get("POS")[:n_act]
    assert np.isfinite(act).all()
    sim.close()


def test_velocity_blanking_moves_particle_to_tail():
    sc = scenes.small_scene()
    sim = api.Simulation.from_scene(sc)
    sim.step()
    v = sim.get("VEL")
    ids = sim.get("ID")
    k = int(np.where(ids == 77)[0][0])
    v[k, 0] = 10.0  # above the 4 cm/us blanking speed
    sim.set("VEL", v)
    sim.step()
    n_act, n_init = sim.counts()
    assert n_act == n_init - 1 and sim.get("ID")[n_init - 1] == 77
    sim.close()


def test_all_particles_leaving_the_box_is_reported():
    """The reference prints and exits when every particle has left the box
    (grid_gpu_base.cu:159-163); here the next call returns MFREE_ERR_EMPTY."""
    sc = scenes.orthogonal_cutting(10, 6, 5)
    sim = api.Simulation.from_scene(sc)
    sim.set_blanking(sc.blank_bbmin, sc.blank_bbmax, sc.blank_vmax, bbvel=np.array([100.0, 0, 0], np.float32))
    with pytest.raises(api.MfreeError) as e:
        for _ in range(5):
            sim.step()
        sim.sync()
    assert e.value.status == -6
    sim.close()


def test_secant_iteration_limit_is_reported():
    """With the iteration limit at 1 the radial return reports failures
    through the counters instead of printing (actions_gpu.cu:415-418)."""
    sc = scenes.small_scene()
    sim = api.Simulation.from_scene(sc, max_secant_iter=1)
    for _ in range(15):
        sim.step()
    assert sim.counters()["secant_failures"] > 0
    assert np.isfinite(sim.get("S")).all()
    sim.close()


def test_field_round_trip_and_reference_layout():
    sc = scenes.small_scene()
    sim = api.Simulation.from_scene(sc)
    sim.step()
    S = sim.get("S").reshape(-1, 3, 3)
    np.testing.assert_array_equal(S, np.transpose(S, (0, 2, 1)))  # symmetric, GLM column-major
    for name in ("POS", "VEL", "S", "T", "EPS_PL", "FT", "VEL_T"):
        a = sim.get(name)
        sim.set(name, a)
        np.testing.assert_array_equal(sim.get(name), a)
    assert set(sim.get("IDX")) == set(range(sc.n))
    sim.close()


def test_moving_grid_and_blanking_box():
    """Locked grid and blanking box moving with a velocity (the reference's
    moving-window setup, grid_gpu_base.cu:166-183, blanking.cpp:43-51)."""
    sc = scenes.small_scene()
    sim = api.Simulation.from_scene(sc)
    orc = oracle.Oracle(sc, prec=64)
    v = np.array([3.8, 0.0, 0.0], np.float32)  # the box's -x face sweeps past ~40 % of the block in 20 steps
    sim.set_grid_velocity(v)
    sim.set_blanking(sc.blank_bbmin, sc.blank_bbmax, sc.blank_vmax, bbvel=v)
    import ctypes as C
    oracle.lib().orc_set_grid_velocity(orc.h, v.ctypes.data_as(C.POINTER(C.c_float)))
    oracle.lib().orc_set_blanking(orc.h, sc.blank_bbmin.ctypes.data_as(C.POINTER(C.c_float)),
                                  sc.blank_bbmax.ctypes.data_as(C.POINTER(C.c_float)),
                                  v.ctypes.data_as(C.POINTER(C.c_float)), sc.blank_vmax)
    for _ in range(20):
        sim.step()
        orc.step()
    assert sim.counts()[0] == orc.counts()[0]
    assert 0.3 * sc.n < sc.n - sim.counts()[0] < 0.6 * sc.n
    err = compare(gpu_state(sim), oracle_state(orc), sc)
    assert err["blank_mismatch"] == 0
    sim.close()


def test_compact_arrays_match_the_reference_layout_fields():
    """mfree_get_array / mfree_set_array: the library's own float4 arrays hold
    the same values as the reference-layout fields, and writing a field
    through either path steps on identically."""
    sc = scenes.small_scene()
    sim = api.Simulation.from_scene(sc, precision=1)
    sim.advance(5, use_graph=True)
    A = {n: sim.get_array(n).copy() for n in api.ARRAYS}
    np.testing.assert_array_equal(A["POS_H"][:, :3], sim.get("POS")[:, :3])
    np.testing.assert_array_equal(A["POS_H"][:, 3], sim.get("H"))
    np.testing.assert_array_equal(A["VEL_RHO"][:, 3], sim.get("RHO"))
    S = sim.get("S").reshape(-1, 9)  # GLM column-major m[col][row]
    np.testing.assert_array_equal(A["S_A"], S[:, [0, 4, 8, 1]])
    np.testing.assert_array_equal(A["S_B"][:, :2], S[:, [2, 5]])
    np.testing.assert_array_equal(A["S_B"][:, 2], sim.get("T"))
    np.testing.assert_array_equal(A["S_B"][:, 3], sim.get("EPS_PL"))
    np.testing.assert_array_equal(A["S_T_B"][:, 3], sim.get("FIXED"))
    np.testing.assert_array_equal(A["FC"][:, 3], sim.get("TOOL_PARTICLE"))
    np.testing.assert_array_equal(A["FT"][:, 3], sim.get("BLANKED"))
    np.testing.assert_array_equal(A["VEL_BC"][:, 3].view(np.int32), sim.get("ID"))
    p64 = sim.get64("POS")[:, :3]
    np.testing.assert_array_equal(p64, A["POS_H"][:, :3].astype(np.float64) + A["LO"][:, :3])
    ptr = sim.array_device_ptr("POS_H")
    sim.step()
    assert ptr != 0 and sim.array_device_ptr("POS_H") != ptr  # the other copy after a step

    a = api.Simulation.from_scene(sc)
    b = api.Simulation.from_scene(sc)
    for s in (a, b):
        s.advance(3, use_graph=True)
    T = b.get("T") + np.float32(25.0)
    b.set("T", T)
    sb = a.get_array("S_B").copy()
    sb[:, 2] = T
    a.set_array("S_B", sb)
    for s in (a, b):
        s.advance(4, use_graph=True)
    for name in ("POS", "VEL", "S", "T", "EPS_PL", "ID"):
        np.testing.assert_array_equal(a.get(name), b.get(name), err_msg=name)
    for s in (sim, a, b):
        s.close()


@pytest.mark.parametrize("precision", [0, 1])
def test_fp64_energy_and_cfl_reductions_match_the_fields(precision):
    """mfree_get_energies: FP64 device reductions of the current state against
    the same sums in numpy FP64 from the fields; repeated calls give the same
    bits.  In the precision form the velocity is hi + lo of the compensated
    accumulation (the FP64 field read)."""
    sc = scenes.small_scene(precision=precision)
    sim = api.Simulation.from_scene(sc)
    sim.advance(20, use_graph=True)
    e1, e2 = sim.energies(), sim.energies()
    assert e1 == e2
    n_act = sim.counts()[0]
    vel = sim.get64("VEL")[:n_act, :3] if precision else sim.get("VEL")[:n_act, :3].astype(np.float64)
    if precision:  # the low parts are in the sum: hi alone differs
        hi = sim.get("VEL")[:n_act, :3].astype(np.float64)
        assert np.any(vel != hi)
    rho = sim.get("RHO")[:n_act].astype(np.float64)
    S = sim.get("S").reshape(-1, 9)[:n_act].astype(np.float64)
    T = sim.get("T")[:n_act].astype(np.float64)
    h = sim.get("H")[:n_act].astype(np.float64)
    wp = (sim.get("TOOL_PARTICLE")[:n_act] != 1.0) & (sim.get("BLANKED")[:n_act] != 1.0)
    m, K, G, rho0 = (np.float64(np.float32(sc.phys[k])) for k in ("mass", "K", "G", "rho0"))
    c0sq = np.float64(np.float32(np.sqrt(np.float32(sc.phys["K"]) / np.float32(sc.phys["rho0"]))) ** 2)
    v2 = (vel ** 2).sum(axis=1)
    ss = (S ** 2).sum(axis=1)
    p = c0sq * (rho - rho0)
    terms = dict(kinetic=(0.5 * m * v2)[wp],
                 elastic_deviatoric=((m / rho) * ss / (4 * G))[wp],
                 elastic_volumetric=((m / rho) * p * p / (2 * K))[wp],
                 thermal=(m * np.float64(np.float32(sc.trml_wp["cp"])) *
                          (T - np.float64(np.float32(sc.trml_wp["T_init"]))))[wp])
    for k, t in terms.items():  # sums: within 1e-9 of the sum of magnitudes (summation order)
        assert abs(e1[k] - t.sum()) <= 1e-9 * np.abs(t).sum() + 1e-300, (k, e1[k], t.sum())
    cfl = (h / (np.sqrt(K / rho) + np.sqrt(v2)))[wp].min()
    assert abs(e1["cfl_dt"] - cfl) <= 1e-12 * cfl, (e1["cfl_dt"], cfl)
    assert e1["kinetic"] > 0 and e1["elastic_deviatoric"] > 0 and e1["cfl_dt"] > 0
    sim.close()
