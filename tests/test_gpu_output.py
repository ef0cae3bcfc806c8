"""Output in the reference's formats (mfree_write_vtk*, mfree_append_force_log):
the legacy VTK text of vtk_writer.cpp and the force log of tool_forces::report,
checked line by line against the context's fields.  The particle file is
written in the background: it must hold the state of the moment of the call
even when the caller keeps stepping."""
import numpy as np
import pytest

from iwf_mfree_gpu_3d_b200 import api, scenes

pytestmark = pytest.mark.gpu


def _read_sections(path):
    lines = open(path).read().split("\n")
    assert lines[:5] == ["# vtk DataFile Version 2.0", "mfree iwf", "ASCII", "", "DATASET UNSTRUCTURED_GRID"]
    return lines


def _block(lines, head, count, start=0):
    k = next(i for i in range(start, len(lines)) if lines[i].startswith(head))
    return k, lines[k + 1:k + 1 + count]


def test_particle_vtk_holds_the_state_of_the_call():
    sim = api.Simulation.from_scene(scenes.small_scene())
    sim.advance(5, use_graph=True)
    pos = sim.get("POS")
    rho = sim.get("RHO")
    T = sim.get("T")
    eps = sim.get("EPS_PL")
    blanked = sim.get("BLANKED")
    fixed = sim.get("FIXED")
    S = sim.get("S").reshape(-1, 3, 3)
    p = sim.get("P")
    fc = sim.get("FC")
    import tempfile, os
    d = tempfile.mkdtemp()
    path = os.path.join(d, "vtk_out_000005.vtk")
    sim.write_vtk(path)
    sim.advance(7, use_graph=True)  # the file keeps the state of the call
    sim.output_wait()
    lines = _read_sections(path)
    keep = np.nonzero(blanked != 1.0)[0]
    m = len(keep)
    assert lines[5] == f"POINTS {m} float"
    pts = np.array([list(map(float, l.split())) for l in lines[6:6 + m]])
    np.testing.assert_allclose(pts, pos[keep, :3], atol=1e-6)
    assert lines[6 + m] == ""
    assert lines[7 + m] == f"CELLS {m} {2 * m}"
    assert lines[8 + m:8 + 2 * m] == [f"1 {i}" for i in keep]
    k, types = _block(lines, "CELL_TYPES", m)
    assert lines[k] == f"CELL_TYPES {m}" and types == ["1"] * m
    k, _ = _block(lines, "POINT_DATA", 0)
    assert lines[k] == f"POINT_DATA {m}"
    svm_ref = []
    for i in keep:
        s = S[i].astype(np.float64)
        sxx, syy, szz = s[0, 0] - p[i], s[1, 1] - p[i], s[2, 2] - p[i]
        s2 = sxx * sxx + syy * syy + szz * szz - sxx * syy - sxx * szz - syy * szz + \
            3 * (s[0, 1] ** 2 + s[1, 2] ** 2 + s[0, 2] ** 2)
        svm_ref.append(np.sqrt(s2) if s2 > 0 else 0.0)
    expect = {"density": rho[keep], "contact": (np.linalg.norm(fc[keep], axis=1) > 0).astype(float),
              "Temperature": T[keep], "Fixed": fixed[keep], "Tool": np.zeros(m),
              "EquivAccumPlasticStrain": eps[keep], "Svm": np.array(svm_ref)}
    start = 0
    for name, ref in expect.items():
        k, vals = _block(lines, f"SCALARS {name} float 1", m + 1, start)
        assert vals[0] == "LOOKUP_TABLE default"
        got = np.array([float(v) for v in vals[1:]])
        np.testing.assert_allclose(got, ref, rtol=1e-5, atol=1e-6, err_msg=name)
        start = k + 1
    sim.close()


def test_tool_and_blanking_vtk_and_force_log(tmp_path):
    sc = scenes.small_scene()
    sim = api.Simulation.from_scene(sc)
    for _ in range(3):
        sim.step(record_forces=True)
        sim.append_force_log(str(tmp_path / "forces_new.txt"))
    f_last = sim.tool_forces()
    dt, t = sim.time()
    t_last = t - dt  # the time of the last step
    sim.write_vtk_tools(str(tmp_path / "vtk_tool_000003.vtk"))
    lines = _read_sections(tmp_path / "vtk_tool_000003.vtk")
    tool = sc.tools[0]
    nv, nt = len(tool.verts), len(tool.tris)
    assert lines[5] == f"POINTS {nv} float"
    pts = np.array([list(map(float, l.split())) for l in lines[6:6 + nv]])
    np.testing.assert_allclose(pts, tool.verts + tool.vel[None, :] * np.float32(t_last), atol=2e-6)
    k, cells = _block(lines, "CELLS", nt)
    assert lines[k] == f"CELLS {nt} {4 * nt}"
    assert cells == [f"3 {a} {b} {c}" for a, b, c in tool.tris]
    k, ids = _block(lines, "SCALARS id float 1", nv + 1)
    assert ids[1:] == ["0"] * nv
    k, act = _block(lines, "SCALARS active float 1", nv + 1)
    assert act[1:] == ["1"] * nv
    sim.write_vtk_blanking(str(tmp_path / "vtk_bbox_000003.vtk"))
    lines = _read_sections(tmp_path / "vtk_bbox_000003.vtk")
    assert lines[5] == "POINTS 8 float"
    corners = np.array([list(map(float, l.split())) for l in lines[6:14]])
    lo, hi = sc.blank_bbmin, sc.blank_bbmax
    np.testing.assert_allclose(corners[0], lo, atol=1e-6)
    np.testing.assert_allclose(corners[6], hi, atol=1e-6)
    k, quads = _block(lines, "CELLS 6 30", 6)
    assert quads[0] == "4 0 1 2 3" and quads[5] == "4 4 5 6 7"
    log = open(tmp_path / "forces_new.txt").read().split("\n")
    assert len(log) == 4 and log[3] == ""
    last = [float(v) for v in log[2].split()]
    np.testing.assert_allclose(last, f_last.reshape(-1), rtol=1e-8)
    sim.close()


def test_fields_into_page_locked_memory_equal_the_host_path():
    """mfree_get_field into page-locked memory (the device writes the field in
    the reference layout) gives the same bits as into pageable memory (copied
    and converted on the host), for every state field, in both forms."""
    import torch

    for precision in (0, 1):
        sim = api.Simulation.from_scene(scenes.small_scene(), precision=precision)
        sim.advance(7, use_graph=True)
        for name in ("POS", "VEL", "VEL_BC", "H", "RHO", "S", "S_T", "FC", "FT", "POS_T", "VEL_T", "FIXED",
                     "EPS_PL_DOT", "BLANKED", "TOOL_PARTICLE", "EPS_PL", "T", "RHO_T", "T_T", "ID", "IDX", "HASH"):
            ref = sim.get(name)
            tdt = torch.int32 if ref.dtype == np.int32 else torch.float32
            pinned = torch.full((ref.size,), -7, dtype=tdt, pin_memory=True).numpy()
            got = sim.get(name, out=pinned)
            np.testing.assert_array_equal(got.view(np.uint32), ref.view(np.uint32), err_msg=name)
        sim.close()
