"""CPU checks of the C ABI library and of the host-side logic (no GPU calls)."""
import os
import re

import numpy as np
import pytest

from iwf_mfree_gpu_3d_b200 import api, scenes

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_library_exports_every_declared_symbol():
    L = api.lib()
    decl = set(re.findall(r"\b(mfree_[a-z0-9_]+)\s*\(", open(os.path.join(ROOT, "include", "mfree.h")).read()))
    missing = [s for s in decl if not hasattr(L, s)]
    assert not missing, missing
    assert decl == set(api.EXPORTS)


def test_field_widths_follow_reference_layout():
    L = api.lib()
    w = {n: L.mfree_field_width(i) for i, n in enumerate(api.FIELDS)}
    assert w["POS"] == 4 and w["VEL"] == 4 and w["S"] == 9 and w["R"] == 9 and w["S_T"] == 9
    assert w["FC"] == 3 and w["POS_T"] == 3 and w["RHO"] == 1 and w["HASH"] == 1
    assert L.mfree_field_width(len(api.FIELDS)) == -1


def _write_json_mesh(path, verts, tris):
    v = ", ".join(f"{x:.9g}" for x in verts.reshape(-1))
    t = ", ".join(str(int(x)) for x in tris.reshape(-1))
    path.write_text(
        '{\n  "vertices" :\n  [\n    {\n      "name" : "position_buffer",\n      "size" : 3,\n'
        f'      "values" :\n      [\n        {v}\n      ]\n    }}\n  ],\n  "connectivity" :\n  [\n'
        f'    {{\n      "mode" : "triangles_list",\n      "indices" :\n      [\n        {t}\n      ]\n    }}\n  ]\n}}\n')


def test_read_json_mesh(tmp_path):
    verts, tris = scenes.wedge_tool(0.0, 0.0, -0.01, 0.01, 1e-3)
    p = tmp_path / "wedge.json"
    _write_json_mesh(p, verts, tris)
    v, t = api.read_mesh(str(p))
    np.testing.assert_allclose(v, verts, rtol=1e-7)
    np.testing.assert_array_equal(t, tris)


def _tet_mesh():
    # a cube split into 5 tetrahedra
    v = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]], float)
    tets = [(0, 1, 3, 4), (1, 2, 3, 6), (1, 4, 5, 6), (3, 4, 6, 7), (1, 3, 4, 6)]
    return v, tets


def _write_k(path, v, tets):
    lines = ["$# test", "*KEYWORD", "*NODE", "$#   nid  x  y  z  tc  rc"]
    for i, p in enumerate(v):
        lines.append(f"{i + 1:10d} {p[0]:.9g} {p[1]:.9g} {p[2]:.9g} 0 0")
    lines += ["*ELEMENT_SOLID", "$#   eid     pid      n1      n2      n3      n4      n5      n6      n7      n8"]
    for e, t in enumerate(tets):
        n = [x + 1 for x in t]
        lines.append(f"{e + 1:8d}{1:8d}{n[0]:8d}{n[1]:8d}{n[2]:8d}{n[3]:8d}{n[3]:8d}{n[3]:8d}{n[3]:8d}{n[3]:8d}")
    lines.append("*END")
    path.write_text("\n".join(lines) + "\n")


def test_read_ldynak_tet_mesh_surface(tmp_path):
    v, tets = _tet_mesh()
    p = tmp_path / "cube.k"
    _write_k(p, v, tets)
    verts, tris = api.read_mesh(str(p))
    assert verts.shape == (8, 3) and tris.shape == (12, 3)  # the 12 boundary faces of the cube
    # every boundary face lies on the cube surface, interior faces are gone
    P = verts[tris]
    on_face = np.zeros(len(tris), bool)
    for d in range(3):
        for val in (0.0, 1.0):
            on_face |= np.all(P[:, :, d] == val, axis=1)
    assert on_face.all()
    # the surface is closed: every edge belongs to two faces
    edges = {}
    for t in tris:
        for a, b in ((t[0], t[1]), (t[1], t[2]), (t[2], t[0])):
            k = (min(a, b), max(a, b))
            edges[k] = edges.get(k, 0) + 1
    assert set(edges.values()) == {2}


def test_read_mesh_errors(tmp_path):
    with pytest.raises(api.MfreeError):
        api.read_mesh(str(tmp_path / "missing.k"))
    bad = tmp_path / "bad.json"
    bad.write_text("nothing here\n")
    with pytest.raises(api.MfreeError):
        api.read_mesh(str(bad))


def test_scene_is_deterministic_and_in_reference_order():
    a = scenes.small_scene()
    b = scenes.small_scene()
    np.testing.assert_array_equal(a.pos, b.pos)
    c = scenes.small_scene(seed=3)
    assert not np.array_equal(a.pos, c.pos)
    # x-major lattice, z = -k dx (benchmarks_single_grain.cu:720-737)
    n = a.pos.reshape(40, 20, 10, 4)
    assert np.all(np.diff(n[:, 0, 0, 0]) > 0) and np.all(np.diff(n[0, 0, :, 2]) < 0)
    jit = a.pos[:, 0] - np.repeat(np.arange(40), 200) * 1e-3
    assert np.abs(jit).max() <= 0.0100001e-3
    # one fixed bottom layer
    assert a.fixed.sum() == 40 * 20


def test_wedge_is_closed_manifold():
    v, t = scenes.wedge_tool(0.0, -5e-3, -0.01, 0.01, 1e-3)
    assert t.shape == (12, 3)
    edges = {}
    for tri in t:
        for a, b in ((tri[0], tri[1]), (tri[1], tri[2]), (tri[2], tri[0])):
            edges[(a, b)] = edges.get((a, b), 0) + 1
    # consistently oriented: each directed edge once, its reverse once
    for (a, b), c in edges.items():
        assert c == 1 and edges.get((b, a)) == 1


def test_icosphere_grain_closed():
    v, f = scenes.truncated_grain(0.02)
    assert f.shape == (1280, 3)
    edges = {}
    for tri in f:
        for a, b in ((tri[0], tri[1]), (tri[1], tri[2]), (tri[2], tri[0])):
            edges[(min(a, b), max(a, b))] = edges.get((min(a, b), max(a, b)), 0) + 1
    assert set(edges.values()) == {2}


def test_time_step_formula():
    # dt = 0.5 * CFL * h / (sqrt(v_tool) + c0) (benchmarks_single_grain.cu:849-851)
    sc = scenes.small_scene()
    c0 = np.sqrt(sc.phys["K"] / sc.phys["rho0"])
    assert sc.dt == pytest.approx(0.5 * 0.3 * 1.3e-3 / (np.sqrt(1e-3) + c0), rel=1e-6)
    assert sc.dt == pytest.approx(4.0468e-4, rel=1e-4)
