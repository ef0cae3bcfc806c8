"""Scene setup against the reference's own host code (golden file).

tests/golden/ref_setup.npz holds what the reference's readers and tool setup
(json_reader.cpp, ldynak_reader.cpp, surface_tri_mesh.cpp, grid_cpu_tri.cpp,
tool_3d.cpp, compiled unchanged by oracle/build_ref.sh) make of the reference's
own mesh assets (Release/*.json, Release/*.k), of a seeded hexahedral block and
of the benchmark scenes' tool meshes (tests/golden/make_ref_setup_golden.py).

* The library's readers give the reference's vertices and triangles in the
  reference's order (its std::unordered_map iteration order; closest-triangle
  ties in the contact search break by it) -- on the assets when the reference
  checkout is at hand, and on the hexahedral block always.
* The oracle's tool setup gives the reference's face, vertex and edge normals,
  normal flip and triangle grid: its FP32 form bit for bit, its FP64 form the
  same grid with normals within FP32 rounding.
* (GPU) The library's own tool setup does the same, and a block cut by the
  reference's pin25 grain mesh steps within the FP64 oracle's tolerances.
"""
import os

import numpy as np
import pytest

import oracle
from iwf_mfree_gpu_3d_b200 import api, scenes

from helpers import check, compare, gpu_state, hex_block_k, oracle_state

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden", "ref_setup.npz")
ASSETS = {"cube_rot": ("cube_rot.json", False), "sphere_coarse": ("sphere_coarse.json", False),
          "pin25": ("pin25_reduziert_20062018.k", False),
          "diamant": ("Diamant_von_Mansur_04072018_SDB1125-2025-D851.k", False)}
MESHES = ["cube_rot", "sphere_coarse", "pin25", "diamant", "hex_block", "wedge", "grain"]


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLD)


def mesh(gold, name):
    return gold[f"{name}_verts"], gold[f"{name}_tris"]


def tool_scene(V, T) -> "scenes.Scene":
    sc = scenes.orthogonal_cutting(6, 4, 4)
    sc.tools = [scenes.Tool(verts=np.asarray(V, np.float32), tris=np.asarray(T, np.int32),
                            vel=np.array([-1e-3, 0.0, 0.0], np.float32))]
    return sc


def expect_tool(gold, name, info, normals, cells, boxed, rtol: float = 0.0):
    """The tool setup equals the reference's: the triangle grid exactly, the
    normals, box and cell edge bit for bit (rtol = 0) or within rtol."""
    g = lambda k: gold[f"{name}_tool_{k}"]  # noqa: E731
    assert tuple(info["n3"]) == tuple(int(x) for x in g("n3")), (name, info["n3"], g("n3"))
    assert info["num_boxed"] == len(g("boxed")), name
    np.testing.assert_array_equal(cells, g("cells"), err_msg=name)
    np.testing.assert_array_equal(boxed, g("boxed"), err_msg=name)
    for got, want in ((info["bbmin"], g("bbmin")), (info["bbmax"], g("bbmax")), (info["dx"], g("dx")),
                      (np.asarray(normals, np.float64).reshape(-1, 21), g("normals"))):
        if rtol == 0.0:
            np.testing.assert_array_equal(np.float32(got), want, err_msg=name)
        else:  # unit normals and coordinates: relative to the largest entry
            want = np.asarray(want, np.float64)
            np.testing.assert_allclose(np.asarray(got, np.float64), want, rtol=0,
                                       atol=rtol * max(np.abs(want).max(), 1e-30), err_msg=name)


@pytest.mark.parametrize("name", list(ASSETS))
def test_readers_give_the_reference_readers_output_on_its_assets(gold, name):
    path = os.path.join(oracle.reference_root(), "Release", ASSETS[name][0])
    if not os.path.exists(path):
        pytest.skip("the reference checkout (its Release/ meshes) is not at hand")
    V, T = api.read_mesh(path, hexahedra=ASSETS[name][1])
    gv, gt = mesh(gold, name)
    np.testing.assert_array_equal(V, gv)
    np.testing.assert_array_equal(T, gt)


def test_hexahedral_reader_gives_the_reference_readers_output(gold, tmp_path):
    p = tmp_path / "hex.k"
    p.write_text(hex_block_k())
    V, T = api.read_mesh(str(p), hexahedra=True)
    gv, gt = mesh(gold, "hex_block")
    assert len(T) == 2 * 2 * (3 * 2 + 3 * 2 + 2 * 2)  # two triangles per boundary face of a 3x2x2 block
    np.testing.assert_array_equal(V, gv)
    np.testing.assert_array_equal(T, gt)


def test_hexahedral_reader_rejects_tetrahedral_lines(tmp_path):
    p = tmp_path / "short.k"
    p.write_text("*NODE\n 1 0 0 0\n*ELEMENT_SOLID\n 1 1 1 2 3 4\n*END\n")
    with pytest.raises(api.MfreeError):
        api.read_mesh(str(p), hexahedra=True)


@pytest.mark.parametrize("prec", [32, 64])
@pytest.mark.parametrize("name", MESHES)
def test_oracle_tool_setup_is_the_reference_tool_setup(oracle_lib, gold, name, prec):
    orc = oracle.Oracle(tool_scene(*mesh(gold, name)), prec=prec)
    cells, boxed = orc.tool_cells(0)
    # the FP32 form is the reference's arithmetic; the FP64 form computes the
    # normals and the grid box in double (measured within 6e-6 of the largest
    # entry) and must still give the same grid
    expect_tool(gold, name, orc.tool_info(0), orc.tool_normals(0), cells, boxed, rtol=0.0 if prec == 32 else 2e-5)


@pytest.mark.gpu
@pytest.mark.parametrize("name", MESHES)
def test_library_tool_setup_is_the_reference_tool_setup(gold, name):
    sim = api.Simulation.from_scene(tool_scene(*mesh(gold, name)))
    cells, boxed = sim.tool_cells(0)
    expect_tool(gold, name, sim.tool_info(0), sim.tool_normals(0), cells, boxed)
    sim.close()


@pytest.mark.gpu
def test_cutting_with_the_reference_pin25_grain_mesh():
    """A 30x15x10 block cut by the reference's own LS-DYNA grain mesh (placed as
    its single-grain setup places it), 100 steps against the FP64 oracle."""
    V, T = mesh(np.load(GOLD), "pin25")
    # its flat bottom face ends 2.1 dx behind its front, whose lowest point is
    # 2 dx higher: place the front just inside the top layer (0.05 dx) and the
    # bottom face just outside the block's -x face, so the first contact is as
    # gentle as the wedge scenes'
    dx = 1e-3
    zb = V[:, 2].min()
    xb = V[V[:, 2] == zb, 0].max()
    zf = V[V[:, 0] > xb, 2].min()
    sc = scenes.mesh_tool_scene(V, T, depth=(zf - zb) / dx + 0.05, engage=(V[:, 0].max() - xb) / dx - 0.05)
    sim = api.Simulation.from_scene(sc)
    orc = oracle.Oracle(sc, prec=64)
    # the first step's contact: the particles the grain overlaps are pushed out
    sim.step(record_forces=True)
    orc.step(record=True)
    fg, fo = np.asarray(sim.tool_forces(), np.float64), orc.tool_forces().astype(np.float64)
    assert np.linalg.norm(fo) > 0, "the grain must start in contact"
    assert np.linalg.norm(fg - fo) < 1e-5 * np.linalg.norm(fo), (fg, fo)
    for k in range(99):
        sim.step()
        orc.step()
    err = compare(gpu_state(sim), oracle_state(orc), sc)
    g = gpu_state(sim)
    sim.close()
    print("pin25 grain, 100-step relative L2:", {k: f"{v:.2e}" for k, v in err.items()})
    check(err, "pin25_100")
    # the reference's own GPU step on the same scene, when built
    from baseline import refgpu
    if refgpu.available(refgpu.variant_of(sc)):
        st = refgpu.run(sc, 0, 100, state=True)["state"]
        ids = st["ID"]
        names = ["POS", "VEL", "S", "EPS_PL", "T", "RHO"]
        r = {}
        for n in names + ["BLANKED"]:
            r[n] = np.empty(st[n].shape, np.float64)
            r[n][ids] = st[n]
        e_ref = compare(r, oracle_state(orc, names), sc, names)
        e_cuda = compare(g, r, sc, names)
        print("reference GPU step vs FP64 oracle:", {k: f"{v:.2e}" for k, v in e_ref.items()})
        print("CUDA path vs reference GPU step:", {k: f"{v:.2e}" for k, v in e_cuda.items()})
        check(e_ref, "pin25_100")
        check(e_cuda, "pin25_100")
