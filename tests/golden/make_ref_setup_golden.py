"""Generate tests/golden/ref_setup.npz from the reference's own scene setup.

Outputs come from oracle/_ref/libref_host.so: the reference's readers
(json_read_triangles, ldynak_read_triangles_from_tetmesh and _quadmesh) and
tool setup (mesh_compute_vertex_normals, mesh_average_edge_length, tool_3d:
normal flip and triangle grid) compiled unchanged from its sources by
oracle/build_ref.sh.  Inputs:

  * the reference's own mesh assets, Release/cube_rot.json,
    Release/sphere_coarse.json, Release/pin25_reduziert_20062018.k and
    Release/Diamant_von_Mansur_04072018_SDB1125-2025-D851.k, read from the
    reference checkout (the file stores what the reference's readers make of
    them: vertices and triangles in the reader's order);
  * a seeded hexahedral block (tests/helpers.py ``hex_block_k``) for the
    hexahedral reader;
  * the tool meshes of the benchmark scenes (scenes.py: the wedge and the
    truncated-icosphere grain).

For every mesh it also stores the reference's tool setup: per triangle the
face, vertex and edge normals, the triangle grid (cells, boxed triangles as
input indices, cell counts, box, cell edge) and the mesh's average edge length.
Run in a checkout that has the reference sources:
  python tests/golden/make_ref_setup_golden.py
"""
import ctypes as C
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

import oracle  # noqa: E402
from helpers import hex_block_k  # noqa: E402
from iwf_mfree_gpu_3d_b200 import scenes  # noqa: E402

ASSETS = {"cube_rot": ("cube_rot.json", "json"), "sphere_coarse": ("sphere_coarse.json", "json"),
          "pin25": ("pin25_reduziert_20062018.k", "tet"),
          "diamant": ("Diamant_von_Mansur_04072018_SDB1125-2025-D851.k", "tet")}


def ref_host():
    lib = os.path.join(ROOT, "oracle", "_ref", "libref_host.so")
    if not os.path.exists(lib):
        raise SystemExit("oracle/_ref/libref_host.so is missing (build it with oracle/build_ref.sh)")
    return C.CDLL(lib)


def ref_read(R, kind: str, path: str):
    fn = {"json": R.ref_read_json, "tet": R.ref_read_ldynak_tet, "quad": R.ref_read_ldynak_quad}[kind]
    v, t = C.POINTER(C.c_float)(), C.POINTER(C.c_int)()
    nv, nt = C.c_int(), C.c_int()
    fn(path.encode(), C.byref(v), C.byref(nv), C.byref(t), C.byref(nt))
    V = np.ctypeslib.as_array(v, (3 * nv.value,)).reshape(-1, 3).copy()
    T = np.ctypeslib.as_array(t, (3 * nt.value,)).reshape(-1, 3).copy()
    R.ref_free(v)
    R.ref_free(t)
    return V.astype(np.float32), T.astype(np.int32)


def ref_tool(R, V, T):
    R.ref_tool_setup.restype = C.c_float
    fp = C.POINTER(C.c_float)
    ip = C.POINTER(C.c_int)
    V = np.ascontiguousarray(V, np.float32)
    T = np.ascontiguousarray(T, np.int32)
    h = R.ref_tool_setup(V.ctypes.data_as(fp), len(V), T.ctypes.data_as(ip), len(T))
    n3 = np.zeros(3, np.int32)
    lo = np.zeros(3, np.float32)
    hi = np.zeros(3, np.float32)
    dx = C.c_float()
    nc, nb = C.c_int(), C.c_int()
    R.ref_tool_info(n3.ctypes.data_as(ip), lo.ctypes.data_as(fp), hi.ctypes.data_as(fp), C.byref(dx), C.byref(nc),
                    C.byref(nb))
    normals = np.zeros((len(T), 21), np.float32)
    cells = np.zeros(nc.value + 1, np.int32)
    boxed = np.zeros(nb.value, np.int32)
    R.ref_tool_arrays(normals.ctypes.data_as(fp), cells.ctypes.data_as(ip), boxed.ctypes.data_as(ip))
    return dict(normals=normals, cells=cells, boxed=boxed, n3=n3, bbmin=lo, bbmax=hi,
                dx=np.float32(dx.value), h=np.float32(h))


def meshes(R, ref_root: str):
    out = {}
    for name, (fname, kind) in ASSETS.items():
        out[name] = ref_read(R, kind, os.path.join(ref_root, "Release", fname))
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "hex.k")
        with open(p, "w") as f:
            f.write(hex_block_k())
        out["hex_block"] = ref_read(R, "quad", p)
    w = scenes.small_scene().tools[0]
    out["wedge"] = (w.verts.astype(np.float32), w.tris.astype(np.int32))
    g = scenes.single_grain(40, 20, 12, tool_particles=False).tools[0]
    out["grain"] = (g.verts.astype(np.float32), g.tris.astype(np.int32))
    return out


def main():
    R = ref_host()
    root = oracle.reference_root()
    data = {}
    for name, (V, T) in meshes(R, root).items():
        data[f"{name}_verts"] = V
        data[f"{name}_tris"] = T
        for k, v in ref_tool(R, V, T).items():
            data[f"{name}_tool_{k}"] = v
    out = os.path.join(HERE, "ref_setup.npz")
    np.savez_compressed(out, **data)
    print("wrote", out)


if __name__ == "__main__":
    main()
