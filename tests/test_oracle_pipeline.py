"""CPU checks of the oracle's integer pipeline and of its step invariants."""
import numpy as np
import pytest

import oracle
from iwf_mfree_gpu_3d_b200 import scenes


def _grid(sc):
    orc = oracle.Oracle(sc, prec=32)
    return orc.grid()


def test_hash_matches_reference_formula_and_sort_is_stable():
    sc = scenes.small_scene()
    (nx, ny, nz), lo, dx = _grid(sc)
    rng = np.random.default_rng(5)
    pos = sc.pos.copy()
    pos[:, :3] += rng.normal(scale=0.4e-3, size=(sc.n, 3)).astype(np.float32)
    blanked = (rng.random(sc.n) < 0.01).astype(np.float32)
    h = oracle.hash_fp32(pos, blanked, np.array(lo, np.float32), dx, (nx, ny, nz))
    lo32 = np.array(lo, np.float32)
    ix = ((pos[:, 0] - lo32[0]) / np.float32(dx)).astype(np.int32)
    iy = ((pos[:, 1] - lo32[1]) / np.float32(dx)).astype(np.int32)
    iz = ((pos[:, 2] - lo32[2]) / np.float32(dx)).astype(np.int32)
    ref = ix * ny * nz + iy * nz + iz
    ref[blanked == 1] = np.iinfo(np.int32).max
    np.testing.assert_array_equal(h, ref)
    n_act = int((blanked == 0).sum())
    idx, sh, cs, ce = oracle.sort_cells(h, n_act, nx * ny * nz)
    np.testing.assert_array_equal(idx, np.argsort(h, kind="stable"))
    np.testing.assert_array_equal(sh, h[idx])
    # cell ranges: -1 for empty, [start, end) covering exactly the cell's particles
    occ = np.unique(sh[:n_act])
    assert (cs[occ] >= 0).all()
    empty = np.setdiff1d(np.arange(nx * ny * nz), occ)
    assert (cs[empty] == -1).all() and (ce[empty] == -1).all()
    for c in occ[:: max(1, len(occ) // 200)]:
        assert (sh[cs[c]:ce[c]] == c).all()
        assert (cs[c] == 0 or sh[cs[c] - 1] != c) and (ce[c] == n_act or sh[ce[c]] != c)


def test_neighbor_counts_brute_force():
    sc = scenes.orthogonal_cutting(12, 8, 6)
    (nx, ny, nz), lo, dx = _grid(sc)
    h = oracle.hash_fp32(sc.pos, None, np.array(lo, np.float32), dx, (nx, ny, nz))
    idx, sh, cs, ce = oracle.sort_cells(h, sc.n, nx * ny * nz)
    p = sc.pos[idx]
    cnt = oracle.neighbor_counts_fp32(p, sc.h[idx], sh, cs, ce, sc.n, (nx, ny, nz))
    d = p[:, None, :3] - p[None, :, :3]
    r2 = ((d[..., 0] * d[..., 0] + d[..., 1] * d[..., 1]) + d[..., 2] * d[..., 2]).astype(np.float32)
    hh = sc.h[idx][:, None]
    four = (np.float32(4.0) * hh) * hh
    brute = ((r2 < four) & (r2 > np.float32(9.99999994e-9))).sum(1)
    np.testing.assert_array_equal(cnt, brute)
    assert 30 < cnt.mean() < 81


def test_fp32_and_fp64_oracles_agree_over_steps():
    sc = scenes.orthogonal_cutting(16, 8, 6)
    a = oracle.Oracle(sc, prec=64)
    b = oracle.Oracle(sc, prec=32)
    for _ in range(20):
        a.step()
        b.step()
    ia, ib = a.field("ID").astype(int), b.field("ID").astype(int)
    pa = np.empty((sc.n, 4)); pa[ia] = a.field("POS")
    pb = np.empty((sc.n, 4)); pb[ib] = b.field("POS")
    va = np.empty((sc.n, 4)); va[ia] = a.field("VEL")
    vb = np.empty((sc.n, 4)); vb[ib] = b.field("VEL")
    d0 = sc.pos[:, :3]
    e = np.linalg.norm((pa - pb)[:, :3]) / np.linalg.norm(pa[:, :3] - d0)
    ev = np.linalg.norm(va - vb) / np.linalg.norm(va)
    assert e < 1e-2 and ev < 1e-2


def test_oracle_step_invariants():
    sc = scenes.small_scene()
    o = oracle.Oracle(sc, prec=64)
    for _ in range(10):
        o.step()
    ids = o.field("ID").astype(int)
    assert sorted(ids) == list(range(sc.n))
    fixed = o.field("FIXED")
    v = o.field("VEL")
    assert np.abs(v[fixed == 1]).max() == 0.0        # fixed particles carry vel_bc = 0
    T = o.field("T")
    assert np.all(T[fixed == 1] == 300.0)             # thermal boundary condition
    S = o.field("S").reshape(-1, 3, 3)
    np.testing.assert_array_equal(S, np.transpose(S, (0, 2, 1)))
    assert o.counts() == (sc.n, sc.n)


def test_tool_setup_oracle_wedge():
    sc = scenes.small_scene()
    o = oracle.Oracle(sc, prec=32)
    info = o.tool_info()
    assert info["num_tris"] == 12 and info["num_boxed"] >= 12
    nrm = o.tool_normals()
    np.testing.assert_allclose(np.linalg.norm(nrm, axis=2), 1.0, atol=1e-6)
    # normals point into the tool after the flip test (tool_3d.cpp:321-358)
    v = sc.tools[0].verts.astype(np.float64)
    t = sc.tools[0].tris
    centre = v.mean(0)
    fc = v[t].mean(1)
    assert np.all(np.einsum("ij,ij->i", nrm[:, 0], centre - fc) > 0)
    cells, src = o.tool_cells()
    assert cells[-1] == info["num_boxed"] and set(src) == set(range(12))


def test_oracle_unlocked_grid_follows_the_particles():
    """grid_gpu_green(max_cell, N): the oracle's grid after a step is the
    bounding box of the particles at its start (FP32 build arithmetic), and
    the FP32 and FP64 oracles with an unlocked grid still agree."""
    from helpers import unlocked_grid
    sc = scenes.orthogonal_cutting(16, 8, 6)
    sc.grid_max_cell = 100000
    b = oracle.Oracle(sc, prec=32)
    b.step()
    n3, bbmin, dx = unlocked_grid(sc.pos, sc.h, sc.n)
    g_n3, g_lo, g_dx = b.grid()
    assert tuple(int(v) for v in g_n3) == n3
    np.testing.assert_array_equal(np.float32(g_lo), bbmin)
    assert np.float32(g_dx) == dx
    a = oracle.Oracle(sc, prec=64)
    a.step()
    for _ in range(15):
        a.step()
        b.step()
    ia, ib = a.field("ID").astype(int), b.field("ID").astype(int)
    pa = np.empty((sc.n, 4)); pa[ia] = a.field("POS")
    pb = np.empty((sc.n, 4)); pb[ib] = b.field("POS")
    d0 = sc.pos[:, :3]
    assert np.linalg.norm((pa - pb)[:, :3]) / np.linalg.norm(pa[:, :3] - d0) < 1e-2


def test_oracle_unlocked_grid_beyond_max_cell_fails():
    sc = scenes.orthogonal_cutting(16, 8, 6)
    sc.grid_max_cell = 100
    o = oracle.Oracle(sc, prec=32)
    with pytest.raises(RuntimeError):
        o.step()
