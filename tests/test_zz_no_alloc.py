"""mfree_cell_list_static: the cell-list build for callers that cannot
allocate device memory while they run (a host whose device memory is reserved
up front by its own allocator, or code that cannot afford the device
synchronisation a cudaMalloc may cause).  Its scratch is a fixed-size
__device__ array of the library.

The test calls it through the C ABI twice in a row on the same positions and
compares both results with the cell-list build of the existing entry point
(mfree_step's sort permutation and cell ranges): integer outputs, so bit-exact.
This file is collected last, so a run that stops at the first failure has run
every other test before it.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_static_cell_list_matches_the_step_on_two_calls():
    import torch

    from iwf_mfree_gpu_3d_b200 import api, scenes

    sc = scenes.small_scene()
    sim = api.Simulation.from_scene(sc)
    (nx, ny, nz), lo, dx = sim.grid()
    ncell = nx * ny * nz
    pos = sim.get("POS")  # positions the first step sorts (creation order)
    sim.step()
    idx_ref = sim.get("IDX")
    cs, ce = sim.cells()
    sim.close()
    first_ref = np.concatenate([[0], np.cumsum(np.where(cs >= 0, ce - cs, 0))]).astype(np.int32)

    L = api.lib()
    dev = torch.device("cuda:0")
    d_pos = torch.from_numpy(np.ascontiguousarray(pos, np.float32)).to(dev)
    bbmin = (C.c_float * 3)(*lo)
    for call in range(2):
        d_perm = torch.full((sc.n,), -7, dtype=torch.int32, device=dev)
        d_first = torch.full((ncell + 1,), -7, dtype=torch.int32, device=dev)
        torch.cuda.synchronize()
        st = L.mfree_cell_list_static(C.c_void_p(d_pos.data_ptr()), sc.n, bbmin, float(dx), nx, ny, nz,
                                      C.c_void_p(d_perm.data_ptr()), C.c_void_p(d_first.data_ptr()), None)
        assert st == 0, (call, L.mfree_last_error())
        torch.cuda.synchronize()
        np.testing.assert_array_equal(d_perm.cpu().numpy(), idx_ref, err_msg=f"call {call}")
        np.testing.assert_array_equal(d_first.cpu().numpy(), first_ref, err_msg=f"call {call}")


def test_static_cell_list_rejects_sizes_beyond_its_limits():
    from iwf_mfree_gpu_3d_b200 import api

    L = api.lib()
    bbmin = (C.c_float * 3)(0.0, 0.0, 0.0)
    dummy = C.c_void_p(16)  # never dereferenced: the size check comes first
    st = L.mfree_cell_list_static(dummy, 262144 + 1, bbmin, 1.0, 4, 4, 4, dummy, dummy, None)
    assert st == -1 and b"static limit" in L.mfree_last_error()
    st = L.mfree_cell_list_static(dummy, 1000, bbmin, 1.0, 1000, 1000, 1, dummy, dummy, None)
    assert st == -1 and b"static limit" in L.mfree_last_error()


def _expected_cell_list(pos, lo, dx, n3):
    """Cell list of the same positions restated in numpy: float32 IEEE
    subtraction and division as the device hash, truncation toward zero, a
    stable sort by cell id, positions outside the grid or not finite last."""
    nx, ny, nz = n3
    ncell = nx * ny * nz
    p = np.asarray(pos, np.float32)[:, :3]
    with np.errstate(invalid="ignore", over="ignore"):
        q = (p - np.asarray(lo, np.float32)) / np.float32(dx)
        finite = np.all(np.isfinite(p), axis=1)
        ijk = np.trunc(np.where(np.isfinite(q), q, -1.0)).astype(np.int64)
    inside = finite & np.all((ijk >= 0) & (ijk < np.array([nx, ny, nz])), axis=1)
    key = np.where(inside, (ijk[:, 0] * ny + ijk[:, 1]) * nz + ijk[:, 2], ncell)
    perm = np.argsort(key, kind="stable").astype(np.int32)
    counts = np.bincount(key[inside], minlength=ncell)
    first = np.concatenate([[0], np.cumsum(counts)]).astype(np.int32)
    return perm, first


def test_static_cell_list_sends_outside_and_nan_positions_to_the_tail():
    import torch

    from iwf_mfree_gpu_3d_b200 import api

    rng = np.random.default_rng(5)
    n3 = (9, 7, 5)
    lo = (-0.25, 0.5, -1.0)
    dx = 0.125
    n = 3000
    hi = np.array(lo) + dx * np.array(n3)
    pos = np.zeros((n, 4), np.float32)
    # most positions inside, some beyond each face, some less than a cell
    # below the lower corner (cell 0 by truncation), some NaN and infinite
    pos[:, :3] = rng.uniform(np.array(lo) - 1.5 * dx, hi + 1.5 * dx, size=(n, 3))
    pos[::97, 0] = np.nan
    pos[5::101, 2] = np.inf
    pos[7::103, 1] = -np.inf
    exp_perm, exp_first = _expected_cell_list(pos, lo, dx, n3)
    assert exp_first[-1] < n - 200  # the tail holds out-of-grid and non-finite positions

    L = api.lib()
    dev = torch.device("cuda:0")
    d_pos = torch.from_numpy(pos).to(dev)
    bbmin = (C.c_float * 3)(*lo)
    ncell = n3[0] * n3[1] * n3[2]
    for call in range(2):
        d_perm = torch.full((n,), -7, dtype=torch.int32, device=dev)
        d_first = torch.full((ncell + 1,), -7, dtype=torch.int32, device=dev)
        torch.cuda.synchronize()
        st = L.mfree_cell_list_static(C.c_void_p(d_pos.data_ptr()), n, bbmin, float(dx), *n3,
                                      C.c_void_p(d_perm.data_ptr()), C.c_void_p(d_first.data_ptr()), None)
        assert st == 0, (call, L.mfree_last_error())
        torch.cuda.synchronize()
        np.testing.assert_array_equal(d_perm.cpu().numpy(), exp_perm, err_msg=f"call {call}")
        np.testing.assert_array_equal(d_first.cpu().numpy(), exp_first, err_msg=f"call {call}")
