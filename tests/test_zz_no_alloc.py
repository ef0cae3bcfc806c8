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
