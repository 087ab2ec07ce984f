"""The allocation-free compliance entry point t3d_compliance_noalloc, called through the C-ABI on
device buffers the caller owns, agrees with the context-based t3d_compliance on the same inputs.

It exists for callers that cannot allocate device memory when they call the library (hosts that own
the whole device heap, serving loops that must not enter the allocator, callers without a context):
its only scratch is a static device array, so the test also checks two calls in a row with different
inputs (the shared scratch and its arrival counter are reused).  Element compliances must be
bit-identical (same per-element arithmetic); the total C is summed in a different order (one partial
per 256 cells instead of the context path's fixed grid), so it must agree to 1e-13 relative.
This file is collected last on purpose, and it does not depend on any other test.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def grid_layout(P):
    """index maps from the reference layouts (Morton elements, free DOFs) to the device grid layout"""
    nx, ny, nz = P.res
    full = P.ele_map_back().astype(np.int64)          # ny*nx*cz + ny*cx + cy
    cz, rem = np.divmod(full, nx * ny)
    cx, cy = np.divmod(rem, ny)
    cell = ((cz + 1) * (ny + 2) + cy + 1) * (nx + 2) + cx + 1
    ncell_arr = (nx + 2) * (ny + 2) * (nz + 2)
    NN = (nx + 1) * (ny + 1) * (nz + 1)
    fd = P.free_dofs().astype(np.int64)
    node_idx = (fd % 3) * NN + fd // 3
    return cell, ncell_arr, node_idx, 3 * NN


@pytest.mark.parametrize("dims", [(10, 20, 10), (30, 60, 30)])
def test_noalloc_compliance_matches_context_path(dims):
    import torch
    import algorithmengineering_altproject_b200 as t3d

    lib = t3d.library()
    P = t3d.Problem(*dims)
    cell, ncell_arr, node_idx, nvec = grid_layout(P)
    ke = np.ascontiguousarray(P.ke().ravel())
    rng = np.random.default_rng(2026)
    stream = torch.cuda.current_stream()
    for call in range(2):
        E = rng.uniform(1e-6, 1.0, P.ne) * (1.0 + call)
        u = rng.standard_normal(P.nf)
        C_ref, ce_ref = P.ComputeCompliance(E, u)

        Eg = np.zeros(ncell_arr)
        Eg[cell] = E
        ug = np.zeros(nvec)
        ug[node_idx] = u
        dE = torch.tensor(Eg, dtype=torch.float64, device="cuda")
        du = torch.tensor(ug, dtype=torch.float64, device="cuda")
        dce = torch.full((ncell_arr,), float("nan"), dtype=torch.float64, device="cuda")
        dC = torch.full((1,), float("nan"), dtype=torch.float64, device="cuda")
        nely, nelx, nelz = dims
        rc = lib.t3d_compliance_noalloc(nely, nelx, nelz, ke, C.c_void_p(dE.data_ptr()), C.c_void_p(du.data_ptr()),
                                        C.c_void_p(dce.data_ptr()), C.c_void_p(dC.data_ptr()),
                                        C.c_void_p(stream.cuda_stream))
        assert rc == 0, lib.t3d_last_error().decode()
        stream.synchronize()
        ce = dce.cpu().numpy()[cell]
        C_na = float(dC.cpu().item())
        np.testing.assert_array_equal(ce, ce_ref)
        assert abs(C_na - C_ref) <= 1e-13 * abs(C_ref), (call, C_na, C_ref)


def test_noalloc_rejects_grids_beyond_its_scratch():
    import algorithmengineering_altproject_b200 as t3d

    lib = t3d.library()
    ke = np.zeros(576)
    dummy = C.c_void_p(16)   # never dereferenced: the size check fails first
    rc = lib.t3d_compliance_noalloc(256, 512, 256, ke, dummy, dummy, dummy, dummy, None)
    assert rc == t3d.T3D_ERR_UNSUPPORTED
    assert "too large" in lib.t3d_last_error().decode()
