"""The no-allocation pressure solve (pvof_Pressure_solve_cg_noalloc).

Some callers cannot call cudaMalloc -- they own a fixed device pool, or run
where allocation is not allowed -- so this entry point takes the caller's
device buffers and keeps every temporary in a fixed array inside the
library.  This test calls it through the C ABI, twice in a row, and checks
the correction against the context-based entry points
(pvof_Pressure_compute_preconditioner + pvof_Pressure_solve_cg) on the same
inputs, within the tolerance the parity tests use (relative L2 1e-12 with the
solver converged to near machine precision).  The test allocates its device
buffers with torch; the entry point itself allocates nothing.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu


def _case(kind):
    from pvof import cases
    if kind == "planar":
        return cases.rayleigh_taylor(128, 512, Lx=1.0, Ly=4.0, Cn=0.01, velocity_seed=6, velocity_amp=0.05,
                                     P_CG_ETOL=1e-6, P_CG_MAXIT=4000)
    # axisymmetric: the radius tables (r_u, r_c, 1/r_c) and the row-weighted
    # right-hand side take a branch of their own
    return cases.rising_bubble(NXM=96, NYM=192, rmax=1.0, zmax=2.0, radius=0.3, zc=0.7, Cn=0.02, velocity_seed=4,
                               velocity_amp=0.05, P_CG_ETOL=1e-9, P_CG_MAXIT=4000)


@pytest.mark.parametrize("kind", ["planar", "axisym"])
def test_noalloc_pressure_solve_matches_context_solve(kind):
    import torch
    from pvof import abi, cases, runtime

    grid, params, planes = _case(kind)
    g = runtime.Solver(grid, params, device=0)
    g.set_cluster_solvers(False)   # the grid-wide kernel, as the entry point uses
    g.set_pressure_pairs(0)        # one cell per thread and trip, the entry point's summation order
    g.set_planes(planes)
    g.initialize()
    g.set_stage(1, 1e-4)
    g.call("Pressure_set_RHS")
    rho = g.get("RHO")
    rhs = g.get("P_RHS")
    g.call("Pressure_compute_preconditioner")
    st = abi.Stats()
    it_ctx = g.call("Pressure_solve_cg", C.byref(st))
    ref = g.get("DELTAP")
    assert 0 < it_ctx < params.P_CG_MAXIT
    NX, NY, _ = cases.dims(grid)
    assert rho.shape == (NY + 6, NX + 6)

    L = runtime.load()
    L.pvof_Pressure_solve_cg_noalloc.argtypes = [C.POINTER(abi.GridDesc), C.POINTER(abi.Params), C.c_void_p,
                                                 C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(C.c_int),
                                                 C.POINTER(C.c_double)]
    L.pvof_noalloc_last_error.restype = C.c_char_p
    torch.cuda.set_device(0)
    d_rho = torch.from_numpy(np.ascontiguousarray(rho)).cuda()
    d_rhs = torch.from_numpy(np.ascontiguousarray(rhs)).cuda()
    interior = (slice(3, 3 + NY - 1), slice(3, 3 + NX - 1))
    for call in range(2):
        d_phi = torch.zeros_like(d_rho)
        torch.cuda.synchronize()
        its, res = C.c_int(), C.c_double()
        rc = L.pvof_Pressure_solve_cg_noalloc(C.byref(grid), C.byref(params), d_rho.data_ptr(), d_rhs.data_ptr(),
                                              d_phi.data_ptr(), None, C.byref(its), C.byref(res))
        assert rc >= 0, L.pvof_noalloc_last_error()
        phi = d_phi.cpu().numpy()
        assert abs(its.value - it_ctx) <= 2, (call, its.value, it_ctx)
        assert rel_l2(phi[interior], ref[interior]) <= 1e-12, (call, rel_l2(phi[interior], ref[interior]))
        assert res.value < params.P_CG_ETOL
        assert abs(res.value - st.p_res) <= 1e-12 * st.p_res

    # a grid beyond the fixed scratch is refused, not run
    big, bparams, _ = cases.rayleigh_taylor(512, 512, Lx=1.0, Ly=1.0, Cn=0.01)
    rc = L.pvof_Pressure_solve_cg_noalloc(C.byref(big), C.byref(bparams), d_rho.data_ptr(), d_rhs.data_ptr(),
                                          d_rho.data_ptr(), None, None, None)
    assert rc == abi.EINVAL
    assert b"72000" in L.pvof_noalloc_last_error()
    # so is an axisymmetric grid whose radial direction is marked periodic
    if kind == "axisym":
        bad = abi.GridDesc.from_buffer_copy(grid)
        bad.periodic[0] = 1
        rc = L.pvof_Pressure_solve_cg_noalloc(C.byref(bad), C.byref(params), d_rho.data_ptr(), d_rhs.data_ptr(),
                                              d_rho.data_ptr(), None, None, None)
        assert rc == abi.EINVAL
        assert b"axis" in L.pvof_noalloc_last_error()
