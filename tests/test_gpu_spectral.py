"""The spectral pressure preconditioner (pvof_params.pressure_preconditioner = 1)
against the reference's Jacobi-PCG.

  constant density      the preconditioner is the exact inverse of the
                        operator: every pressure solve stops within two
                        iterations (the second clears rounding at a 1e-13
                        tolerance), and its correction equals the Jacobi-PCG's
                        (both solved to 1e-13) within 1e-9 relative L2
  two-phase instability after 20 steps the fields stay within 1e-7 relative
                        L2 of the Jacobi path (both stop at the reference's
                        absolute tolerance on sqrt(r^T D^-1 r)); the spectral
                        form needs at least 5x fewer pressure iterations
  unsupported grids     refused at creation (PVOF_EINVAL)
  resolved cylinders    all four forms against the plain path: fields within
                        2e-6 (measured 7e-7 for the velocity, 1e-8 for C_L and
                        P: the flow starts at rest and the plain path's
                        stalled momentum residual is a share of the still
                        small velocity), positions within 1e-9 after 6 steps
"""
import numpy as np
import pytest

from conftest import g_range, physical

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def one_substep(grid, params, planes, precond):
    from pvof import runtime
    params.pressure_preconditioner = precond
    s = runtime.Solver(grid, params, device=0)
    s.set_planes(planes)
    s.initialize()
    s.set_stage(0, 1e-3)
    st = s.substep()
    out = {f: physical(grid, g_range(grid, s.get(f)), f) for f in ("DELTAP", "U", "V")}
    s.close()
    return st, out


def test_constant_density_is_solved_in_two_iterations():
    from pvof import cases
    grid, params, planes = cases.rayleigh_taylor(64, 128, Lx=1.0, Ly=2.0, Cn=0.04, atwood=0.0, velocity_seed=5,
                                                 velocity_amp=0.05, P_CG_MAXIT=5000, P_CG_ETOL=1e-13)
    st_j, a = one_substep(grid, params, planes, 0)
    st_s, b = one_substep(grid, params, planes, 1)
    print("pressure iterations: Jacobi %d, spectral %d (passes %d, %d)"
          % (st_j.p_iters_total, st_s.p_iters_total, st_j.poisson_passes, st_s.poisson_passes))
    assert st_s.p_iters_total <= 2 * st_s.poisson_passes
    assert st_j.p_iters_total > 20 * st_s.p_iters_total
    for f in ("DELTAP", "U", "V"):
        assert rel(b[f], a[f]) <= 1e-9, (f, rel(b[f], a[f]))


@pytest.mark.parametrize("NXM", [96, 80, 48])
def test_mixed_radix_widths_solve_constant_density_exactly(NXM):
    """x cell counts 3 x 2^a and 5 x 2^a (the row transforms' radix-3 and
    radix-5 combining pass): at constant density the preconditioner is still
    the operator's exact inverse, two iterations per solve, and the correction
    equals the Jacobi-PCG's within 1e-9."""
    from pvof import cases
    grid, params, planes = cases.rayleigh_taylor(NXM, 2 * NXM, Lx=1.0, Ly=2.0, Cn=0.04, atwood=0.0, velocity_seed=5,
                                                 velocity_amp=0.05, P_CG_MAXIT=5000, P_CG_ETOL=1e-13)
    st_j, a = one_substep(grid, params, planes, 0)
    st_s, b = one_substep(grid, params, planes, 1)
    print("NXM %d: pressure iterations Jacobi %d, spectral %d" % (NXM, st_j.p_iters_total, st_s.p_iters_total))
    assert st_s.p_iters_total <= 2 * st_s.poisson_passes
    for f in ("DELTAP", "U", "V"):
        assert rel(b[f], a[f]) <= 1e-9, (f, rel(b[f], a[f]))


def test_spectral_form_stays_within_tolerance_of_jacobi():
    from pvof import cases, runtime
    grid, params, planes = cases.rayleigh_taylor(128, 512, Lx=1.0, Ly=4.0, Cn=0.01, P_CG_MAXIT=2000)
    out = {}
    for precond in (0, 1):
        params.pressure_preconditioner = precond
        s = runtime.Solver(grid, params, device=0)
        s.set_planes(planes)
        s.initialize()
        iters = 0
        for n in range(20):
            for rk in range(3):
                if n > 0 and rk == 0:
                    s.call("Velocity_cell_center")
                s.set_stage(rk, 1e-4)
                iters += s.substep().p_iters_total
        out[precond] = (iters, {f: physical(grid, g_range(grid, s.get(f)), f) for f in ("C_L", "U", "V", "P")})
        s.close()
    print("pressure iterations over 20 steps: Jacobi %d, spectral %d" % (out[0][0], out[1][0]))
    for f in ("C_L", "U", "V", "P"):
        r = rel(out[1][1][f], out[0][1][f])
        print("%s rel L2 %.2e" % (f, r))
        assert r <= 1e-7, (f, r)
    assert 5 * out[1][0] <= out[0][0]


def test_wide_grid():
    """1024 x cells (the widest supported; eight rows of them fill 128 KB of
    shared memory per block): the correction equals the Jacobi-PCG's at a
    1e-12 tolerance."""
    from pvof import cases
    grid, params, planes = cases.rayleigh_taylor(1024, 16, Lx=8.0, Ly=0.125, Cn=0.01, atwood=0.5, y0=0.0625,
                                                 velocity_seed=3, velocity_amp=0.05, P_CG_MAXIT=20000,
                                                 P_CG_ETOL=1e-12)
    st_j, a = one_substep(grid, params, planes, 0)
    st_s, b = one_substep(grid, params, planes, 1)
    print("pressure iterations: Jacobi %d, spectral %d" % (st_j.p_iters_total, st_s.p_iters_total))
    assert st_s.p_iters_total < st_j.p_iters_total
    for f in ("DELTAP", "U", "V"):
        assert rel(b[f], a[f]) <= 1e-8, (f, rel(b[f], a[f]))


@pytest.mark.parametrize("NXM,NYM", [(56, 64), (2048, 16), (64, 2048), (36, 64)])
def test_unsupported_grids_are_refused(NXM, NYM):
    from pvof import cases, runtime
    grid, params, planes = cases.rayleigh_taylor(NXM, NYM, Lx=1.0, Ly=2.0, Cn=0.04)
    params.pressure_preconditioner = 1
    with pytest.raises(runtime.PvofError, match="spectral pressure preconditioner"):
        runtime.Solver(grid, params, device=0)


def test_forms_with_resolved_cylinders():
    """Two mobile cylinders and a fixed one on the interface, surface tension
    and a 70 degree contact angle: the four forms together (spectral pressure
    preconditioner, unregularised momentum CG, FP32 stencils, warm start)
    against the plain path after 6 steps: fields within 2e-6 relative L2,
    particle positions within 1e-9, at least 10x fewer pressure iterations."""
    from pvof import cases, runtime
    cyl = [(1, 0.25, 1.0, 0.08, 0, 0, 0, 2.5), (1, 0.75, 1.3, 0.08, 0, 0, 0, 2.5), (0, 0.5, 0.6, 0.1, 0, 0, 0, 2.5)]
    out = {}
    for forms in (0, 1):
        grid, params, planes = cases.rayleigh_taylor(64, 128, Lx=1.0, Ly=2.0, Cn=0.02, P_CG_MAXIT=2000,
                                                     surface_tension=True, We=100.0)
        params.contact_angle_deg = 70.0
        if forms:
            params.stencil_fp32 = params.pressure_warm_start = 1
            params.pressure_preconditioner = params.velocity_cg_unregularized = 1
        s = runtime.Solver(grid, params, device=0)
        s.set_particles(cyl)
        s.set_planes(dict(planes, C_L=planes["F"]))
        s.initialize()
        iters = 0
        for n in range(6):
            for rk in range(3):
                if n > 0 and rk == 0:
                    s.call("Velocity_cell_center")
                s.set_stage(rk, 1e-4)
                iters += s.substep().p_iters_total
        out[forms] = (iters, {f: physical(grid, g_range(grid, s.get(f)), f) for f in ("C_L", "U", "V", "P")},
                      s.get_particles()["X"])
        s.close()
    print("pressure iterations: plain %d, forms %d" % (out[0][0], out[1][0]))
    for f in ("C_L", "U", "V", "P"):
        r = rel(out[1][1][f], out[0][1][f])
        print("%s rel L2 %.2e" % (f, r))
        assert r <= 2e-6, (f, r)
    assert np.abs(out[1][2] - out[0][2]).max() <= 1e-9
    assert 10 * out[1][0] <= out[0][0]
