"""Parity of the CUDA substep (through the C ABI) with the reference and the
CPU oracle.

Tolerances (relative L2 per field, physical cells):
* against the reference's own time step (golden fixtures) with the solver
  tolerances tightened to near machine precision: 1e-12 after every stored
  substep and step;
* with the reference's default tolerances (CG stops at 1e-9 relative / RMS,
  pressure at 1e-7 absolute) the two codes stop the same iterations on
  residuals that differ in the last bits (reductions are summed in a
  different order), so fields agree to 1e-9;
* against the oracle: stencil routines bit for bit on identical inputs,
  1e-12 after one step of the 128x512 planar case, 1e-10 after 100 steps.
"""
import numpy as np
import pytest

from conftest import g_range, load_golden, physical, rel_l2

pytestmark = pytest.mark.gpu

TIGHT = dict(ch_tol=1e-13, ch_iter_max=600, CG_ETOL=1e-15, CG_MAXIT=400, P_CG_ETOL=1e-13, P_CG_MAXIT=2000)
STATE = ["C_L", "C_G", "RHO", "MU", "CH_RHS_N", "U", "V", "P"]


def solver_for(grid, params, planes, grid_solver=False):
    """grid_solver=True forces the grid-wide pressure PCG even where the
    cluster-resident one fits."""
    from pvof import runtime
    g = runtime.Solver(grid, params, device=0)
    if grid_solver:
        g.set_cluster_solvers(False)
    g.set_planes(planes)
    g.initialize()
    return g


def oracle_for(grid, params, planes):
    import pyoracle as po
    o = po.Oracle(grid, params)
    o.set_planes(planes)
    o.initialize()
    return o


def compare(grid, get_a, get_b, fields, tol, what):
    worst = {}
    for f in fields:
        a = physical(grid, get_a(f), f)
        b = physical(grid, get_b(f), f)
        worst[f] = rel_l2(a, b)
    bad = {f: r for f, r in worst.items() if not r <= tol}
    assert not bad, "%s: %s" % (what, bad)
    return worst


@pytest.mark.parametrize("name,tol", [("rt_tight", 1e-12), ("rt_small", 1e-9), ("rt_st_small", 1e-9),
                                      ("rt_fs_tight", 1e-12), ("axi_tight", 1e-12), ("axi_small", 1e-9),
                                      ("axi_st_tight", 1e-12)])
def test_gpu_matches_reference_golden(name, tol):
    grid, params, planes, d, meta = load_golden(name)
    g = solver_for(grid, params, planes)
    fields = STATE + (["PSI_LG"] if params.surface_tension else [])
    tags = sorted({k.split("/")[0] for k in d.files if "/" in k and not k.startswith("init/")})
    iters = []

    def check(tag):
        if tag not in tags:
            return
        compare(grid, lambda f: g_range(grid, g.get(f)), lambda f: d["%s/%s" % (tag, f)], fields, tol, name + " " + tag)

    check("s0")
    dt = meta["dt"]
    for n in range(1, meta["steps"] + 1):
        for rk in range(3):
            if n > 1 and rk == 0:
                g.call("Velocity_cell_center")
            g.set_stage(rk, dt)
            st = g.substep()
            iters.append((st.ch_iters, st.u_iters, st.v_iters, st.p_iters))
            check("s%d_%d" % (n, rk))
    ref_iters = d["iterations"].T
    got = np.array(iters)
    assert np.array_equal(got[:, :3], ref_iters[:, :3]), (got, ref_iters)
    assert np.all(np.abs(got[:, 3] - ref_iters[:, 3]) <= 2), (got, ref_iters)


@pytest.mark.parametrize("geometry", ["planar", "axisym"])
def test_stencil_routines_bitwise_on_equal_inputs(geometry):
    """Every routine that is not an iterative solve rounds exactly like the
    oracle (the library is built without FMA contraction), in the planar and
    in the axisymmetric mode."""
    from pvof import cases
    if geometry == "planar":
        grid, params, planes = cases.rayleigh_taylor(32, 64, Lx=1.0, Ly=2.0, Cn=0.04, surface_tension=True,
                                                     velocity_seed=5, velocity_amp=0.1)
    else:
        grid, params, planes = cases.rising_bubble(NXM=32, NYM=64, rmax=1.0, zmax=2.0, radius=0.3, zc=0.7, Cn=0.04,
                                                   surface_tension=True, velocity_seed=5, velocity_amp=0.1)
    g = solver_for(grid, params, planes)
    o = oracle_for(grid, params, planes)
    for f in STATE + ["U_BC", "V_BC", "F"]:
        assert np.array_equal(g.get(f), o.get_field(f)), f
    g.set_stage(1, 1e-3)
    o.set_stage(1, 1e-3)
    steps = [
        ("ADVECT_WENO5", lambda: g.call("VOF_DIFFUSE_advect_WENO5"), ["CH_RHS_CUR"]),
        ("UPDATE_DENSITY_VISCOSITY", lambda: g.call("VOF_update_density_viscosity"), ["RHO", "MU"]),
        ("U_IMPLICIT_EXPLICIT", lambda: g.call("Velocity_set_implicit_explicit", b"u"),
         ["U_EXPLICIT", "U_IMPLICIT", "U_VISC_EXPLICIT"]),
        ("V_IMPLICIT_EXPLICIT", lambda: g.call("Velocity_set_implicit_explicit", b"v"),
         ["V_EXPLICIT", "V_IMPLICIT", "V_VISC_EXPLICIT"]),
        ("U_SET_RHS", lambda: g.call("Velocity_set_RHS", b"u"), ["U_RHS", "U_EXPLICIT_OLD"]),
        ("V_SET_RHS", lambda: g.call("Velocity_set_RHS", b"v"), ["V_RHS", "V_EXPLICIT_OLD"]),
        ("COMPUTE_PSI_LG", lambda: g.call("VOF_DIFFUSE_compute_psi_LG"), ["PSI_LG", "LAP_C"]),
        ("COMPUTE_F_SIGMA", lambda: g.call("VOF_DIFFUSE_compute_f_sigma"), ["FSIG_NEW_X", "FSIG_NEW_Y"]),
        ("APPLY_F_SIGMA_OLD", lambda: g.call("VOF_apply_f_sigma_old"), ["U_RHS", "V_RHS"]),
        ("ADD_GRAVITY", lambda: g.call("Velocity_add_gravity_2_RHS"), ["U_RHS", "V_RHS"]),
        ("U_UPDATE_BOUNDARIES", lambda: g.call("Velocity_update_boundaries", b"u"), ["U"]),
        ("V_UPDATE_BOUNDARIES", lambda: g.call("Velocity_update_boundaries", b"v"), ["V"]),
        ("PRESSURE_SET_RHS", lambda: g.call("Pressure_set_RHS"), ["P_RHS"]),
        ("CELL_CENTER", lambda: g.call("Velocity_cell_center"), ["U_BC", "V_BC"]),
    ]
    for name, fn, fields in steps:
        o.routine(name)
        fn()
        for f in fields:
            a = g_range(grid, g.get(f))
            b = g_range(grid, o.get_field(f))
            assert np.array_equal(a, b), "%s/%s max diff %.3e" % (name, f, np.abs(a - b).max())


@pytest.mark.parametrize("geometry", ["planar", "axisym"])
def test_solvers_match_oracle_routine_by_routine(geometry):
    from pvof import cases
    if geometry == "planar":
        grid, params, planes = cases.rayleigh_taylor(32, 64, Lx=1.0, Ly=2.0, Cn=0.04, surface_tension=True,
                                                     velocity_seed=9, velocity_amp=0.1, **TIGHT)
    else:
        grid, params, planes = cases.rising_bubble(NXM=32, NYM=64, rmax=1.0, zmax=2.0, radius=0.3, zc=0.7, Cn=0.04,
                                                   surface_tension=True, velocity_seed=9, velocity_amp=0.1, **TIGHT)
    g = solver_for(grid, params, planes)
    o = oracle_for(grid, params, planes)
    g.set_stage(0, 1e-3)
    o.set_stage(0, 1e-3)
    _, so = o.routine("VOF_DIFFUSE_STEP")
    g.call("VOF_DIFFUSE_step", None)
    compare(grid, g.get, o.get_field, ["C_L", "C_G", "CH_RHS_N"], 1e-13, "VOF_DIFFUSE_step")
    for name, call in [("UPDATE_DENSITY_VISCOSITY", ("VOF_update_density_viscosity",)),
                       ("U_IMPLICIT_EXPLICIT", ("Velocity_set_implicit_explicit", b"u")),
                       ("V_IMPLICIT_EXPLICIT", ("Velocity_set_implicit_explicit", b"v")),
                       ("U_SET_RHS", ("Velocity_set_RHS", b"u")), ("V_SET_RHS", ("Velocity_set_RHS", b"v")),
                       ("ADD_GRAVITY", ("Velocity_add_gravity_2_RHS",))]:
        o.routine(name)
        g.call(*call)
    o.routine("U_SOLVE_CG")
    g.call("Velocity_solve_cg", b"u", None)
    o.routine("V_SOLVE_CG")
    g.call("Velocity_solve_cg", b"v", None)
    compare(grid, g.get, o.get_field, ["U", "V"], 1e-13, "Velocity_solve_cg")
    for name, call in [("U_UPDATE_BOUNDARIES", ("Velocity_update_boundaries", b"u")),
                       ("V_UPDATE_BOUNDARIES", ("Velocity_update_boundaries", b"v")),
                       ("PRESSURE_SET_RHS", ("Pressure_set_RHS",)),
                       ("PRESSURE_PRECONDITIONER", ("Pressure_compute_preconditioner",))]:
        o.routine(name)
        g.call(*call)
    o.routine("PRESSURE_SOLVE_CG")
    g.call("Pressure_solve_cg", None)
    compare(grid, g.get, o.get_field, ["DELTAP"], 1e-12, "Pressure_solve_cg")
    o.routine("PRESSURE_PROJECT")
    g.call("Pressure_project_velocity")
    compare(grid, g.get, o.get_field, ["P", "U", "V"], 1e-12, "Pressure_project_velocity")


@pytest.mark.parametrize("grid_solver", [False, True])
def test_planar_128x512_one_step_parity(grid_solver):
    """The planar two-phase instability on its full 128x512 grid, one RK3
    step, solver tolerances near machine precision in both codes; with the
    cluster-resident and with the grid-wide pressure solver."""
    from pvof import cases
    kw = dict(TIGHT, P_CG_MAXIT=4000)
    grid, params, planes = cases.rayleigh_taylor(128, 512, Lx=1.0, Ly=4.0, Cn=0.01, **kw)
    g = solver_for(grid, params, planes, grid_solver=grid_solver)
    o = oracle_for(grid, params, planes)
    sg = g.run_steps(1, 1e-4)
    so = o.run_steps(1, 1e-4)
    compare(grid, g.get, o.get_field, STATE, 1e-12, "128x512 one step")
    assert sg.poisson_passes == so.poisson_passes == 1


def test_hundred_steps_parity():
    from pvof import cases
    grid, params, planes = cases.rayleigh_taylor(32, 128, Lx=1.0, Ly=4.0, Cn=0.04, velocity_seed=2,
                                                 velocity_amp=0.05, **TIGHT)
    g = solver_for(grid, params, planes)
    o = oracle_for(grid, params, planes)
    g.run_steps(100, 5e-4)
    o.run_steps(100, 5e-4)
    compare(grid, g.get, o.get_field, STATE, 1e-10, "100 steps")


def test_hundred_steps_128x512_against_reference():
    """The planar instability on its full 128x512 grid (the benchmark
    workload), 100 RK3 steps at dt 1e-4, solver tolerances near machine
    precision: C_L, u, v and p on the physical cells within 1e-10 relative L2
    of the reference's own time step (fixture rt128x512_100steps, written by
    the reference build)."""
    from pvof import cases
    grid, params, _, d, meta = load_golden("rt128x512_100steps")
    # the initial planes are those of the case builder (no seed), not stored
    _, _, planes = cases.rayleigh_taylor(**meta["builder"])
    g = solver_for(grid, params, planes)
    g.run_steps(meta["steps"], meta["dt"])
    NX, NY, _ = cases.dims(grid)
    worst = {}
    for f in ("C_L", "U", "V", "P"):
        a = g_range(grid, g.get(f))[:NY - 1, :NX - 1]
        worst[f] = rel_l2(a, d["s%d/%s" % (meta["steps"], f)])
    assert all(r <= 1e-10 for r in worst.values()), worst


def test_hundred_steps_axisym_against_reference():
    """The axisymmetric rising bubble with surface tension (32x64, density
    ratio 0.1, We 200), 100 RK3 steps at dt 1e-3, solver tolerances near
    machine precision (pressure 1e-12, above the axisymmetric rounding
    floor): C_L, u, v and p on the physical cells within 1e-10 relative L2 of
    the reference's own time step (fixture axi_st_100steps, written by the
    axi2d_st reference build)."""
    from pvof import cases
    grid, params, _, d, meta = load_golden("axi_st_100steps")
    build = {k: v for k, v in meta["builder"].items() if k != "_builder"}
    _, _, planes = cases.rising_bubble(**build)
    g = solver_for(grid, params, planes)
    g.run_steps(meta["steps"], meta["dt"])
    NX, NY, _ = cases.dims(grid)
    worst = {}
    for f in ("C_L", "U", "V", "P"):
        a = g_range(grid, g.get(f))[:NY - 1, :NX - 1]
        worst[f] = rel_l2(a, d["s%d/%s" % (meta["steps"], f)])
    print(worst)
    assert all(r <= 1e-10 for r in worst.values()), worst


def test_liquid_mass_conserved():
    """Sum of C_L over the physical cells stays at its initial value to 1e-13
    (relative) when the solves are converged and no clamp event happens; the
    clamp's own mass change is reported per substep."""
    from pvof import cases
    grid, params, planes = cases.rayleigh_taylor(32, 64, Lx=1.0, Ly=2.0, Cn=0.04, velocity_seed=4,
                                                 velocity_amp=0.05, **TIGHT)
    g = solver_for(grid, params, planes)
    o = oracle_for(grid, params, planes)
    m0 = g.liquid_mass()
    assert abs(m0 - o.liquid_mass()) <= 1e-14 * abs(m0)  # summation order only
    clamp = 0.0
    for n in range(10):
        for rk in range(3):
            if n > 0 and rk == 0:
                g.call("Velocity_cell_center")
            g.set_stage(rk, 1e-3)
            st = g.substep()
            clamp += st.clamp_mass
    m1 = g.liquid_mass()
    assert abs((m1 - m0) - clamp) <= 1e-13 * abs(m0), (m0, m1, clamp)


def test_errors_are_reported_not_faulted():
    """Bad arguments and a non-converging Poisson loop come back as error
    codes; the context stays usable afterwards."""
    from pvof import abi, cases, runtime
    grid, params, planes = cases.rayleigh_taylor(16, 32, Lx=1.0, Ly=2.0, Cn=0.05, velocity_seed=1,
                                                 velocity_amp=0.5, P_CG_MAXIT=1, P_CG_ETOL=1e-30)
    g = solver_for(grid, params, planes)
    L = runtime.load()
    assert L.pvof_set_stage(g.h, 5, 1e-3) == abi.EINVAL
    assert L.pvof_set_stage(g.h, 0, -1.0) == abi.EINVAL
    assert L.pvof_Velocity_set_RHS(g.h, b"w") == abi.EINVAL
    g.set_stage(0, 1e-3)
    st = abi.Stats()
    import ctypes
    rc = L.pvof_substep(g.h, ctypes.byref(st))
    assert rc == abi.EDIVERGED
    assert st.poisson_passes == 11
    # still usable
    m = g.liquid_mass()
    assert np.isfinite(m)
