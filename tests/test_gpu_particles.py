"""Mobile resolved cylinders through whole time steps, against the reference
(fixture tests/golden/ibm_mobile_st.npz from oracle/ref/ibm_driver.c "steps"
mode on the ibm2d_st build).

The case has a fixed cylinder on the interface, a mobile one across the
periodic x boundary (its periodic copy adds to its momentum integrals and
forces) and a mobile one cutting the interface (the capillary contact force
acts on it), surface tension on, solver tolerances near machine precision.
Checked:

  initialisation (Particle_initialize_velocities: particle velocity from the
  fluid inside it, rigid-body paint of that fluid)   u, v 1e-12; U, Omega 1e-12
  after each of two steps                            state fields 1e-12;
                                                     positions 1e-13 absolute;
                                                     U, Omega, F, T 1e-10

The per-particle sums (momentum integrals, contact-line force) are block
reductions on the device where the reference adds cell by cell, so the
particle quantities agree to rounding rather than bit for bit.
"""
import numpy as np
import pytest

from conftest import g_range, load_golden, physical, rel_l2

pytestmark = pytest.mark.gpu

STATE = ["C_L", "C_G", "RHO", "MU", "CH_RHS_N", "U", "V", "P", "PSI_LG"]


def rel(a, b):
    a, b = np.asarray(a, dtype=float), np.asarray(b, dtype=float)
    scale = max(np.abs(b).max(), 1e-300)
    return np.abs(a - b).max() / scale


def check_particles(s, d, tag, tol_x, tol_v, forces):
    got = s.get_particles()
    assert got["id"].tolist() == d[tag + "/pid"].tolist(), (got["id"], d[tag + "/pid"])
    assert np.abs(got["X"] - d[tag + "/pX"]).max() <= tol_x, (tag, got["X"], d[tag + "/pX"])
    assert rel(got["U"], d[tag + "/pU"]) <= tol_v, (tag, got["U"], d[tag + "/pU"])
    assert rel(got["Omega"], d[tag + "/pOmega"]) <= tol_v, (tag, got["Omega"], d[tag + "/pOmega"])
    if forces:
        assert rel(got["F"], d[tag + "/F"]) <= tol_v, (tag, got["F"], d[tag + "/F"])
        assert rel(got["T"], d[tag + "/T"]) <= tol_v, (tag, got["T"], d[tag + "/T"])


def test_mobile_cylinders_match_reference():
    from pvof import runtime
    grid, params, planes, d, meta = load_golden("ibm_mobile_st")
    s = runtime.Solver(grid, params, device=0)
    s.set_particles([tuple(p) for p in meta["particles"]])
    s.set_planes(dict(planes, C_L=planes["F"]))
    s.initialize()

    def check_fields(tag):
        worst = {f: rel_l2(physical(grid, g_range(grid, s.get(f)), f), physical(grid, d["%s/%s" % (tag, f)], f))
                 for f in STATE}
        bad = {f: r for f, r in worst.items() if not r <= 1e-12}
        assert not bad, "%s: %s" % (tag, bad)

    check_fields("s0")
    check_particles(s, d, "s0", 0.0, 1e-12, False)
    for n in range(1, meta["steps"] + 1):
        for rk in range(3):
            if n > 1 and rk == 0:
                s.call("Velocity_cell_center")
            s.set_stage(rk, meta["dt"])
            s.substep()
        check_fields("s%d" % n)
        check_particles(s, d, "s%d" % n, 1e-13, 1e-10, True)


def test_particles_in_lubrication_range_are_refused():
    """Two mobile cylinders closer than the lubrication range: the collision
    models would act, and they are not built, so the substep says so."""
    from pvof import cases, runtime
    grid, params, planes = cases.rayleigh_taylor(32, 64, Lx=1.0, Ly=2.0, Cn=0.04)
    s = runtime.Solver(grid, params, device=0)
    s.set_particles([(1, 0.3, 0.5, 0.1, 0, 0, 0, 2.5), (1, 0.5, 0.5, 0.09, 0, 0, 0, 2.5)])
    s.set_planes(dict(planes, C_L=planes["F"]))
    s.initialize()
    s.set_stage(0, 1e-3)
    with pytest.raises(runtime.PvofError, match="lubrication range"):
        s.substep()


def test_droplet_on_cylinder_matches_reference():
    """The batching form's case in small (a sessile droplet on a static
    cylinder, contact angle 60 degrees; fixture tests/golden/drop_cyl_st.npz
    from the ibm2d_st reference build): three whole steps, state fields
    within 1e-12, the cylinder's reaction force and torque within 1e-10."""
    from pvof import runtime
    grid, params, planes, d, meta = load_golden("drop_cyl_st")
    s = runtime.Solver(grid, params, device=0)
    s.set_particles([tuple(p) for p in meta["particles"]])
    s.set_planes(dict(planes, C_L=planes["F"]))
    s.initialize()
    for n in range(1, meta["steps"] + 1):
        for rk in range(3):
            if n > 1 and rk == 0:
                s.call("Velocity_cell_center")
            s.set_stage(rk, meta["dt"])
            s.substep()
        worst = {f: rel_l2(physical(grid, g_range(grid, s.get(f)), f), physical(grid, d["s%d/%s" % (n, f)], f))
                 for f in STATE}
        bad = {f: r for f, r in worst.items() if not r <= 1e-12}
        assert not bad, "s%d: %s" % (n, bad)
        check_particles(s, d, "s%d" % n, 0.0, 1e-10, True)


def test_droplet_on_cylinder_fp32_form_and_graphs():
    """The same case as the batching form runs it: FP32 stencils, substeps
    replayed from CUDA graphs (the particle bookkeeping on the device), 6
    steps, against the FP64 path launched step by step: velocity within
    1e-5 relative L2, the liquid volume within 1e-6 relative, the graphs
    replayed."""
    from pvof import cases, runtime
    out = {}
    for fp32 in (0, 1):
        grid, params, planes, parts = cases.droplet_on_cylinder(48, Rd=0.45, Rs=0.3, theta=120.0,
                                                                 P_CG_MAXIT=4000, stencil_fp32=fp32)
        s = runtime.Solver(grid, params, device=0)
        s.set_graphs(bool(fp32))
        s.set_particles(parts)
        s.set_planes(dict(planes, C_L=planes["F"]))
        s.initialize()
        s.run_steps(6, 2e-4)
        out[fp32] = ({f: physical(grid, g_range(grid, s.get(f)), f) for f in ("U", "V", "C_L")}, s.liquid_mass(),
                     s.graph_replays())
        s.close()
    (a, ma, _), (b, mb, replays) = out[0], out[1]
    for f in ("U", "V"):
        r = rel_l2(b[f], a[f])
        print("%s rel L2 %.2e" % (f, r))
        assert r <= 1e-5, (f, r)
    print("volume rel %.2e, graph replays %d" % (abs(mb - ma) / ma, replays))
    assert abs(mb - ma) <= 1e-6 * ma
    assert replays > 0


def test_hundred_steps_axisym_sphere_against_reference():
    """The axisymmetric bubble below the fixed sphere on the axis (32x64,
    surface tension We 200, contact angle 90 degrees, density ratio 0.1),
    100 RK3 steps at dt 1e-3 with tight solver tolerances: C_L, u, v and p on
    the physical cells within 1e-10 relative L2 of the reference's own time
    step (fixture ibm_axi_st_100steps, written by the ibm_axi_st reference
    build), every substep replayed from CUDA graphs after the first few."""
    from pvof import cases, runtime
    grid, params, _, d, meta = load_golden("ibm_axi_st_100steps")
    build = {k: v for k, v in meta["builder"].items() if k != "_builder"}
    _, _, planes = cases.rising_bubble(**build)
    s = runtime.Solver(grid, params, device=0)
    s.set_particles([tuple(p) for p in meta["particles"]])
    s.set_planes(dict(planes, C_L=planes["F"]))
    s.initialize()
    s.run_steps(meta["steps"], meta["dt"])
    NX, NY, _ = cases.dims(grid)
    tag = "s%d" % meta["steps"]
    worst = {f: rel_l2(g_range(grid, s.get(f))[:NY - 1, :NX - 1], d["%s/%s" % (tag, f)]) for f in ("C_L", "U", "V", "P")}
    print(worst, "graph replays", s.graph_replays())
    assert all(r <= 1e-10 for r in worst.values()), worst
    assert s.graph_replays() > 250
