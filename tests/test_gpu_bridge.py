"""The drop-in boundary from the reference's side: PARTIES' own start-up and
time loop (oracle/ref/ref_driver.c, ibm_driver.c), compiled from the
reference's sources with the PARTIES-side bridge
(parties-vof-ibm_b200/bridge/pvof_bridge.c) and linked against libpvof.so,
against the same program built for the CPU.

* substep form (binaries ref_<case>_bridge): the reference's data structures
  are set up by the reference's own code, pvof_bridge_start hands them to
  the device, and pvof_bridge_substep replaces Temporal_int_all_the_equations
  in the RK3 loop;
* routine form (ref_rt2d_routines): the bridge defines the reference's own
  routine names and signatures (VOF_DIFFUSE_step(Cart3d_bag *),
  Pressure_solve_cg(Cart3d_bag *), Velocity_solve_cg(Velocity *,
  Cart3d_bag *), ...) over the device, and the reference's unchanged
  Temporal_int_all_the_equations calls them.

Solver tolerances near machine precision in both builds; every dumped field
after the last step within 1e-12 relative L2 (the solvers sum their inner
products in another order, so the fields agree to rounding, not bit for
bit); the particle position and velocity within 1e-10.  The explicit viscous
histories (ng_visc_explicit_old) are the cross-derivative viscous terms,
which cancel for a divergence-free velocity at uniform viscosity: in the
planar case at viscosity ratio 1 they are rounding noise of order 1e-15, so
their difference is measured against the convective history of the same
component that the momentum right-hand side adds next to them.

The binaries are built from the reference tree (oracle/ref/Makefile,
BRIDGE=substep / BRIDGE=routines); without them the test is skipped with
the reason.
"""
import os
import tempfile

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu

TIGHT = dict(ch_tol=1e-13, ch_iter_max=600, CG_ETOL=1e-15, CG_MAXIT=400, P_CG_ETOL=1e-13, P_CG_MAXIT=2000)
AXI_TIGHT = dict(TIGHT, P_CG_ETOL=1e-12)
FLOW = ["C_L", "C_G", "rho", "mu", "ch_rhs_n", "u", "v", "p"]
NG = ["u_explicit_old", "v_explicit_old", "u_visc_explicit_old", "v_visc_explicit_old"]
ST_FLOW = ["psi_LG"]
ST_NG = ["f_sigma_old_x", "f_sigma_old_y"]


def need(binary_case):
    import pyoracle as po
    if not os.path.exists(po.ref_binary(binary_case)):
        pytest.skip("oracle/_ref/ref_%s is not built (oracle/ref/Makefile needs the reference tree)" % binary_case)


def compare_dumps(grid, cpu_dir, gpu_dir, tag, st, tol=1e-12):
    import pyoracle as po
    worst = {}
    for name in FLOW + (ST_FLOW if st else []):
        a = po.read_reference_field(gpu_dir, tag, name, grid)
        b = po.read_reference_field(cpu_dir, tag, name, grid)
        worst[name] = rel_l2(a, b)
    for name in NG + (ST_NG if st else []):
        a = po.read_reference_field(gpu_dir, tag, name, grid, ng=True)
        b = po.read_reference_field(cpu_dir, tag, name, grid, ng=True)
        if "visc" in name:
            conv = po.read_reference_field(cpu_dir, tag, name.replace("visc_", ""), grid, ng=True)
            worst[name] = float(np.linalg.norm(a - b)) / max(float(np.linalg.norm(b)), float(np.linalg.norm(conv)),
                                                             1e-300)
        else:
            worst[name] = rel_l2(a, b)
    bad = {k: v for k, v in worst.items() if not v <= tol}
    assert not bad, "%s: %s" % (tag, bad)
    return worst


@pytest.mark.parametrize("case,form,builder", [
    ("rt2d", "bridge", "planar"),
    ("rt2d", "routines", "planar"),
    ("axi2d_st", "bridge", "axisym"),
])
def test_reference_time_loop_drives_the_device(case, form, builder):
    """10 RK3 steps of the reference's loop: CPU build against the build
    whose substep (or whose routines) run on the B200 through the bridge."""
    import pyoracle as po
    from pvof import cases
    need(case)
    need(case + "_" + form)
    if builder == "planar":
        grid, params, planes = cases.rayleigh_taylor(24, 48, Lx=1.0, Ly=2.0, Cn=0.04, velocity_seed=3,
                                                     velocity_amp=0.1, **TIGHT)
    else:
        grid, params, planes = cases.rising_bubble(NXM=24, NYM=48, rmax=1.0, zmax=2.0, radius=0.3, zc=0.7, Cn=0.04,
                                                   surface_tension=True, We=200.0, velocity_seed=21,
                                                   velocity_amp=0.1, **AXI_TIGHT)
    steps = 10
    with tempfile.TemporaryDirectory() as cpu, tempfile.TemporaryDirectory() as gpu:
        po.run_reference(case, cpu, grid, params, planes, steps, 1e-3, steps)
        cp = po.run_reference(case + "_" + form, gpu, grid, params, planes, steps, 1e-3, steps)
        assert "REF_TIMING" in cp.stdout
        compare_dumps(grid, cpu, gpu, "s0", bool(params.surface_tension))
        compare_dumps(grid, cpu, gpu, "s%d" % steps, bool(params.surface_tension))


def test_reference_time_loop_with_a_sphere_drives_the_device():
    """The axisymmetric bubble with a fixed sphere on the axis (resolved
    particles, contact angle 90 degrees): 2 steps of the reference's loop on
    the CPU against the bridge's substep on the B200; the particle list goes
    to the device at pvof_bridge_start and its state comes back by ID."""
    import pyoracle as po
    from pvof import cases
    need("ibm_axi_st")
    need("ibm_axi_st_bridge")
    grid, params, planes = cases.rising_bubble(NXM=32, NYM=64, rmax=1.0, zmax=2.0, radius=0.3, zc=0.7, Cn=0.04,
                                               surface_tension=True, We=200.0, velocity_seed=23, velocity_amp=0.1,
                                               **AXI_TIGHT)
    params.contact_angle_deg = 90.0
    sphere = [(0.0, 1.15, 0.2, 0.0, 0.0, 0.0)]
    steps = 2
    with tempfile.TemporaryDirectory() as cpu, tempfile.TemporaryDirectory() as gpu:
        po.run_reference_ibm(cpu, grid, params, planes, sphere, [], 1e-3, 0, case="ibm_axi_st", mode="steps",
                             nsteps=steps)
        po.run_reference_ibm(gpu, grid, params, planes, sphere, [], 1e-3, 0, case="ibm_axi_st_bridge",
                             mode="steps", nsteps=steps)
        compare_dumps(grid, cpu, gpu, "s%d" % steps, True)
        pid_c, X_c, U_c, _ = po.read_reference_particle_state(cpu, "s%d" % steps)
        pid_g, X_g, U_g, _ = po.read_reference_particle_state(gpu, "s%d" % steps)
        assert np.array_equal(pid_c, pid_g)
        assert np.abs(X_g - X_c).max() <= 1e-10
        assert np.abs(U_g - U_c).max() <= 1e-10


def test_reference_3d_time_loop_drives_the_device():
    """The 3D build (x and z periodic, no-slip walls in y, surface tension):
    5 RK3 steps of the reference's loop on the CPU against the same program
    whose substep runs on the B200 through the bridge; every dumped field
    (the whole ghosted block, w included) within 1e-12."""
    import pyoracle as po
    from pvof import cases
    need("rt3d_st")
    need("rt3d_st_bridge")
    grid, params, fields = cases.interface_box(16, 24, 12, Cn=0.1, amp_max=0.1, We=10.0, Re=100.0, rho_ratio=0.1,
                                               mu_ratio=0.1, velocity_seed=6, velocity_amp=0.05,
                                               **dict(TIGHT, CG_ETOL=1e-13))
    steps = 5
    flow = FLOW + ["w", "psi_LG"]
    ng = NG + ["w_explicit_old", "w_visc_explicit_old", "f_sigma_old_x", "f_sigma_old_y", "f_sigma_old_z"]
    with tempfile.TemporaryDirectory() as cpu, tempfile.TemporaryDirectory() as gpu:
        po.run_reference("rt3d_st", cpu, grid, params, fields, steps, 1e-3, steps)
        cp = po.run_reference("rt3d_st_bridge", gpu, grid, params, fields, steps, 1e-3, steps)
        assert "REF_TIMING" in cp.stdout
        worst = {}
        for name in flow + ng:
            a = np.fromfile(os.path.join(gpu, "out", "s%d_%s.bin" % (steps, name)), dtype="<f8")
            b = np.fromfile(os.path.join(cpu, "out", "s%d_%s.bin" % (steps, name)), dtype="<f8")
            worst[name] = rel_l2(a, b)
        bad = {k: v for k, v in worst.items() if not v <= 1e-12}
        assert not bad, bad
