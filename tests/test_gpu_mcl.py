"""Contact line on resolved solids, and whole time steps with resolved
cylinders, against the reference.

Routine fixtures (tests/golden/mcl_theta{60,120,30}.npz, oracle/ref/ibm_driver.c
"mcl" mode on the ibm2d build): two fixed cylinders on a perturbed interface,
one across the periodic x boundary, and a small mobile one; contact angles on
both sides of 90 degrees and one below 45 (the narrower liquid-gas band); and
(mcl_fs_theta45, the ibm2d_fs build) free-slip y walls with the interface and
two cylinders next to the bottom wall, so the characteristics cross it; and
(mcl_axi_theta{60,120}, the ibm_axi_st build) a sphere on the symmetry axis of
an axisymmetric case in the top of a bubble, the normals' parity and the
characteristics folded at the axis.
Each routine gets the reference's input state and is compared with the
reference's output over the whole ghosted plane:

  VOF_DIFFUSE_compute_solid_normals_MCL      nx_IBM, ny_IBM     bit for bit
  VOF_DIFFUSE_apply_contact_angle            C_L                bit for bit
  VOF_DIFFUSE_extend_psi_LG_contact_angle    psi_LG             bit for bit
  VOF_DIFFUSE_init (with its projection)     C_S 1e-15, C_L and C_G 1e-13
                                             (C_S holds CUDA's tanh, within an
                                             ulp of glibc's; the clamp to 1 - C_S
                                             and the projection carry that on)

Step fixtures (tests/golden/ibm_steps{,_st}.npz, the driver's "steps" mode):
two whole time steps of Temporal_int_all_the_equations with fixed cylinders,
with and without surface tension, and (ibm_axi_steps_st) with a fixed sphere
on the axis of an axisymmetric bubble case (the psi_LG extension runs at every third
substep, the C_L projection once per step), solver tolerances near machine
precision: state fields to 1e-12 relative L2 after each step, biharmonic
and momentum iteration counts equal.  The pressure solve stops at an absolute
residual of 1e-13, where its residual has flattened onto rounding noise, so
its count may differ by a few iterations (within 3%) while the fields still
agree to 1e-12.
"""
import numpy as np
import pytest

from conftest import g_range, load_golden, physical, rel_l2

pytestmark = pytest.mark.gpu

MCL = ["mcl_theta60", "mcl_theta120", "mcl_theta30", "mcl_fs_theta45", "mcl_axi_theta60", "mcl_axi_theta120"]


def block(grid, plane):
    """Host block of a flow field whose every k plane is the ghosted plane."""
    from pvof import cases
    b = np.zeros(cases.block_shape(grid, False))
    b[:] = plane[None]
    return b


def solver(name):
    from pvof import runtime
    grid, params, planes, d, meta = load_golden(name)
    s = runtime.Solver(grid, params, device=0)
    s.set_particles([tuple(p) for p in meta["particles"]])
    return s, grid, params, planes, d, meta


def assert_bitwise(a, b, what):
    a, b = np.asarray(a), np.asarray(b)
    assert a.shape == b.shape, (what, a.shape, b.shape)
    bad = np.argwhere(a != b)
    assert bad.size == 0, "%s: %d cells differ, first (j, i) %s, max %.3e" % (
        what, len(bad), bad[:4].tolist(), np.abs(a - b).max())


@pytest.mark.parametrize("name", MCL)
def test_solid_normals_match_reference(name):
    s, grid, _, _, d, _ = solver(name)
    s.upload("C_S", block(grid, d["m1/C_S"]))
    s.call("VOF_DIFFUSE_compute_solid_normals_MCL")
    assert_bitwise(s.get("NX_IBM"), d["m2/nx"], "nx_IBM")
    assert_bitwise(s.get("NY_IBM"), d["m2/ny"], "ny_IBM")


@pytest.mark.parametrize("name", MCL)
def test_contact_angle_projection_matches_reference(name):
    s, grid, _, _, d, _ = solver(name)
    for f, key in (("C_S", "m1/C_S"), ("C_L", "m1/C_L"), ("C_G", "m1/C_G")):
        s.upload(f, block(grid, d[key]))
    s.call("VOF_DIFFUSE_apply_contact_angle")
    out = s.get("C_L")
    # the projection moved the contact cells (around one contact point on the
    # meridian in the axisymmetric cases, several in the planar ones)
    assert np.count_nonzero(out != d["m1/C_L"]) > (5 if "axi" in name else 50)
    assert_bitwise(out, d["m2/C_L"], "C_L after the projection")


@pytest.mark.parametrize("name", MCL)
def test_psi_extension_matches_reference(name):
    s, grid, _, _, d, _ = solver(name)
    for f, key in (("C_S", "m1/C_S"), ("C_L", "m3/C_L"), ("C_G", "m3/C_G"), ("PSI_LG", "m3/psi_LG")):
        s.upload(f, block(grid, d[key]))
    s.call("VOF_DIFFUSE_extend_psi_LG_contact_angle")
    out = s.get("PSI_LG")
    assert np.count_nonzero(out != d["m3/psi_LG"]) > (5 if "axi" in name else 50)
    assert_bitwise(out, d["m4/psi_LG"], "psi_LG after the extension")


@pytest.mark.parametrize("name", MCL)
def test_initialisation_projects_the_contact_angle(name):
    """pvof_initialize with particles: C_S, the clamp and the projection of
    VOF_DIFFUSE_init from the initial F (and C_L = F, as the reference's
    initialisers leave it)."""
    s, grid, _, planes, d, _ = solver(name)
    s.set_planes(dict(planes, C_L=planes["F"]))
    s.initialize()
    for f, key, tol in (("C_S", "i0/C_S", 1e-15), ("C_L", "i0/C_L", 1e-13), ("C_G", "i0/C_G", 1e-13)):
        a, b = s.get(f), d[key]
        err = np.abs(a - b).max()
        assert err <= tol, "%s: max abs diff %.3e" % (f, err)


STATE = ["C_L", "C_G", "RHO", "MU", "CH_RHS_N", "U", "V", "P"]


@pytest.mark.parametrize("name", ["ibm_steps_st", "ibm_steps", "ibm_axi_steps_st"])
def test_steps_with_fixed_cylinders_match_reference(name):
    s, grid, params, planes, d, meta = solver(name)
    s.set_planes(dict(planes, C_L=planes["F"]))
    s.initialize()
    fields = STATE + (["PSI_LG"] if params.surface_tension else [])

    def check(tag):
        worst = {}
        for f in fields:
            worst[f] = rel_l2(physical(grid, g_range(grid, s.get(f)), f), physical(grid, d["%s/%s" % (tag, f)], f))
        bad = {f: r for f, r in worst.items() if not r <= 1e-12}
        assert not bad, "%s %s: %s" % (name, tag, bad)

    check("s0")
    iters = []
    for n in range(1, meta["steps"] + 1):
        for rk in range(3):
            if n > 1 and rk == 0:
                s.call("Velocity_cell_center")
            s.set_stage(rk, meta["dt"])
            st = s.substep()
            iters.append((st.ch_iters, st.u_iters, st.v_iters, st.p_iters))
        check("s%d" % n)
    ref = d["iterations"].T
    got = np.array(iters)
    assert np.array_equal(got[:, :3], ref[:, :3]), (got, ref)
    assert np.all(np.abs(got[:, 3] - ref[:, 3]) <= 0.03 * ref[:, 3]), (got, ref)
