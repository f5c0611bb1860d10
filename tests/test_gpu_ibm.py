"""Resolved solid particles: the immersed-boundary routines of one substep
against the reference's own routines (fixture tests/golden/ibm_small.npz,
made by oracle/ref/ibm_driver.c on the reference build with VOF_IBM and
LAG_PARTICLE_RESOLVED).

The planar case has a fixed cylinder crossing the periodic x boundary (so the
list update adds a periodic copy that carries markers) and a mobile cylinder
with velocity and spin; the axisymmetric case (ibm_axi_small, the ibm_axi_st
build) a fixed sphere on the symmetry axis in the top of a bubble.  Each routine gets the reference's inputs and is compared
with the reference's outputs:

  markers and flags        Lagrangian_flag_points        bit for bit
  C_S                      VOF_DIFFUSE_compute_C_S       1e-15 (tanh of CUDA vs glibc)
  u*, v*                   Velocity_solve_explicit       bit for bit
  RHS, F, T                Lagrangian_force(-1)          bit for bit
  u, v, RHS, F, T          Lagrangian_force(2)           bit for bit
"""
import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu


def ghosted_block(grid, plane):
    """Host block of a flow field whose every k plane is the ghosted plane."""
    from pvof import cases
    blk = np.zeros(cases.block_shape(grid, False))
    blk[:] = plane[None]
    return blk


def ng_block(grid, plane):
    from pvof import cases
    return cases.plane_to_block(grid, plane, ng=True)


def particles_of(meta):
    return [tuple(p) for p in meta["particles"]]


def assert_same(a, b, what, tol=0.0):
    a, b = np.asarray(a), np.asarray(b)
    assert a.shape == b.shape, (what, a.shape, b.shape)
    err = np.max(np.abs(a - b)) if a.size else 0.0
    scale = max(np.max(np.abs(b)) if b.size else 0.0, 1e-300)
    assert err <= tol * scale, "%s: max abs diff %.3e (scale %.3e)" % (what, err, scale)


@pytest.fixture(scope="module", params=["ibm_small", "ibm_axi_small"])
def case(request):
    """ibm_small: planar cylinders; ibm_axi_small: a sphere on the symmetry
    axis of an axisymmetric case (ring markers, supports folded across the
    axis, ring cell volumes)."""
    return load_golden(request.param)


def test_solid_fraction_matches_reference(case):
    from pvof import runtime
    grid, params, planes, d, meta = case
    s = runtime.Solver(grid, params, device=0)
    s.set_particles(particles_of(meta))
    s.call("VOF_DIFFUSE_compute_C_S")
    cs = s.get("C_S")
    ref = d["i0/C_S"]
    assert ref.max() > 0.5
    assert_same(cs, ref, "C_S", tol=1e-15)


def test_markers_and_flags_match_reference(case):
    from pvof import runtime
    grid, params, planes, d, meta = case
    s = runtime.Solver(grid, params, device=0)
    s.set_particles(particles_of(meta))
    s.set_stage(meta["stage"], meta["dt"])
    n = s.flag_points()
    counts = d["markers/count"]
    assert n == len(counts)
    off = 0
    for e in range(n):
        x, y, vol, fl = s.particle_markers(e)
        c = int(counts[e])
        assert len(x) == c, (e, len(x), c)
        assert_same(x, d["markers/x"][off:off + c], "X_L %d" % e)
        assert_same(y, d["markers/y"][off:off + c], "Y_L %d" % e)
        assert_same(vol, d["markers/vol"][off:off + c], "Vol_L %d" % e)
        assert_same(fl, d["markers/flag"][off:off + c], "flag_L %d" % e)
        off += c
    assert off == counts.sum() and counts.sum() > 0


def test_forcing_sequence_matches_reference(case):
    """Velocity_solve_explicit, Lagrangian_force(-1), Lagrangian_force(2) on
    the reference's inputs, with the boundary updates the substep makes."""
    from pvof import runtime
    grid, params, planes, d, meta = case
    s = runtime.Solver(grid, params, device=0)
    s.set_particles(particles_of(meta))
    s.set_stage(meta["stage"], meta["dt"])
    s.flag_points()
    s.upload("RHO", ghosted_block(grid, d["i0/rho"]))
    s.upload("U", ghosted_block(grid, d["r0/u"]))
    s.upload("V", ghosted_block(grid, d["r0/v"]))
    for f, key in (("U_RHS", "u_rhs"), ("V_RHS", "v_rhs"), ("U_IMPLICIT", "u_implicit"), ("V_IMPLICIT", "v_implicit")):
        s.upload(f, ng_block(grid, d["r0/" + key]))
    # explicit predictor (msolve_direct.c:146-260) and the boundary update
    s.call("Velocity_solve_explicit", b"u")
    s.call("Velocity_solve_explicit", b"v")
    s.call("Velocity_update_boundaries", b"u")
    s.call("Velocity_update_boundaries", b"v")
    assert_same(s.get("U"), d["r1/u"], "u* after Velocity_solve_explicit")
    assert_same(s.get("V"), d["r1/v"], "v* after Velocity_solve_explicit")
    # forcing on the RHS
    s.call("Lagrangian_force", -1)
    assert_same(s.get("U_RHS"), d["r2/u_rhs"], "u RHS after Lagrangian_force(-1)")
    assert_same(s.get("V_RHS"), d["r2/v_rhs"], "v RHS after Lagrangian_force(-1)")
    F, T = s.particle_forces()
    assert_same(F, d["r2/F"], "F after the predictor")
    assert_same(T, d["r2/T"], "T after the predictor")
    assert np.abs(d["r2/F"]).max() > 0.0
    # correctors on the velocity after the implicit solve (the reference's solve result)
    s.upload("U", ghosted_block(grid, d["r3/u"]))
    s.upload("V", ghosted_block(grid, d["r3/v"]))
    s.call("Lagrangian_force", 2)
    s.call("Velocity_update_boundaries", b"u")
    s.call("Velocity_update_boundaries", b"v")
    assert_same(s.get("U"), d["r4/u"], "u after the correctors")
    assert_same(s.get("V"), d["r4/v"], "v after the correctors")
    assert_same(s.get("U_RHS"), d["r4/u_rhs"], "u RHS of the last corrector")
    assert_same(s.get("V_RHS"), d["r4/v_rhs"], "v RHS of the last corrector")
    F, T = s.particle_forces()
    assert_same(F, d["r4/F"], "F after the correctors")
    assert_same(T, d["r4/T"], "T after the correctors")


def test_particle_errors_are_reported():
    from pvof import cases, runtime
    grid, params, _ = cases.rayleigh_taylor(16, 32, Lx=1.0, Ly=2.0, Cn=0.08)
    s = runtime.Solver(grid, params, device=0)
    with pytest.raises(runtime.PvofError):
        s.call("Lagrangian_force", -1)          # before pvof_set_stage / flag_points
    s.set_stage(0, 1e-3)
    with pytest.raises(runtime.PvofError):
        s.call("Lagrangian_force", -1)          # before pvof_Lagrangian_flag_points
    with pytest.raises(runtime.PvofError):
        s.set_particles([(0, 0.5, 1.0, -0.1, 0, 0, 0, 2.5)])   # negative radius
