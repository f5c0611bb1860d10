"""The FP32 stencil form against the plain FP64 path.

With pvof_params.stencil_fp32 = 1 the WENO5 face fluxes, the explicit
chemical-potential diffusion, psi_LG and the surface-tension face force are
evaluated in single precision (the fields, the global sums, the biharmonic,
momentum and pressure solves stay FP64).  Targets for the form:

  velocity   relative L2 error against the FP64 path   <= 1e-5
  volume     relative change of the discrete sum of C
             against the FP64 path                     <= 1e-6

measured here after 20 steps of the 128x512 planar instability (no surface
tension) and of a 64x256 case with surface tension.  The face fluxes are
stored once per face and shared by the two cells beside it, so the
advection still telescopes.
"""
import numpy as np
import pytest

from conftest import g_range, physical

pytestmark = pytest.mark.gpu


def run(grid, params, planes, fp32, nsteps, dt):
    from pvof import runtime
    params.stencil_fp32 = 1 if fp32 else 0
    s = runtime.Solver(grid, params, device=0)
    s.set_planes(planes)
    s.initialize()
    m0 = s.liquid_mass()
    s.run_steps(nsteps, dt)
    out = {f: physical(grid, g_range(grid, s.get(f)), f) for f in ("C_L", "U", "V")}
    out["mass0"], out["mass"] = m0, s.liquid_mass()
    s.close()
    return out


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.mark.parametrize("label,builder", [
    ("rt128x512", dict(NXM=128, NYM=512, Lx=1.0, Ly=4.0, Cn=0.01, P_CG_MAXIT=2000)),
    ("st64x256", dict(NXM=64, NYM=256, Lx=1.0, Ly=4.0, Cn=0.02, surface_tension=True, We=50.0, P_CG_MAXIT=2000,
                      velocity_seed=5, velocity_amp=0.05)),
])
def test_fp32_stencil_form_within_targets(label, builder):
    from pvof import cases
    grid, params, planes = cases.rayleigh_taylor(**builder)
    a = run(grid, params, planes, False, 20, 1e-4)
    b = run(grid, params, planes, True, 20, 1e-4)
    vel = max(rel(b["U"], a["U"]), rel(b["V"], a["V"]))
    vol = abs(b["mass"] - a["mass"]) / abs(a["mass"])
    cl = rel(b["C_L"], a["C_L"])
    print("%s: velocity %.2e, C_L %.2e, volume %.2e" % (label, vel, cl, vol))
    assert 0.0 < cl                  # the single-precision stencils ran
    assert vel <= 1e-5, vel
    assert vol <= 1e-6, vol
