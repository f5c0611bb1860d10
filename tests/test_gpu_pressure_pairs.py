"""The grid-wide pressure solve over pairs of cells (16-byte accesses; the
context's choice from two cells per resident thread on) against the same
solve over single cells, whose results are bit for bit those of the
parity-tested first form: the same iteration, so the same fields to
rounding and the same iteration counts within a couple.  Covers a row of odd
length (each row ends in a single cell), the axisymmetric row weights and
the automatic choice on a grid large enough for pairs."""
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu

FIELDS = ("C_L", "U", "V", "P")
# solver tolerances near machine precision (the parity tests' TIGHT set), so
# that a solve stopping one iteration earlier or later moves the fields by
# rounding only; the axisymmetric pressure residual's floor is 2e-13 to 5e-13
TIGHT = dict(ch_tol=1e-13, ch_iter_max=600, CG_ETOL=1e-15, CG_MAXIT=400, P_CG_ETOL=1e-13, P_CG_MAXIT=20000)


def _steps(builder, kw, mode, steps, dt):
    from pvof import runtime
    grid, params, planes = builder(**kw)
    s = runtime.Solver(grid, params, device=0)
    s.set_cluster_solvers(False)
    s.set_pressure_pairs(mode)
    s.set_planes(planes)
    s.initialize()
    s.set_solver_timing(True)
    s.run_steps(steps, dt)
    it = s.solver_timing(2)["iterations"]
    name = s.solver_kernel(2)
    out = {f: s.get(f) for f in FIELDS}
    s.close()
    return out, it, name


@pytest.mark.parametrize("case", ["planar_odd_width", "axisym"])
def test_pairs_match_single_cells(case):
    from pvof import cases
    if case == "planar_odd_width":
        builder, kw, dt = cases.rayleigh_taylor, dict(NXM=257, NYM=514, Lx=1.0, Ly=2.0, Cn=0.01, **TIGHT), 1e-4
    else:
        builder, kw, dt = cases.rising_bubble, dict(NXM=161, NYM=322, rmax=1.0, zmax=2.0, radius=0.3, zc=0.7,
                                                    Cn=0.02, rho_ratio=0.1, mu_ratio=0.1, surface_tension=True,
                                                    **dict(TIGHT, P_CG_ETOL=1e-12)), 1e-4
    one, it1, n1 = _steps(builder, kw, 0, 2, dt)
    two, it2, n2 = _steps(builder, kw, 1, 2, dt)
    assert n1 == "k_cg_pressure_fw" and n2 == "k_cg_pressure_fwp", (n1, n2)
    errs = {f: rel_l2(two[f], one[f]) for f in FIELDS}
    print(case, errs, it1, it2)
    assert all(e <= 1e-11 for e in errs.values()), errs
    assert abs(it1 - it2) <= 2 * 6, (it1, it2)   # within two of each of the six substeps' stopping iterations


def test_automatic_choice_by_size():
    from pvof import cases, runtime
    small = cases.rayleigh_taylor(NXM=256, NYM=512, Lx=1.0, Ly=2.0)
    large = cases.rayleigh_taylor(NXM=1024, NYM=512, Lx=2.0, Ly=1.0)
    names = []
    for grid, params, planes in (small, large):
        s = runtime.Solver(grid, params, device=0)
        names.append(s.solver_kernel(2))
        s.close()
    assert names == ["k_cg_pressure_fw", "k_cg_pressure_fwp"], names
