"""Constant-density Poisson solver by Fourier transform in x and tridiagonal
solves in y (Pressure_solve_xz_period, psolve_fft.c:638-983) against the
reference's own solver (fixtures tests/golden/fft_*.npz from
oracle/ref/fft_driver.c: a power-of-two and a non-power-of-two x count).

CPU: the reference's solution satisfies the discrete Poisson problem the
solver states (x periodic, Neumann walls, the mean mode pinned at j = 0).
GPU: the library's transforms and Thomas solves reproduce it to 1e-12
relative L2 (the transforms round differently from the reference's).
"""
import numpy as np
import pytest

from conftest import load_golden, rel_l2

CASES = ["fft_small", "fft_odd"]


def spacing(grid):
    from pvof import cases
    NX, NY, _ = cases.dims(grid)
    return (grid.xmax - grid.xmin) / (NX - 1), (grid.ymax - grid.ymin) / (NY - 1)


@pytest.mark.parametrize("name", CASES)
def test_reference_solution_solves_the_discrete_problem(name):
    grid, params, planes, d, meta = load_golden(name)
    phi, rhs = d["deltap"], d["rhs"]
    ny, nx = phi.shape
    dx, dy = spacing(grid)
    P = np.pad(phi, ((1, 1), (0, 0)), mode="edge")            # Neumann walls in y
    P = np.concatenate([P[:, -1:], P, P[:, :1]], axis=1)      # periodic in x
    lap = (P[1:-1, 2:] - 2 * P[1:-1, 1:-1] + P[1:-1, :-2]) / dx ** 2 + \
          (P[2:, 1:-1] - 2 * P[1:-1, 1:-1] + P[:-2, 1:-1]) / dy ** 2
    assert np.abs(lap - rhs[:ny, :nx]).max() < 1e-10 * np.abs(rhs).max()
    assert abs(phi[0].mean()) < 1e-13                         # the pinned mean mode


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_gpu_fft_poisson_matches_reference(name):
    from pvof import cases, runtime
    grid, params, planes, d, meta = load_golden(name)
    s = runtime.Solver(grid, params, device=0)
    s.upload("P_RHS", cases.plane_to_block(grid, d["rhs"]))
    s.call("Pressure_solve_fft")
    G = cases.G
    ny, nx = d["deltap"].shape
    phi = s.get("DELTAP")[G:G + ny, G:G + nx]
    err = rel_l2(phi, d["deltap"])
    assert err <= 1e-12, err


@pytest.mark.gpu
def test_fft_poisson_rejects_walls_in_x():
    from pvof import cases, runtime
    grid = cases.planar_grid(16, 32, 1.0, 2.0, periodic_x=False)
    params = cases.default_params()
    s = runtime.Solver(grid, params, device=0)
    with pytest.raises(runtime.PvofError):
        s.call("Pressure_solve_fft")
