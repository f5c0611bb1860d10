"""Host-side layout helpers: the reference's block layout of flow and
no-ghost fields (PARTIES/src/Memory.c:36-89, :270-323)."""
import numpy as np

from pvof import cases


def test_block_roundtrip():
    grid, params, planes = cases.rayleigh_taylor(16, 24, Ly=1.5, Cn=0.05)
    NX, NY, NZ = cases.dims(grid)
    assert (NX, NY, NZ) == (17, 25, 2)
    blk = cases.plane_to_block(grid, planes["F"])
    assert blk.shape == (NZ + 6, NY + 6, NX + 6)
    pl = cases.block_plane(grid, blk)
    assert np.array_equal(pl[3:3 + NY, 3:3 + NX], planes["F"])
    assert np.all(blk[:3] == 0) and np.all(blk[3 + NZ:] == 0)
    ng = cases.plane_to_block(grid, planes["F"], ng=True)
    assert ng.shape == (NZ, NY, NX)
    assert np.array_equal(cases.block_plane(grid, ng, ng=True), planes["F"])


def test_rayleigh_taylor_profile():
    grid, params, planes = cases.rayleigh_taylor(128, 512, Lx=1.0, Ly=4.0, Cn=0.01)
    assert abs(grid.slab_thickness - 1.0 / 128) < 1e-15
    C = planes["F"]
    assert C.min() >= 0.0 and C.max() <= 1.0
    # heavy fluid (C = 1) on top
    assert C[-2, :].min() > 0.999 and C[0, :].max() < 1e-3
    assert abs(params.rho2 - 1.0 / 3.0) < 1e-15
    assert abs(params.Pe_CH - 100.0) < 1e-12
