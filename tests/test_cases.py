"""The synthetic case builders the benchmark and the batch tests use, on the
CPU: the batching form's droplet-on-cylinder cases are seeded and
reproducible, their widths are the ones the spectral preconditioner's row
transforms take, and their parameters stay in the stated ranges."""
import math

import numpy as np


def test_smooth_widths():
    from pvof.cases import smooth_widths
    w = smooth_widths(64, 512)
    assert w == [64, 80, 96, 128, 160, 192, 256, 320, 384, 512]
    for x in smooth_widths(2, 1024):
        odd = x
        while odd % 2 == 0:
            odd //= 2
        assert odd in (1, 3, 5) and x % 2 == 0


def test_droplet_batch_is_seeded_and_in_range():
    from pvof import cases
    a = cases.droplet_batch(12, seed=5, nxm_max=128)
    b = cases.droplet_batch(12, seed=5, nxm_max=128)
    widths = cases.smooth_widths(64, 128)
    for (ga, pa, pla, parta), (gb, pb, plb, partb) in zip(a, b):
        assert ga.NXM == gb.NXM and ga.NYM == 2 * ga.NXM and ga.NXM in widths
        assert np.array_equal(pla["F"], plb["F"]) and parta == partb
        assert 30.0 <= pa.contact_angle_deg <= 150.0
        (mobile, x, y, R, u, v, om, rho_s), = parta
        assert mobile == 0 and (x, y) == (1.0, 1.0) and 0.2 <= R <= 0.4
        h = 2.0 / ga.NXM
        assert math.isclose(pa.Cn, max(0.01, 0.75 * h))
        assert pa.rho2 == 1e-3 and pa.grav[1] == 0.0 and pa.surface_tension == 1
        F = pla["F"]
        assert F.min() >= 0.0 and F.max() <= 1.0 + 1e-15
        # the droplet holds liquid: about pi Rd^2 minus its overlap with the cylinder
        vol = F[:-1, :-1].sum() * h * h
        assert 0.2 < vol < math.pi * 0.6 ** 2
    c = cases.droplet_batch(12, seed=6, nxm_max=128)
    assert any(not np.array_equal(x[2]["F"], y[2]["F"]) for x, y in zip(a, c))


def test_interface_box_is_seeded_periodic_and_cubic():
    """The 3D precision-form case: cubic cells (the reference's uniform grid
    needs dx = dy = dz), x and z periodic with the interface modes periodic
    over the box, liquid below gas, the same fields for the same seed."""
    from pvof import abi, cases
    g, p, f = cases.interface_box(16, 24, 12, seed=3, Cn=0.1, amp_max=0.1)
    g2, _, f2 = cases.interface_box(16, 24, 12, seed=3, Cn=0.1, amp_max=0.1)
    assert g.geometry == abi.GEOM_3D and list(g.periodic) == [1, 0, 1]
    hx = (g.xmax - g.xmin) / g.NXM
    assert math.isclose((g.ymax - g.ymin) / g.NYM, hx) and math.isclose((g.zmax - g.zmin) / g.NZM, hx)
    NX, NY, NZ = cases.dims(g)
    C = f["F"]
    assert C.shape == (NZ, NY, NX) and np.array_equal(C, f2["F"])
    assert p.rho2 == 1e-3 and p.mu2 == 1e-2 and p.surface_tension == 1 and p.grav[1] == -1.0
    # the half cells at i = NX-1 and k = NZ-1 repeat the first cells (periodic modes)
    assert np.allclose(C[:, :, NX - 1], C[:, :, 0], atol=1e-12)
    assert np.allclose(C[NZ - 1], C[0], atol=1e-12)
    assert C[:, 0, :].min() > 0.99 and C[:, NY - 2, :].max() < 0.01
    blk = cases.field_to_block(g, C)
    assert blk.shape == cases.block_shape(g) and blk[cases.G:cases.G + NZ, cases.G:cases.G + NY, cases.G:cases.G + NX].sum() == C.sum()
    _, _, f3 = cases.interface_box(16, 24, 12, seed=4, Cn=0.1, amp_max=0.1)
    assert not np.array_equal(C, f3["F"])
