"""Synthetic two-phase cases and the reference field layout on the host.

Each case returns a grid description, the solver parameters and the initial
fields on the G range of one k plane ([j][i], i fastest, NX = NXM+1 by
NY = NYM+1 values, the half cell included).  ``plane_to_block`` expands such a
plane into the reference's ghosted block layout (PARTIES/src/Memory.c:36-89)
the same way the reference's arrays hold it: values on the G range of every k
plane, zeros in the ghost frame.

The initial conditions are injected directly because the reference's own
initialisers (PARTIES/src/IO/VoF_Init.c) use other amplitudes and profiles.
"""
import math

import numpy as np

from . import abi

G = 3  # ghost_nodes


def dims(grid):
    return grid.NXM + 1, grid.NYM + 1, grid.NZM + 1


def block_shape(grid, ng=False):
    NX, NY, NZ = dims(grid)
    if ng:
        return (NZ, NY, NX)
    return (NZ + 2 * G, NY + 2 * G, NX + 2 * G)


def plane_to_block(grid, plane, ng=False):
    """Expand a G-range plane (NY, NX) into a host block of the field layout."""
    NX, NY, NZ = dims(grid)
    plane = np.asarray(plane, dtype=np.float64)
    assert plane.shape == (NY, NX), (plane.shape, (NY, NX))
    blk = np.zeros(block_shape(grid, ng), dtype=np.float64)
    if ng:
        blk[:, :, :] = plane[None]
    else:
        blk[G:G + NZ, G:G + NY, G:G + NX] = plane[None]
    return blk


def block_plane(grid, block, ng=False):
    """The k = 0 plane of a host block, ghosts included for flow fields:
    shape (NY+2G, NX+2G) for flow fields, (NY, NX) for no-ghost fields."""
    blk = np.asarray(block).reshape(block_shape(grid, ng))
    return blk[0] if ng else blk[G]


def interior(grid, plane2d, ghosted=True):
    """Physical cells (i < NX-1, j < NY-1) of a k = 0 plane."""
    NX, NY, _ = dims(grid)
    if ghosted:
        return plane2d[G:G + NY - 1, G:G + NX - 1]
    return plane2d[:NY - 1, :NX - 1]


def default_params(**kw):
    p = abi.Params()
    p.Re = 100.0
    p.We = 1.0
    p.rho1 = 1.0
    p.rho2 = 1.0
    p.mu1 = 1.0
    p.mu2 = 1.0
    p.Cn = 0.01
    p.Pe_CH = 100.0
    p.grav[0], p.grav[1], p.grav[2] = 0.0, -1.0, 0.0
    p.richardson = 1.0
    p.dp_dx = 0.0
    p.weno_order = 5
    p.ch_iter_max = 300
    p.ch_tol = 1e-9
    p.CG_MAXIT = 120
    p.CG_ETOL = 1e-9
    p.P_CG_MAXIT = 300
    p.P_CG_ETOL = 1e-7
    p.surface_tension = 0
    p.gravity = 1
    p.contact_angle_deg = 90.0
    p.N_forcing_loops = 2
    p.stencil_fp32 = 0
    p.pressure_warm_start = 0
    p.pressure_preconditioner = 0
    p.velocity_cg_unregularized = 0
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def planar_grid(NXM, NYM, xmax, ymax, periodic_x=True, wall_y=abi.WALL_NOSLIP):
    g = abi.GridDesc()
    g.NXM, g.NYM, g.NZM = NXM, NYM, 1
    g.ghost_nodes = G
    g.geometry = abi.GEOM_PLANAR
    g.periodic[0], g.periodic[1], g.periodic[2] = (1 if periodic_x else 0), 0, 1
    for f in range(6):
        g.wall[f] = abi.WALL_NOSLIP
    g.wall[abi.BOTTOM] = wall_y
    g.wall[abi.TOP] = wall_y
    g.xmin, g.xmax = 0.0, float(xmax)
    g.ymin, g.ymax = 0.0, float(ymax)
    # 2D slab: thickness = min(hx, hy) (PARTIES/src/IO/Input.c:51-67)
    hx = (g.xmax - g.xmin) / float(NXM)
    hy = (g.ymax - g.ymin) / float(NYM)
    g.slab_thickness = min(hx, hy)
    g.zmin, g.zmax = 0.0, g.slab_thickness
    g.theta_span = 2.0 * math.pi
    return g


def cell_centres(grid):
    NX, NY, _ = dims(grid)
    dx = (grid.xmax - grid.xmin) / float(NX - 1)
    dy = (grid.ymax - grid.ymin) / float(NY - 1)
    xc = grid.xmin + (0.5 + np.arange(NX)) * dx
    yc = grid.ymin + (0.5 + np.arange(NY)) * dy
    xu = grid.xmin + np.arange(NX) * dx
    yv = grid.ymin + np.arange(NY) * dy
    return xc, yc, xu, yv


def rayleigh_taylor(NXM=128, NYM=512, Lx=1.0, Ly=4.0, Cn=0.01, amp=0.05,
                    atwood=0.5, Re=3000.0, surface_tension=False, We=100.0,
                    velocity_seed=None, velocity_amp=0.0, wall_y=abi.WALL_NOSLIP, y0=None, **param_kw):
    """Planar two-phase instability: x periodic, no-slip walls in y, heavy
    fluid (C = 1) on top of an interface at mid-height perturbed by
    amp*cos(2 pi x / Lx); C = 0.5 (1 + tanh(d / (sqrt(2) Cn))).

    ``velocity_seed`` adds a seeded random divergence-carrying velocity of
    size ``velocity_amp`` (for parity cases that exercise the advection and
    projection from the first substep); ``wall_y`` is the wall type of both
    y walls, ``y0`` the interface height (default mid-height)."""
    grid = planar_grid(NXM, NYM, Lx, Ly, wall_y=wall_y)
    rho2 = (1.0 - atwood) / (1.0 + atwood)
    params = default_params(Re=Re, rho1=1.0, rho2=rho2, mu1=1.0, mu2=1.0,
                            Cn=Cn, Pe_CH=1.0 / Cn,
                            surface_tension=1 if surface_tension else 0,
                            We=We, **param_kw)
    xc, yc, xu, yv = cell_centres(grid)
    X, Y = np.meshgrid(xc, yc)
    d = Y - ((0.5 * Ly if y0 is None else y0) + amp * np.cos(2.0 * np.pi * X / Lx))
    C = 0.5 * (1.0 + np.tanh(d / (math.sqrt(2.0) * Cn)))
    NX, NY, _ = dims(grid)
    u = np.zeros((NY, NX))
    v = np.zeros((NY, NX))
    p = np.zeros((NY, NX))
    if velocity_seed is not None:
        rng = np.random.default_rng(velocity_seed)
        Xu, Yc = np.meshgrid(xu, yc)
        Xc, Yv = np.meshgrid(xc, yv)
        k1, k2 = rng.integers(1, 4, size=2)
        ph = rng.uniform(0, 2 * np.pi, size=4)
        u = velocity_amp * (np.sin(2 * np.pi * k1 * Xu / Lx + ph[0]) * np.sin(np.pi * Yc / Ly)
                            + 0.3 * rng.standard_normal((NY, NX)))
        v = velocity_amp * (np.cos(2 * np.pi * k2 * Xc / Lx + ph[1]) * np.sin(np.pi * Yv / Ly)
                            + 0.3 * rng.standard_normal((NY, NX)))
        p = velocity_amp * rng.standard_normal((NY, NX))
    return grid, params, {"F": C, "U": u, "V": v, "P": p}


def axisym_grid(NXM, NYM, rmax, zmax):
    """Axisymmetric (r, z) grid: the symmetry axis at r = 0 (left), no-slip
    walls at r = rmax and at z = 0, zmax; full 2 pi ring."""
    g = abi.GridDesc()
    g.NXM, g.NYM, g.NZM = NXM, NYM, 1
    g.ghost_nodes = G
    g.geometry = abi.GEOM_AXISYM
    g.periodic[0], g.periodic[1], g.periodic[2] = 0, 0, 1
    for f in range(6):
        g.wall[f] = abi.WALL_NOSLIP
    g.xmin, g.xmax = 0.0, float(rmax)
    g.ymin, g.ymax = 0.0, float(zmax)
    hx = (g.xmax - g.xmin) / float(NXM)
    hy = (g.ymax - g.ymin) / float(NYM)
    g.slab_thickness = min(hx, hy)
    g.zmin, g.zmax = 0.0, g.slab_thickness
    g.theta_span = 2.0 * math.pi
    return g


def rising_bubble(NXM=64, NYM=128, rmax=2.0, zmax=4.0, radius=0.5, zc=1.0, Cn=0.04, rho_ratio=0.1,
                  mu_ratio=0.1, Re=100.0, surface_tension=False, We=200.0, velocity_seed=None, velocity_amp=0.0,
                  **param_kw):
    """Axisymmetric bubble (C = 0 inside a sphere of ``radius`` on the axis at
    z = zc) in liquid (C = 1); C = 0.5 (1 + tanh((d - radius) / (sqrt(2) Cn)))."""
    grid = axisym_grid(NXM, NYM, rmax, zmax)
    params = default_params(Re=Re, rho1=1.0, rho2=rho_ratio, mu1=1.0, mu2=mu_ratio, Cn=Cn, Pe_CH=1.0 / Cn,
                            surface_tension=1 if surface_tension else 0, We=We, **param_kw)
    xc, yc, xu, yv = cell_centres(grid)
    X, Y = np.meshgrid(xc, yc)
    dist = np.sqrt(X * X + (Y - zc) ** 2)
    C = 0.5 * (1.0 + np.tanh((dist - radius) / (math.sqrt(2.0) * Cn)))
    NX, NY, _ = dims(grid)
    u = np.zeros((NY, NX))
    v = np.zeros((NY, NX))
    p = np.zeros((NY, NX))
    if velocity_seed is not None:
        rng = np.random.default_rng(velocity_seed)
        Xu, Yc = np.meshgrid(xu, yc)
        Xc, Yv = np.meshgrid(xc, yv)
        u = velocity_amp * (np.sin(np.pi * Xu / rmax) * np.sin(np.pi * Yc / zmax) + 0.3 * rng.standard_normal((NY, NX)))
        v = velocity_amp * (np.sin(np.pi * Xc / rmax) * np.sin(np.pi * Yv / zmax) + 0.3 * rng.standard_normal((NY, NX)))
        p = velocity_amp * rng.standard_normal((NY, NX))
    return grid, params, {"F": C, "U": u, "V": v, "P": p}



def sinking_cylinders(NXM=1024, NYM=1024, L=1.0, Cn=0.005, rho_ratio=1e-3, R=0.1, rho_s=2.5, theta=110.0,
                      Re=100.0, We=100.0, y0=0.6, **param_kw):
    """Three mobile cylinders (radius R, solid/liquid density rho_s) centred on
    a flat interface at y0 of an L x L box (x periodic, no-slip walls in y),
    liquid (C = 1) below, gas of density ratio rho_ratio above, surface
    tension with contact angle theta (degrees): the learned-warm-start
    benchmark case.  Returns (grid, params, planes, particles), particles as
    rows (mobile, x, y, R, u, v, omega_z, rho_s)."""
    grid, params, planes = rayleigh_taylor(NXM, NYM, Lx=L, Ly=L, Cn=Cn, amp=0.0, atwood=(1 - rho_ratio) /
                                           (1 + rho_ratio), Re=Re, surface_tension=True, We=We, y0=y0, **param_kw)
    # liquid below the interface: flip the heavy-fluid-on-top profile
    planes["F"] = 1.0 - planes["F"]
    params.rho1, params.rho2 = 1.0, rho_ratio
    params.contact_angle_deg = theta
    parts = [(1, L * x, y0, R, 0.0, 0.0, 0.0, rho_s) for x in (0.2, 0.5, 0.8)]
    return grid, params, planes, parts


def droplet_on_cylinder(NXM=128, Rd=0.5, Rs=0.3, theta=90.0, Cn=0.01, rho_ratio=1e-3, mu_ratio=1e-2, Re=100.0,
                        We=10.0, **param_kw):
    """Sessile droplet on a static cylinder, the synthetic stand-in for the
    reference's VoF_init_planar_droplet_on_static_cylinder_theta
    (IO/VoF_Init.c:2496-2597) with seeded radii: that case is the half of a
    symmetric problem on a free-slip symmetry plane; here the whole problem
    sits in a box x in [0, 2] (periodic) by y in [0, 4] (no-slip walls) of
    NXM x 2 NXM square cells.  The fixed cylinder of radius Rs is centred at
    (1, 1), the liquid droplet of radius Rd at (1, 1 + 0.75 (Rs + Rd)) (the
    reference's centre distance 0.75 at Rs = Rd = 0.5); gas of density ratio
    rho_ratio and viscosity ratio mu_ratio around, surface tension with
    contact angle theta (degrees), no gravity.  C is the reference's cell
    average over 5 x 5 sub-samples of 0.5 (1 + tanh(s / (2 sqrt 2 Cn))), s the
    signed distance to the droplet's circle, capped by 1 - C_S of the
    cylinder's diffuse profile.  Cn is raised to 0.75 h where h is too coarse
    to resolve it (the reference's own value for an unset Cn).  Returns
    (grid, params, planes, particles), particles as rows (mobile, x, y, R, u,
    v, omega_z, rho_s)."""
    NYM = 2 * NXM
    grid = planar_grid(NXM, NYM, 2.0, 4.0)
    h = 2.0 / NXM
    cn = max(Cn, 0.75 * h)
    params = default_params(Re=Re, rho1=1.0, rho2=rho_ratio, mu1=1.0, mu2=mu_ratio, Cn=cn, Pe_CH=1.0 / cn,
                            surface_tension=1, We=We, **param_kw)
    params.grav[0], params.grav[1], params.grav[2] = 0.0, 0.0, 0.0
    params.contact_angle_deg = theta
    xs, ys = 1.0, 1.0
    xd, yd = xs, ys + 0.75 * (Rs + Rd)
    xc, yc, _, _ = cell_centres(grid)
    S = 5
    off = (np.arange(S) + 0.5) / S - 0.5
    bw = 2.0 * math.sqrt(2.0) * cn
    shift_S = math.sqrt(2.0) * math.log(19.0) * cn
    denom_S = 2.0 * math.sqrt(2.0) * cn
    C = np.zeros((yc.size, xc.size))
    for oy in off:
        Y = (yc + oy * h)[:, None]
        for ox in off:
            X = (xc + ox * h)[None, :]
            cl = 0.5 * (1.0 + np.tanh((Rd - np.sqrt((X - xd) ** 2 + (Y - yd) ** 2)) / bw))
            cs = 0.5 - 0.5 * np.tanh((np.sqrt((X - xs) ** 2 + (Y - ys) ** 2) - (Rs - shift_S)) / denom_S)
            C += np.clip(np.minimum(cl, np.maximum(1.0 - cs, 0.0)), 0.0, None) / (S * S)
    z = np.zeros_like(C)
    return grid, params, {"F": C, "U": z, "V": z.copy(), "P": z.copy()}, [(0, xs, ys, Rs, 0.0, 0.0, 0.0, 1.0)]


def smooth_widths(lo, hi):
    """x cell counts in [lo, hi] of the form 2^a, 3 2^a or 5 2^a (the widths
    the spectral pressure preconditioner's row transforms take)."""
    out = set()
    for r in (1, 3, 5):
        w = r * 2
        while w <= hi:
            if w >= lo:
                out.add(w)
            w *= 2
    return sorted(out)


def droplet_batch(n=64, seed=0, nxm_min=64, nxm_max=512, **kw):
    """The batching form's cases: n sessile droplets on static cylinders
    (droplet_on_cylinder) with NXM drawn log-uniformly in [nxm_min, nxm_max]
    and taken to the nearest (in log) of smooth_widths (64, 80, 96, 128, 160,
    192, 256, 320, 384, 512 for the default range; NYM = 2 NXM), droplet
    radius U(0.3, 0.6), cylinder radius U(0.2, 0.4), contact angle
    U(30, 150) degrees, all seeded.  Returns a list of (grid, params, planes,
    particles)."""
    rng = np.random.default_rng(seed)
    widths = smooth_widths(nxm_min, nxm_max)
    out = []
    for _ in range(n):
        x = rng.uniform(math.log(nxm_min), math.log(nxm_max))
        nxm = min(widths, key=lambda w: (abs(math.log(w) - x), w))
        Rd, Rs, th = rng.uniform(0.3, 0.6), rng.uniform(0.2, 0.4), rng.uniform(30.0, 150.0)
        out.append(droplet_on_cylinder(nxm, Rd=Rd, Rs=Rs, theta=th, **kw))
    return out


def box_grid(NXM, NYM, NZM, Lx=2.0, Ly=2.0, Lz=2.0, wall_y=abi.WALL_NOSLIP):
    """3D box: x and z periodic, walls of type ``wall_y`` at y = 0 and Ly."""
    g = abi.GridDesc()
    g.NXM, g.NYM, g.NZM = NXM, NYM, NZM
    g.ghost_nodes = G
    g.geometry = abi.GEOM_3D
    g.periodic[0], g.periodic[1], g.periodic[2] = 1, 0, 1
    for f in range(6):
        g.wall[f] = abi.WALL_NOSLIP
    g.wall[abi.BOTTOM] = wall_y
    g.wall[abi.TOP] = wall_y
    g.xmin, g.xmax = 0.0, float(Lx)
    g.ymin, g.ymax = 0.0, float(Ly)
    g.zmin, g.zmax = 0.0, float(Lz)
    hx = (g.xmax - g.xmin) / float(NXM)
    hy = (g.ymax - g.ymin) / float(NYM)
    g.slab_thickness = min(hx, hy)
    g.theta_span = 2.0 * math.pi
    return g


def field_to_block(grid, arr, ng=False):
    """A host block of the field layout from a G-range plane (NY, NX), copied
    to every k plane, or a G-range array (NZ, NY, NX)."""
    arr = np.asarray(arr, dtype=np.float64)
    if arr.ndim == 2:
        return plane_to_block(grid, arr, ng)
    NX, NY, NZ = dims(grid)
    assert arr.shape == (NZ, NY, NX), (arr.shape, (NZ, NY, NX))
    blk = np.zeros(block_shape(grid, ng), dtype=np.float64)
    if ng:
        blk[:] = arr
    else:
        blk[G:G + NZ, G:G + NY, G:G + NX] = arr
    return blk


def interface_box(NXM=256, NYM=256, NZM=256, L=2.0, seed=3, modes=16, amp_max=0.02, Cn=0.005, rho_ratio=1e-3,
                  mu_ratio=1e-2, Re=1000.0, We=100.0, velocity_seed=None, velocity_amp=0.0, **param_kw):
    """3D liquid layer under gas in an L^3 box (x, z periodic, no-slip walls in
    y), the precision form's case: the interface height is
    h(x, z) = L/2 + sum_k a_k cos(pi (n_x x + n_z z) + phi_k) over ``modes``
    seeded (n_x, n_z) in {1..4}^2, a_k ~ U(0, amp_max), phi_k ~ U(0, 2 pi);
    liquid (C = 1) below, C = 0.5 (1 + tanh((h - y) / (sqrt(2) Cn))); gas of
    density ratio ``rho_ratio`` and viscosity ratio ``mu_ratio``; surface
    tension at Weber number We and gravity -y.  The cells are cubes of side
    L / NXM (the reference's uniform grid needs dx = dy = dz), so the box is
    L x (NYM/NXM) L x (NZM/NXM) L and the modes are cos(2 pi (n_x x / Lx +
    n_z z / Lz) + phi_k), the same as above for a cube.  ``velocity_seed`` adds
    a seeded random velocity of size ``velocity_amp`` (parity cases).  Returns
    (grid, params, fields) with G-range arrays (NZ, NY, NX)."""
    h = L / float(NXM)
    Lx, Ly, Lz = L, h * NYM, h * NZM
    grid = box_grid(NXM, NYM, NZM, Lx, Ly, Lz)
    params = default_params(Re=Re, rho1=1.0, rho2=rho_ratio, mu1=1.0, mu2=mu_ratio, Cn=Cn, Pe_CH=1.0 / Cn,
                            surface_tension=1, We=We, **param_kw)
    rng = np.random.default_rng(seed)
    nx = rng.integers(1, 5, size=modes)
    nz = rng.integers(1, 5, size=modes)
    a = rng.uniform(0.0, amp_max, size=modes)
    ph = rng.uniform(0.0, 2.0 * np.pi, size=modes)
    NX, NY, NZ = dims(grid)
    xc = (0.5 + np.arange(NX)) * h
    yc = (0.5 + np.arange(NY)) * h
    zc = (0.5 + np.arange(NZ)) * h
    Z, X = np.meshgrid(zc, xc, indexing="ij")
    H = 0.5 * Ly + sum(a[q] * np.cos(2.0 * np.pi * (nx[q] * X / Lx + nz[q] * Z / Lz) + ph[q]) for q in range(modes))
    C = 0.5 * (1.0 + np.tanh((H[:, None, :] - yc[None, :, None]) / (math.sqrt(2.0) * Cn)))
    fields = {"F": C}
    shape = (NZ, NY, NX)
    if velocity_seed is not None:
        vr = np.random.default_rng(velocity_seed)
        fields["U"] = velocity_amp * vr.standard_normal(shape)
        fields["V"] = velocity_amp * vr.standard_normal(shape)
        fields["W"] = velocity_amp * vr.standard_normal(shape)
        fields["P"] = velocity_amp * vr.standard_normal(shape)
    else:
        for k in ("U", "V", "W", "P"):
            fields[k] = np.zeros(shape)
    return grid, params, fields
