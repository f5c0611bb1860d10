"""Generate the golden fixtures of the two-phase substep from the reference.

Runs the reference's own time-step code, compiled from its sources by
oracle/ref/Makefile into oracle/_ref/ref_<case>, on small seeded cases and
stores the inputs, parameters, solver iteration counts and the fields after
every RK substep in tests/golden/<name>.npz.  The resolved-particle fixtures
(IBM_CASES) hold the inputs and outputs of the immersed-boundary routines of
one substep, from the routine driver oracle/ref/ibm_driver.c; the contact-line
fixtures (MCL_CASES) those of the contact-angle projection and the psi_LG
extension, from the same driver's "mcl" mode.

    python tests/golden/make_golden.py [--refsrc PATH]

This needs the reference source tree (REFSRC, default the mounted
reference); the fixtures it writes are committed so that the tests need
neither the tree nor the binaries.
"""
import argparse
import os
import re
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "oracle"))
sys.path.insert(0, os.path.join(REPO, "parties-vof-ibm_b200"))
import pyoracle as po  # noqa: E402
from pvof import abi, cases  # noqa: E402

FLOW_FIELDS = {"C_L": "C_L", "C_G": "C_G", "rho": "RHO", "mu": "MU", "ch_rhs_n": "CH_RHS_N",
               "u": "U", "v": "V", "p": "P"}
NG_FIELDS = {"u_explicit_old": "U_EXPLICIT_OLD", "v_explicit_old": "V_EXPLICIT_OLD",
             "u_visc_explicit_old": "U_VISC_EXPLICIT_OLD", "v_visc_explicit_old": "V_VISC_EXPLICIT_OLD"}
ST_FLOW = {"psi_LG": "PSI_LG"}
ST_NG = {"f_sigma_old_x": "FSIG_OLD_X", "f_sigma_old_y": "FSIG_OLD_Y"}

TIGHT = dict(ch_tol=1e-13, ch_iter_max=600, CG_ETOL=1e-15, CG_MAXIT=400, P_CG_ETOL=1e-13, P_CG_MAXIT=1000)

AXI_GRID = dict(NXM=24, NYM=48, rmax=1.0, zmax=2.0, radius=0.3, zc=0.7, Cn=0.04)
# axisymmetric cases with a resolved sphere on the axis: the bubble's top
# reaches into the sphere's diffuse shell
AXI_GRID_IBM = dict(NXM=32, NYM=64, rmax=1.0, zmax=2.0, radius=0.3, zc=0.7, Cn=0.04)
AXI_SPHERE = [(0, 0.0, 1.15, 0.2, 0.0, 0.0, 0.0, 2.5)]
# In the axisymmetric mode the pressure residual sqrt(r.M^-1 r) stalls at
# 2e-13 to 5e-13 (its rounding floor; the rows carry the weight r_c), where
# 1e-13 would make the stopping iteration depend on rounding: the tight
# axisymmetric cases stop the pressure solve at 1e-12, above that floor.
AXI_TIGHT = dict(TIGHT, P_CG_ETOL=1e-12)

# name, reference case, builder kwargs, steps, dt, snapshots kept (None = all)
CASES = [
    ("rt_small", "rt2d", dict(NXM=24, NYM=48, Lx=1.0, Ly=2.0, Cn=0.04, velocity_seed=5, velocity_amp=0.1), 2, 1e-3, None),
    ("rt_st_small", "rt2d_st", dict(NXM=24, NYM=48, Lx=1.0, Ly=2.0, Cn=0.04, surface_tension=True, We=100.0,
                                   velocity_seed=11, velocity_amp=0.1), 1, 1e-3, None),
    ("rt_tight", "rt2d", dict(NXM=24, NYM=48, Lx=1.0, Ly=2.0, Cn=0.04, velocity_seed=3, velocity_amp=0.1, **TIGHT),
     2, 1e-3, ["s0", "s1_0", "s1_2", "s2_2"]),
    # free-slip walls in y (BOTTOM/TOP_WALL_VELOCITY_FREESLIP)
    ("rt_fs_tight", "rt2d_fs", dict(NXM=24, NYM=48, Lx=1.0, Ly=2.0, Cn=0.04, velocity_seed=9, velocity_amp=0.1,
                                    wall_y=abi.WALL_FREESLIP, **TIGHT), 2, 1e-3, ["s0", "s1_0", "s1_2", "s2_2"]),
    # axisymmetric (r, z) bubble on the axis (AXISYM_RZ builds; the pressure
    # right-hand side carries the operator's row weight, oracle/ref/shim/axisym_rhs.c)
    ("axi_small", "axi2d", dict(_builder="rising_bubble", **AXI_GRID, velocity_seed=5, velocity_amp=0.1), 2, 1e-3,
     None),
    ("axi_tight", "axi2d", dict(_builder="rising_bubble", **AXI_GRID, velocity_seed=3, velocity_amp=0.1, **AXI_TIGHT), 2,
     1e-3, ["s0", "s1_0", "s1_2", "s2_2"]),
    ("axi_st_tight", "axi2d_st", dict(_builder="rising_bubble", **AXI_GRID, surface_tension=True, We=200.0,
                                      velocity_seed=21, velocity_amp=0.1, **AXI_TIGHT), 2, 1e-3,
     ["s0", "s1_0", "s1_2", "s2_2"]),
]

# long runs on a benchmark grid, only the end state kept (physical cells of
# C_L, u, v, p): name, reference case, builder kwargs, steps, dt.  The first is
# the planar instability on its full 128x512 grid (dt 1e-4, zero initial
# velocity), solver tolerances near machine precision.
LONG_CASES = [
    ("rt128x512_100steps", "rt2d", dict(NXM=128, NYM=512, Lx=1.0, Ly=4.0, Cn=0.01, **dict(TIGHT, P_CG_MAXIT=4000)),
     100, 1e-4),
    # the axisymmetric bubble with surface tension, 100 steps
    ("axi_st_100steps", "axi2d_st", dict(_builder="rising_bubble", NXM=32, NYM=64, rmax=1.0, zmax=2.0, radius=0.3,
                                         zc=0.7, Cn=0.04, surface_tension=True, We=200.0, **AXI_TIGHT), 100, 1e-3),
]

# long resolved-particle cases (final state only): the axisymmetric bubble below
# the fixed sphere on the axis, surface tension, contact angle 90 degrees
LONG_IBM_CASES = [
    ("ibm_axi_st_100steps", "ibm_axi_st", dict(_builder="rising_bubble", **AXI_GRID_IBM, surface_tension=True,
                                               We=200.0, **AXI_TIGHT), AXI_SPHERE, 90.0, 100, 1e-3),
]

# resolved-particle routine cases (oracle/ref/ibm_driver.c on the ibm2d build):
# name, builder kwargs, particles (mobile, x, y, R, u, v, omega_z, rho_s), dt, stage
IBM_CASES = [
    ("ibm_small", dict(NXM=32, NYM=128, Lx=1.0, Ly=4.0, Cn=0.04, velocity_seed=7, velocity_amp=0.1),
     [(0, 0.06, 1.2, 0.2, 0.0, 0.0, 0.0, 2.5), (1, 0.55, 2.7, 0.15, 0.2, -0.1, 0.7, 2.5)], 1e-3, 1),
    # axisymmetric (ibm_axi_st build): a fixed sphere on the axis cutting the
    # top of a bubble, its ring markers folded across the axis by the gathers
    # and spreads
    ("ibm_axi_small", dict(_builder="rising_bubble", _refcase="ibm_axi_st", **AXI_GRID_IBM, surface_tension=True,
                           We=200.0, velocity_seed=7, velocity_amp=0.1, _theta=90.0),
     AXI_SPHERE, 1e-3, 1),
]

# contact-line cases (oracle/ref/ibm_driver.c "mcl" mode on the ibm2d build):
# name, builder arguments, particles, contact angle in degrees.  Two fixed
# cylinders sit on the interface (one across the periodic x boundary) and a
# small mobile one just below it.
MCL_PARTICLES = [(0, 0.5, 1.0, 0.2, 0.0, 0.0, 0.0, 2.5), (0, 0.03, 1.04, 0.15, 0.0, 0.0, 0.0, 2.5),
                 (1, 0.78, 0.98, 0.07, 0.0, 0.0, 0.0, 2.5)]
MCL_GRID = dict(NXM=48, NYM=96, Lx=1.0, Ly=2.0, Cn=0.04)
MCL_CASES = [("mcl_theta60", MCL_GRID, MCL_PARTICLES, 60.0),
             ("mcl_theta120", MCL_GRID, MCL_PARTICLES, 120.0),
             ("mcl_theta30", MCL_GRID, MCL_PARTICLES, 30.0),
             # free-slip walls in y (ibm2d_fs): the interface and two cylinders
             # next to the bottom wall, so the characteristics cross it
             ("mcl_fs_theta45", dict(NXM=48, NYM=48, Lx=1.0, Ly=1.0, Cn=0.04, y0=0.12, amp=0.02,
                                     wall_y=abi.WALL_FREESLIP, _refcase="ibm2d_fs"),
              [(0, 0.5, 0.13, 0.1, 0.0, 0.0, 0.0, 2.5), (0, 0.03, 0.15, 0.08, 0.0, 0.0, 0.0, 2.5)], 45.0),
             # axisymmetric: the sphere on the axis in the bubble's top, the
             # characteristics folded at the axis
             ("mcl_axi_theta60", dict(_builder="rising_bubble", _refcase="ibm_axi_st", **AXI_GRID_IBM), AXI_SPHERE,
              60.0),
             ("mcl_axi_theta120", dict(_builder="rising_bubble", _refcase="ibm_axi_st", **AXI_GRID_IBM), AXI_SPHERE,
              120.0)]

# whole time steps with resolved cylinders (oracle/ref/ibm_driver.c "steps"
# mode): name, reference build, builder arguments, particles, contact angle,
# steps, dt.  Solver tolerances near machine precision.  The mobile case has
# one cylinder across the periodic x boundary and one on the interface.
IBM_STEP_PARTICLES = [(0, 0.5, 1.0, 0.2, 0.0, 0.0, 0.0, 2.5), (0, 0.03, 1.04, 0.15, 0.0, 0.0, 0.0, 2.5)]
IBM_MOBILE_PARTICLES = [(0, 0.5, 1.0, 0.2, 0.0, 0.0, 0.0, 2.5), (1, 0.02, 1.5, 0.1, 0.0, 0.0, 0.0, 2.5),
                        (1, 0.88, 1.0, 0.08, 0.0, 0.0, 0.0, 2.5)]
IBM_STEP_CASES = [
    ("ibm_mobile_st", "ibm2d_st", dict(NXM=32, NYM=64, Lx=1.0, Ly=2.0, Cn=0.04, surface_tension=True, We=100.0,
                                       velocity_seed=19, velocity_amp=0.1, **TIGHT), IBM_MOBILE_PARTICLES, 70.0, 2,
     1e-3),
    ("ibm_steps_st", "ibm2d_st", dict(NXM=32, NYM=64, Lx=1.0, Ly=2.0, Cn=0.04, surface_tension=True, We=100.0,
                                      velocity_seed=13, velocity_amp=0.1, **TIGHT), IBM_STEP_PARTICLES, 60.0, 2, 1e-3),
    ("ibm_steps", "ibm2d", dict(NXM=32, NYM=64, Lx=1.0, Ly=2.0, Cn=0.04, velocity_seed=17, velocity_amp=0.1, **TIGHT),
     IBM_STEP_PARTICLES, 120.0, 2, 1e-3),
    # axisymmetric: the static sphere on the axis in the top of a bubble
    # (the bubble-and-sphere benchmark case in small), surface tension
    ("ibm_axi_steps_st", "ibm_axi_st", dict(_builder="rising_bubble", **AXI_GRID_IBM, surface_tension=True, We=200.0,
                                            velocity_seed=23, velocity_amp=0.1, **AXI_TIGHT), AXI_SPHERE, 90.0, 2,
     1e-3),
    # the batching form's case in small: a sessile droplet on a static
    # cylinder (pvof.cases.droplet_on_cylinder), contact angle 60 degrees
    ("drop_cyl_st", "ibm2d_st", dict(_builder="droplet_on_cylinder", NXM=32, Rd=0.5, Rs=0.3, theta=60.0, **TIGHT),
     [(0, 1.0, 1.0, 0.3, 0.0, 0.0, 0.0, 1.0)], 60.0, 3, 1e-3),
]

# constant-density FFT Poisson cases (oracle/ref/fft_driver.c on the fft2d build):
# name, NXM, NYM, Lx, Ly, seed
FFT_CASES = [("fft_small", 32, 64, 1.0, 2.0, 1), ("fft_odd", 24, 40, 1.5, 2.5, 2)]

PARAM_KEYS = [k for k, _ in abi.Params._fields_]
GRID_KEYS = [k for k, _ in abi.GridDesc._fields_]


def struct_to_dict(s):
    out = {}
    for k, _ in s._fields_:
        v = getattr(s, k)
        out[k] = list(v) if hasattr(v, "__len__") else v
    return out


def parse_iterations(log):
    """Per-substep solver iteration counts from the reference's progress log."""
    ch = [int(m) for m in re.findall(r"VOF diffuse biharmonic \S+ to \S+ after (\d+) iterations", log)]
    u = [int(m) for m in re.findall(r"u-component of velocity converged to \S+ after (\d+) iterations", log)]
    v = [int(m) for m in re.findall(r"v-component of velocity converged to \S+ after (\d+) iterations", log)]
    p = [int(m) for m in re.findall(r"pressure converged to \S+ after (\d+) iterations", log)]
    w = [int(m) for m in re.findall(r"w-component of velocity converged to \S+ after (\d+) iterations", log)]
    if w:
        return np.array([ch, u, v, p, w], dtype=np.int64)
    return np.array([ch, u, v, p], dtype=np.int64)


def g_range(grid, plane, ng):
    """G-range part (NY, NX) of a k = 0 plane."""
    if ng:
        return plane
    NX, NY, _ = cases.dims(grid)
    G = cases.G
    return plane[G:G + NY, G:G + NX]


def build_case(kw):
    """(grid, params, planes, reference build) of a builder-kwargs dict whose
    optional keys _builder (a pvof.cases function, default rayleigh_taylor)
    and _refcase (default None) select the case."""
    build = dict(kw)
    builder = getattr(cases, build.pop("_builder", "rayleigh_taylor"))
    refcase = build.pop("_refcase", None)
    theta = build.pop("_theta", None)
    grid, params, planes = builder(**build)[:3]
    if theta is not None:
        params.contact_angle_deg = theta
    return grid, params, planes, refcase


def make(name, refcase, kw, steps, dt, keep, outdir, refsrc=None):
    grid, params, planes, _ = build_case(kw)
    if not os.path.exists(po.ref_binary(refcase)):
        po.build_reference(refcase, refsrc)
    with tempfile.TemporaryDirectory() as wd:
        cp = po.run_reference(refcase, wd, grid, params, planes, steps, dt, 1, substeps=True)
        data = {}
        st = bool(params.surface_tension)
        tags = ["s0"] + ["s%d_%d" % (n, rk) for n in range(1, steps + 1) for rk in range(3)]
        if keep is not None:
            tags = [t for t in tags if t in keep]
        for tag in tags:
            flow = dict(FLOW_FIELDS, **(ST_FLOW if st else {}))
            ngf = dict(NG_FIELDS, **(ST_NG if st else {}))
            for fname, pname in flow.items():
                a = po.read_reference_field(wd, tag, fname, grid)
                data["%s/%s" % (tag, pname)] = g_range(grid, a, False)
            for fname, pname in ngf.items():
                a = po.read_reference_field(wd, tag, fname, grid, ng=True)
                data["%s/%s" % (tag, pname)] = a
        data["iterations"] = parse_iterations(cp.stdout)
    for k, v in planes.items():
        data["init/" + k] = v
    meta = {"grid": struct_to_dict(grid), "params": struct_to_dict(params), "steps": steps, "dt": dt,
            "refcase": refcase, "builder": kw}
    data["meta"] = np.array(repr(meta))
    path = os.path.join(outdir, name + ".npz")
    np.savez_compressed(path, **data)
    return path


def make_long(name, refcase, kw, steps, dt, outdir, refsrc=None):
    build = dict(kw)
    builder = getattr(cases, build.pop("_builder", "rayleigh_taylor"))
    grid, params, planes = builder(**build)
    if not os.path.exists(po.ref_binary(refcase)):
        po.build_reference(refcase, refsrc)
    NX, NY, _ = cases.dims(grid)
    data = {}
    with tempfile.TemporaryDirectory() as wd:
        cp = po.run_reference(refcase, wd, grid, params, planes, steps, dt, steps, substeps=False, timeout=7200)
        tag = "s%d" % steps
        for fname, pname in (("C_L", "C_L"), ("u", "U"), ("v", "V"), ("p", "P")):
            a = g_range(grid, po.read_reference_field(wd, tag, fname, grid), False)
            data["%s/%s" % (tag, pname)] = a[:NY - 1, :NX - 1]
        data["iterations"] = parse_iterations(cp.stdout)
    # the initial planes are the builder's (deterministic); they are not stored
    meta = {"grid": struct_to_dict(grid), "params": struct_to_dict(params), "steps": steps, "dt": dt,
            "refcase": refcase, "builder": kw, "physical_only": True}
    data["meta"] = np.array(repr(meta))
    path = os.path.join(outdir, name + ".npz")
    np.savez_compressed(path, **data)
    return path


def make_long_ibm(name, refcase, kw, particles, theta, steps, dt, outdir, refsrc=None):
    """steps whole steps of the immersed-boundary driver (oracle/ref/ibm_driver.c
    "steps" mode); only the final state's physical cells are kept."""
    grid, params, planes, _ = build_case(kw)
    params.contact_angle_deg = theta
    if not os.path.exists(po.ref_binary(refcase)):
        po.build_reference(refcase, refsrc)
    NX, NY, _ = cases.dims(grid)
    fixed = [p[1:7] for p in particles if not p[0]]
    mobile = [p[1:7] for p in particles if p[0]]
    data = {}
    with tempfile.TemporaryDirectory() as wd:
        cp = po.run_reference_ibm(wd, grid, params, planes, fixed, mobile, dt, 0, case=refcase, mode="steps",
                                  nsteps=steps, timeout=7200)
        tag = "s%d" % steps
        for fname, pname in (("C_L", "C_L"), ("u", "U"), ("v", "V"), ("p", "P")):
            a = g_range(grid, po.read_reference_field(wd, tag, fname, grid), False)
            data["%s/%s" % (tag, pname)] = a[:NY - 1, :NX - 1]
        pid, X, U, Om = po.read_reference_particle_state(wd, tag)
        data[tag + "/pid"], data[tag + "/pX"], data[tag + "/pU"] = pid, X, U
        data["iterations"] = parse_iterations(cp.stdout)
    meta = {"grid": struct_to_dict(grid), "params": struct_to_dict(params), "particles": [list(p) for p in particles],
            "steps": steps, "dt": dt, "builder": kw, "refcase": refcase, "physical_only": True}
    data["meta"] = np.array(repr(meta))
    path = os.path.join(outdir, name + ".npz")
    np.savez_compressed(path, **data)
    return path


def make_ibm(name, kw, particles, dt, stage, outdir, refsrc=None):
    grid, params, planes, refcase = build_case(kw)
    refcase = refcase or "ibm2d"
    if not os.path.exists(po.ref_binary(refcase)):
        po.build_reference(refcase, refsrc)
    fixed = [p[1:7] for p in particles if not p[0]]
    mobile = [p[1:7] for p in particles if p[0]]
    data = {}
    with tempfile.TemporaryDirectory() as wd:
        cp = po.run_reference_ibm(wd, grid, params, planes, fixed, mobile, dt, stage, case=refcase)
        for fname in ["C_S", "C_L", "rho", "mu", "u", "v"]:
            data["i0/" + fname] = po.read_reference_field(wd, "i0", fname, grid)
        for tag, rhs in (("r0", True), ("r1", False), ("r2", True), ("r3", False), ("r4", True)):
            for fname in ["u", "v"]:
                data["%s/%s" % (tag, fname)] = po.read_reference_field(wd, tag, fname, grid)
            if rhs:
                for fname in ["u_rhs", "v_rhs", "u_implicit", "v_implicit"]:
                    data["%s/%s" % (tag, fname)] = po.read_reference_field(wd, tag, fname, grid, ng=True)
        for tag in ("r2", "r4"):
            F, T = po.read_reference_particles(wd, tag)
            data[tag + "/F"], data[tag + "/T"] = F, T
        mk = po.read_reference_markers(wd)
        data["markers/count"] = np.array([len(m[0]) for m in mk], dtype=np.int64)
        for q, key in enumerate(["x", "y", "vol", "flag"]):
            data["markers/" + key] = np.concatenate([m[q] for m in mk]) if mk else np.zeros(0)
        data["log"] = np.array(cp.stdout[-2000:])
    for k, v in planes.items():
        data["init/" + k] = v
    meta = {"grid": struct_to_dict(grid), "params": struct_to_dict(params), "dt": dt, "stage": stage,
            "particles": [list(p) for p in particles], "builder": kw, "refcase": refcase}
    data["meta"] = np.array(repr(meta))
    path = os.path.join(outdir, name + ".npz")
    np.savez_compressed(path, **data)
    return path


def make_mcl(name, kw, particles, theta, outdir, refsrc=None):
    grid, params, planes, refcase = build_case(kw)
    refcase = refcase or "ibm2d"
    build = {k: v for k, v in kw.items() if k != "_refcase"}
    params.contact_angle_deg = theta
    if not os.path.exists(po.ref_binary(refcase)):
        po.build_reference(refcase, refsrc)
    fixed = [p[1:7] for p in particles if not p[0]]
    mobile = [p[1:7] for p in particles if p[0]]
    data = {}
    with tempfile.TemporaryDirectory() as wd:
        po.run_reference_ibm(wd, grid, params, planes, fixed, mobile, 1e-3, 0, case=refcase, mode="mcl")
        for tag, names in (("i0", ["C_S", "C_L", "C_G"]), ("m1", ["C_L", "C_G", "C_S"]),
                           ("m2", ["C_L", "nx", "ny"]), ("m3", ["psi_LG", "C_L", "C_G"]), ("m4", ["psi_LG"])):
            for fname in names:
                data["%s/%s" % (tag, fname)] = po.read_reference_field(wd, tag, fname, grid)
    for k, v in planes.items():
        data["init/" + k] = v
    meta = {"grid": struct_to_dict(grid), "params": struct_to_dict(params), "particles": [list(p) for p in particles],
            "builder": build, "refcase": refcase}
    data["meta"] = np.array(repr(meta))
    path = os.path.join(outdir, name + ".npz")
    np.savez_compressed(path, **data)
    return path


def make_ibm_steps(name, refcase, kw, particles, theta, steps, dt, outdir, refsrc=None):
    grid, params, planes, _ = build_case(kw)
    params.contact_angle_deg = theta
    if not os.path.exists(po.ref_binary(refcase)):
        po.build_reference(refcase, refsrc)
    fixed = [p[1:7] for p in particles if not p[0]]
    mobile = [p[1:7] for p in particles if p[0]]
    st = bool(params.surface_tension)
    data = {}
    with tempfile.TemporaryDirectory() as wd:
        cp = po.run_reference_ibm(wd, grid, params, planes, fixed, mobile, dt, 0, case=refcase, mode="steps",
                                  nsteps=steps)
        for tag in ["s%d" % n for n in range(steps + 1)]:
            flow = dict(FLOW_FIELDS, C_S="C_S", **(ST_FLOW if st else {}))
            ngf = dict(NG_FIELDS, **(ST_NG if st else {}))
            for fname, pname in flow.items():
                if fname == "C_S":
                    if tag != "s0":
                        continue
                    a = po.read_reference_field(wd, "i0", "C_S", grid)
                else:
                    a = po.read_reference_field(wd, tag, fname, grid)
                data["%s/%s" % (tag, pname)] = g_range(grid, a, False)
            for fname, pname in ngf.items():
                data["%s/%s" % (tag, pname)] = po.read_reference_field(wd, tag, fname, grid, ng=True)
            F, T = po.read_reference_particles(wd, tag)
            data[tag + "/F"], data[tag + "/T"] = F, T
            pid, X, U, Om = po.read_reference_particle_state(wd, tag)
            data[tag + "/pid"], data[tag + "/pX"], data[tag + "/pU"], data[tag + "/pOmega"] = pid, X, U, Om
        data["iterations"] = parse_iterations(cp.stdout)
    for k, v in planes.items():
        data["init/" + k] = v
    meta = {"grid": struct_to_dict(grid), "params": struct_to_dict(params), "particles": [list(p) for p in particles],
            "steps": steps, "dt": dt, "builder": kw, "refcase": refcase}
    data["meta"] = np.array(repr(meta))
    path = os.path.join(outdir, name + ".npz")
    np.savez_compressed(path, **data)
    return path


def make_fft(name, NXM, NYM, Lx, Ly, seed, outdir, refsrc=None):
    """The reference's FFT solver runs in 3D with NZM = 2 (it needs an even
    z count) on a z-independent right-hand side; its k = 0 plane is the 2D
    solution.  The fixture keeps the 2D grid the library solves on."""
    grid, params, _ = cases.rayleigh_taylor(NXM, NYM, Lx=Lx, Ly=Ly, Cn=0.04)
    if not os.path.exists(po.ref_binary("fft2d")):
        po.build_reference("fft2d", refsrc)
    NX, NY, _ = cases.dims(grid)
    rng = np.random.default_rng(seed)
    rhs = np.zeros((NY, NX))
    rhs[:NY - 1, :NX - 1] = rng.standard_normal((NY - 1, NX - 1))
    rhs[:NY - 1, :NX - 1] -= rhs[:NY - 1, :NX - 1].mean()
    grid3 = abi.GridDesc.from_buffer_copy(grid)
    grid3.NZM = 2
    grid3.zmax = grid3.zmin + 2.0 * (grid.xmax - grid.xmin) / NXM
    with tempfile.TemporaryDirectory() as wd:
        po.write_parties_inp(os.path.join(wd, "parties.inp"), grid3, params)
        rhs.astype("<f8").tofile(os.path.join(wd, "rhs.bin"))
        subprocess.run([po.ref_binary("fft2d"), wd], check=True, capture_output=True, text=True, timeout=600)
        a = np.fromfile(os.path.join(wd, "out", "fft_deltap.bin"), dtype="<f8")
    G = cases.G
    blk = a.reshape(3 + 2 * G, NY + 2 * G, NX + 2 * G)
    data = {"rhs": rhs, "deltap": blk[G, G:G + NY - 1, G:G + NX - 1]}
    meta = {"grid": struct_to_dict(grid), "params": struct_to_dict(params), "refcase": "fft2d"}
    data["meta"] = np.array(repr(meta))
    path = os.path.join(outdir, name + ".npz")
    np.savez_compressed(path, **data)
    return path


# 3D cases (the reference built without TWOD_* flags, oracle/ref/cfg/rt3d_st.h):
# x and z periodic, no-slip walls in y, surface tension, gravity -y.  Fixtures
# hold the G range (NZ, NY, NX) of the flow fields and the no-ghost arrays.
BOX_FLOW = {"C_L": "C_L", "C_G": "C_G", "rho": "RHO", "mu": "MU", "ch_rhs_n": "CH_RHS_N", "u": "U", "v": "V",
            "w": "W", "p": "P", "psi_LG": "PSI_LG"}
BOX_NG = {"u_explicit_old": "U_EXPLICIT_OLD", "v_explicit_old": "V_EXPLICIT_OLD", "w_explicit_old": "W_EXPLICIT_OLD",
          "u_visc_explicit_old": "U_VISC_EXPLICIT_OLD", "v_visc_explicit_old": "V_VISC_EXPLICIT_OLD",
          "w_visc_explicit_old": "W_VISC_EXPLICIT_OLD", "f_sigma_old_x": "FSIG_OLD_X",
          "f_sigma_old_y": "FSIG_OLD_Y", "f_sigma_old_z": "FSIG_OLD_Z"}
BOX_TIGHT = dict(TIGHT, CG_ETOL=1e-13)
BOX_GRID = dict(NXM=16, NYM=24, NZM=12, Cn=0.1, amp_max=0.1, We=10.0, Re=100.0)
# name, reference case, builder kwargs, steps, dt, snapshots kept (None: the last only)
BOX_CASES = [
    ("box_st_tight", "rt3d_st", dict(BOX_GRID, rho_ratio=0.1, mu_ratio=0.1, velocity_seed=5, velocity_amp=0.05,
                                     **BOX_TIGHT), 2, 1e-3, ["s1_0", "s2_2"]),
    # the precision form's density and viscosity ratios on a small cube
    ("box_rho1e-3", "rt3d_st", dict(NXM=16, NYM=16, NZM=16, Cn=0.1, amp_max=0.1, We=100.0, Re=1000.0,
                                    rho_ratio=1e-3, mu_ratio=1e-2, velocity_seed=8, velocity_amp=0.02, **BOX_TIGHT),
     2, 1e-3, ["s2_2"]),
]
BOX_LONG = [("box_st_100steps", "rt3d_st", dict(BOX_GRID, rho_ratio=0.1, mu_ratio=0.1, **BOX_TIGHT), 100, 1e-3)]


def make_3d(name, refcase, kw, steps, dt, keep, outdir, refsrc=None):
    """A 3D fixture: the reference's fields after the kept substeps (or the
    last step), the initial fields and the solver iteration counts."""
    build = dict(kw)
    grid, params, fields = cases.interface_box(**build)
    if not os.path.exists(po.ref_binary(refcase)):
        po.build_reference(refcase, refsrc)
    NX, NY, NZ = cases.dims(grid)
    G = cases.G
    with tempfile.TemporaryDirectory() as wd:
        cp = po.run_reference(refcase, wd, grid, params, fields, steps, dt, 1 if keep else steps,
                              substeps=bool(keep), timeout=7200)
        data = {}
        tags = keep if keep else ["s%d" % steps]
        for tag in tags:
            for fname, pname in BOX_FLOW.items():
                a = np.fromfile(os.path.join(wd, "out", "%s_%s.bin" % (tag, fname)), dtype="<f8")
                a = a.reshape(cases.block_shape(grid))[G:G + NZ, G:G + NY, G:G + NX]
                data["%s/%s" % (tag, pname)] = a
            for fname, pname in BOX_NG.items():
                a = np.fromfile(os.path.join(wd, "out", "%s_%s.bin" % (tag, fname)), dtype="<f8")
                data["%s/%s" % (tag, pname)] = a.reshape(cases.block_shape(grid, ng=True))
        data["iterations"] = parse_iterations(cp.stdout)
    for k, v in fields.items():
        data["init/" + k] = v
    meta = {"grid": struct_to_dict(grid), "params": struct_to_dict(params), "steps": steps, "dt": dt,
            "refcase": refcase, "builder": kw}
    data["meta"] = np.array(repr(meta))
    path = os.path.join(outdir, name + ".npz")
    np.savez_compressed(path, **data)
    return path


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--refsrc", default=None)
    ap.add_argument("--out", default=HERE)
    ap.add_argument("--only", default=None, help="comma-separated fixture names")
    a = ap.parse_args()
    ap_only = a.only.split(",") if a.only else None
    for name, refcase, kw, steps, dt, keep in CASES:
        if ap_only is None or name in ap_only:
            print(make(name, refcase, kw, steps, dt, keep, a.out, a.refsrc))
    for name, refcase, kw, steps, dt in LONG_CASES:
        if ap_only is not None and name in ap_only:   # minutes of CPU: only on request
            print(make_long(name, refcase, kw, steps, dt, a.out, a.refsrc))
    for name, refcase, kw, parts, theta, steps, dt in LONG_IBM_CASES:
        if ap_only is not None and name in ap_only:
            print(make_long_ibm(name, refcase, kw, parts, theta, steps, dt, a.out, a.refsrc))
    for name, kw, parts, dt, stage in IBM_CASES:
        if ap_only is None or name in ap_only:
            print(make_ibm(name, kw, parts, dt, stage, a.out, a.refsrc))
    for name, kw, parts, theta in MCL_CASES:
        if ap_only is None or name in ap_only:
            print(make_mcl(name, kw, parts, theta, a.out, a.refsrc))
    for name, refcase, kw, parts, theta, steps, dt in IBM_STEP_CASES:
        if ap_only is None or name in ap_only:
            print(make_ibm_steps(name, refcase, kw, parts, theta, steps, dt, a.out, a.refsrc))
    for name, NXM, NYM, Lx, Ly, seed in FFT_CASES:
        if ap_only is None or name in ap_only:
            print(make_fft(name, NXM, NYM, Lx, Ly, seed, a.out, a.refsrc))
    for name, refcase, kw, steps, dt, keep in BOX_CASES:
        if ap_only is None or name in ap_only:
            print(make_3d(name, refcase, kw, steps, dt, keep, a.out, a.refsrc))
    for name, refcase, kw, steps, dt in BOX_LONG:
        if ap_only is not None and name in ap_only:
            print(make_3d(name, refcase, kw, steps, dt, None, a.out, a.refsrc))


if __name__ == "__main__":
    main()
