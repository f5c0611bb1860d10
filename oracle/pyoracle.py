"""Python access to the oracles.  TEST INFRASTRUCTURE ONLY.

* ``Oracle``: ctypes wrapper of liboracle.so, the CPU restatement of the
  reference's substep (pvof_oracle.c).
* ``run_reference``: runs the reference's own time-step code, compiled from
  its sources into oracle/_ref/ref_<case> (oracle/ref/Makefile), on a case
  directory written from the same initial planes.

Only the tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` use this module, as the checker; the product path never does.
"""
import ctypes as C
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(REPO, "parties-vof-ibm_b200"))
from pvof import abi, cases  # noqa: E402

LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")

ROUTINES = [
    "VOF_DIFFUSE_INIT", "VOF_DIFFUSE_STEP", "ADVECT_WENO5",
    "UPDATE_DENSITY_VISCOSITY", "COMPUTE_PSI_LG", "COMPUTE_F_SIGMA",
    "APPLY_F_SIGMA_OLD", "SWAP_F_SIGMA", "ADD_GRAVITY", "CELL_CENTER",
    "U_IMPLICIT_EXPLICIT", "V_IMPLICIT_EXPLICIT", "U_SET_RHS", "V_SET_RHS",
    "U_SOLVE_CG", "V_SOLVE_CG", "U_UPDATE_BOUNDARIES", "V_UPDATE_BOUNDARIES",
    "PRESSURE_SET_RHS", "PRESSURE_PRECONDITIONER", "PRESSURE_SOLVE_CG",
    "PRESSURE_PROJECT", "PRESSURE_DIVERGENCE",
]
ROUTINE = {n: i for i, n in enumerate(ROUTINES)}

_lib = None


def build():
    """Compile liboracle.so (make -C oracle)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        P = C.POINTER
        L.orc_create.argtypes = [P(abi.GridDesc), P(abi.Params), P(C.c_void_p)]
        L.orc_destroy.argtypes = [C.c_void_p]
        L.orc_destroy.restype = None
        L.orc_field_block_count.argtypes = [C.c_void_p, C.c_int]
        L.orc_field_block_count.restype = C.c_size_t
        L.orc_set_field.argtypes = [C.c_void_p, C.c_int, P(C.c_double), C.c_size_t]
        L.orc_get_field.argtypes = [C.c_void_p, C.c_int, P(C.c_double), C.c_size_t]
        L.orc_set_stage.argtypes = [C.c_void_p, C.c_int, C.c_double]
        L.orc_routine.argtypes = [C.c_void_p, C.c_int, P(abi.Stats)]
        L.orc_substep.argtypes = [C.c_void_p, P(abi.Stats)]
        L.orc_run_steps.argtypes = [C.c_void_p, C.c_int, C.c_double, P(abi.Stats)]
        L.orc_liquid_mass.argtypes = [C.c_void_p]
        L.orc_liquid_mass.restype = C.c_double
        _lib = L
    return _lib


class Oracle:
    """One case held by the CPU restatement."""

    def __init__(self, grid, params):
        self.grid, self.params = grid, params
        self.h = C.c_void_p()
        rc = lib().orc_create(C.byref(grid), C.byref(params), C.byref(self.h))
        if rc != 0:
            raise ValueError("orc_create failed: %d" % rc)

    def close(self):
        if self.h:
            lib().orc_destroy(self.h)
            self.h = C.c_void_p()

    __del__ = close

    def set_field(self, name, block):
        f = abi.FIELD[name]
        a = np.ascontiguousarray(block, dtype=np.float64).ravel()
        rc = lib().orc_set_field(self.h, f, a.ctypes.data_as(C.POINTER(C.c_double)), a.size)
        if rc != 0:
            raise ValueError("orc_set_field(%s) failed" % name)

    def get_field(self, name):
        f = abi.FIELD[name]
        n = lib().orc_field_block_count(self.h, f)
        a = np.empty(n, dtype=np.float64)
        lib().orc_get_field(self.h, f, a.ctypes.data_as(C.POINTER(C.c_double)), n)
        return cases.block_plane(self.grid, a, ng=f in abi.NG_FIELDS)

    def set_planes(self, planes):
        for name, plane in planes.items():
            ng = abi.FIELD[name] in abi.NG_FIELDS
            self.set_field(name, cases.plane_to_block(self.grid, plane, ng=ng))

    def set_stage(self, stage, dt):
        lib().orc_set_stage(self.h, stage, dt)

    def initialize(self):
        return self.routine("VOF_DIFFUSE_INIT")

    def routine(self, name):
        st = abi.Stats()
        rc = lib().orc_routine(self.h, ROUTINE[name], C.byref(st))
        return rc, st

    def substep(self):
        st = abi.Stats()
        rc = lib().orc_substep(self.h, C.byref(st))
        return rc, st

    def run_steps(self, n, dt):
        st = abi.Stats()
        rc = lib().orc_run_steps(self.h, n, dt, C.byref(st))
        if rc != 0:
            raise RuntimeError("orc_run_steps failed: %d" % rc)
        return st

    def liquid_mass(self):
        return lib().orc_liquid_mass(self.h)


# ---------------------------------------------------------------------------
# the reference's own code (oracle/_ref)
# ---------------------------------------------------------------------------

def write_parties_inp(path, grid, params):
    """The reference's INI input (PARTIES/src/IO/default.inp sections)."""
    p = params
    lines = [
        "[geometry]",
        "xmin = %.17g" % grid.xmin, "xmax = %.17g" % grid.xmax,
        "ymin = %.17g" % grid.ymin, "ymax = %.17g" % grid.ymax,
        "zmin = %.17g" % grid.zmin, "zmax = %.17g" % grid.zmax,
        "[grid]",
        "NXM = %d" % grid.NXM, "NYM = %d" % grid.NYM, "NZM = %d" % grid.NZM,
        "[twod]",
        "twod_slab_thickness = %.17g" % grid.slab_thickness,
        "axisym_theta_span = %.17g" % grid.theta_span,
        "[simulation]",
        "constant_dt = 1", "ghost_nodes = %d" % grid.ghost_nodes,
        "[flow]",
        "Re = %.17g" % p.Re, "dp_dx = %.17g" % p.dp_dx,
        "[vof]",
        "We = %.17g" % p.We, "rho1 = %.17g" % p.rho1, "rho2 = %.17g" % p.rho2,
        "mu1 = %.17g" % p.mu1, "mu2 = %.17g" % p.mu2,
        "Cn = %.17g" % p.Cn, "Pe_CH = %.17g" % p.Pe_CH,
        "weno_order = %d" % p.weno_order, "ch_iter_max = %d" % p.ch_iter_max,
        "ch_tol = %.17g" % p.ch_tol,
        "contact_angle_deg = %.17g" % p.contact_angle_deg,
        "[particle]",
        "grav = {%.17g, %.17g, %.17g}" % (p.grav[0], p.grav[1], p.grav[2]),
        "N_forcing_loops = %d" % p.N_forcing_loops,
        "[conc]",
        "richardson = {%.17g, 0}" % p.richardson,
        "[lsolve]",
        "P_CG_ETOL = %.17g" % p.P_CG_ETOL, "P_CG_MAXIT = %d" % p.P_CG_MAXIT,
        "CG_ETOL = %.17g" % p.CG_ETOL, "CG_MAXIT = %d" % p.CG_MAXIT,
    ]
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def ref_binary(case):
    return os.path.join(REF_DIR, "ref_" + case)


def build_reference(case, refsrc=None):
    """Compile the reference sources for one case (needs the reference tree)."""
    cmd = ["make", "-s", "-C", os.path.join(HERE, "ref"), "CASE=" + case, "-j8"]
    if refsrc:
        cmd.append("REFSRC=" + refsrc)
    subprocess.run(cmd, check=True)


def run_reference(case, workdir, grid, params, planes, nsteps, dt, dump_every=1,
                  substeps=False, timeout=3600, warmup=0):
    """Run the reference build ``case`` on the initial planes; returns the
    completed process (stdout has the solver log and the REF_TIMING line,
    which leaves out the first ``warmup`` of the ``nsteps`` steps)."""
    os.makedirs(workdir, exist_ok=True)
    write_parties_inp(os.path.join(workdir, "parties.inp"), grid, params)
    names = {"F": "init_C.bin", "U": "init_u.bin", "V": "init_v.bin", "W": "init_w.bin", "P": "init_p.bin"}
    for k, fn in names.items():
        if k in planes:
            np.ascontiguousarray(planes[k], dtype="<f8").tofile(os.path.join(workdir, fn))
    cmd = [ref_binary(case), workdir, str(nsteps), repr(float(dt)), str(dump_every),
           "1" if substeps else "0", str(int(warmup))]
    return subprocess.run(cmd, check=True, capture_output=True, text=True, timeout=timeout)


def run_reference_ibm(workdir, grid, params, planes, fixed, mobile, dt, stage, case="ibm2d", timeout=600,
                      mode="routines", nsteps=1):
    """Run the immersed-boundary driver (oracle/ref/ibm_driver.c) of the
    reference build ``case``: particles are rows (X, Y, R, U, V, Omega_z);
    ``mode`` is "routines", "mcl" or "steps" (``nsteps`` whole steps)."""
    os.makedirs(workdir, exist_ok=True)
    write_parties_inp(os.path.join(workdir, "parties.inp"), grid, params)
    names = {"F": "init_C.bin", "U": "init_u.bin", "V": "init_v.bin", "P": "init_p.bin"}
    for k, fn in names.items():
        if k in planes:
            np.ascontiguousarray(planes[k], dtype="<f8").tofile(os.path.join(workdir, fn))
    for fn, rows in (("particles_fixed.txt", fixed), ("particles_mobile.txt", mobile)):
        with open(os.path.join(workdir, fn), "w") as f:
            for r in rows:
                f.write(" ".join("%.17g" % float(x) for x in r) + "\n")
    cmd = [ref_binary(case), workdir, repr(float(dt)), str(int(stage)), mode, str(int(nsteps))]
    return subprocess.run(cmd, check=True, capture_output=True, text=True, timeout=timeout)


def read_reference_markers(workdir):
    """Markers dumped by the routine driver: one (X_L, Y_L, Vol_L, flag) tuple
    of arrays per list entry (mobile list first, then fixed)."""
    a = np.fromfile(os.path.join(workdir, "out", "markers.bin"), dtype="<f8")
    out, q = [], 0
    while q < a.size:
        n = int(a[q]); q += 1
        xs = a[q:q + n]; ys = a[q + n:q + 2 * n]; vol = a[q + 2 * n:q + 3 * n]; fl = a[q + 3 * n:q + 4 * n]
        q += 4 * n
        out.append((xs, ys, vol, fl))
    return out


def read_reference_particles(workdir, tag):
    """Per list entry F and T dumped by the routine driver, (n, 3) each."""
    a = np.loadtxt(os.path.join(workdir, "out", "particles_%s.txt" % tag), ndmin=2)
    return a[:, 0:3], a[:, 3:6]


def read_reference_particle_state(workdir, tag):
    """Per particle (lists in order, mobile first) ID, (X, Y), (U, V), Omega_z."""
    a = np.loadtxt(os.path.join(workdir, "out", "particles_%s.txt" % tag), ndmin=2)
    return a[:, 6].astype(np.int64), a[:, 7:9], a[:, 9:11], a[:, 11]


def read_reference_field(workdir, tag, name, grid, ng=False):
    """k = 0 plane of a dumped field (full ghosted plane for flow fields)."""
    a = np.fromfile(os.path.join(workdir, "out", "%s_%s.bin" % (tag, name)), dtype="<f8")
    return cases.block_plane(grid, a, ng=ng)
