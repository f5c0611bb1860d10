"""ctypes binding of the CUDA library (pvof/libpvof.so, include/pvof.h).

``Solver`` owns one pvof context: upload the initial planes, initialise,
advance, download.  The library must be present and a CUDA device visible;
otherwise construction raises -- there is no CPU path.
"""
import ctypes as C
import os

import numpy as np

from . import abi, cases

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libpvof.so")
_lib = None


class PvofError(RuntimeError):
    pass


def load():
    """Load libpvof.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise PvofError("libpvof.so is not built (python parties-vof-ibm_b200/build.py)")
    L = C.CDLL(LIB_PATH)
    P = C.POINTER
    V = C.c_void_p
    L.pvof_abi_version.restype = C.c_int
    L.pvof_last_error.restype = C.c_char_p
    L.pvof_device_count.restype = C.c_int
    L.pvof_create.argtypes = [P(abi.GridDesc), P(abi.Params), C.c_int, P(V)]
    L.pvof_destroy.argtypes = [V]
    L.pvof_field_block_count.argtypes = [V, C.c_int]
    L.pvof_field_block_count.restype = C.c_size_t
    L.pvof_upload_field.argtypes = [V, C.c_int, P(C.c_double), C.c_size_t]
    L.pvof_download_field.argtypes = [V, C.c_int, P(C.c_double), C.c_size_t]
    L.pvof_synchronize.argtypes = [V]
    L.pvof_set_stage.argtypes = [V, C.c_int, C.c_double]
    L.pvof_initialize.argtypes = [V]
    for name in ["pvof_VOF_DIFFUSE_init", "pvof_VOF_DIFFUSE_advect_WENO5",
                 "pvof_VOF_update_density_viscosity", "pvof_VOF_DIFFUSE_compute_psi_LG",
                 "pvof_VOF_DIFFUSE_compute_f_sigma", "pvof_VOF_apply_f_sigma_old",
                 "pvof_VOF_swap_f_sigma", "pvof_Velocity_add_gravity_2_RHS",
                 "pvof_Velocity_cell_center", "pvof_Pressure_set_RHS",
                 "pvof_Pressure_compute_preconditioner", "pvof_Pressure_project_velocity"]:
        getattr(L, name).argtypes = [V]
    L.pvof_VOF_DIFFUSE_step.argtypes = [V, P(abi.Stats)]
    for name in ["pvof_Velocity_set_implicit_explicit", "pvof_Velocity_set_RHS",
                 "pvof_Velocity_update_boundaries"]:
        getattr(L, name).argtypes = [V, C.c_char]
    L.pvof_Velocity_solve_cg.argtypes = [V, C.c_char, P(abi.Stats)]
    L.pvof_Pressure_solve_cg.argtypes = [V, P(abi.Stats)]
    L.pvof_Pressure_compute_velocity_divergence.argtypes = [V, P(C.c_double)]
    L.pvof_substep.argtypes = [V, P(abi.Stats)]
    L.pvof_run_steps.argtypes = [V, C.c_int, C.c_double, P(abi.Stats)]
    L.pvof_liquid_mass.argtypes = [V, P(C.c_double)]
    L.pvof_launch_count.argtypes = [V]
    L.pvof_launch_count.restype = C.c_longlong
    L.pvof_timer_start.argtypes = [V]
    L.pvof_timer_stop.argtypes = [V, P(C.c_double)]
    L.pvof_flush_l2.argtypes = [V]
    L.pvof_set_solver_timing.argtypes = [V, C.c_int]
    L.pvof_set_autotune.argtypes = [V, C.c_int]
    L.pvof_autotune_active.argtypes = [V]
    L.pvof_autotune_entries.argtypes = [V]
    L.pvof_autotune_entry.argtypes = [V, C.c_int, P(C.c_char_p), P(C.c_int), P(C.c_int), P(C.c_double),
                                      P(C.c_double)]
    L.pvof_set_graphs.argtypes = [V, C.c_int]
    L.pvof_graph_replays.argtypes = [V]
    L.pvof_graph_replays.restype = C.c_longlong
    L.pvof_set_cluster_solvers.argtypes = [V, C.c_int]
    L.pvof_set_pressure_pairs.argtypes = [V, C.c_int]
    L.pvof_clamp_mass_total.argtypes = [V, P(C.c_double)]
    L.pvof_solver_timing.argtypes = [V, C.c_int, P(C.c_double), P(C.c_longlong), P(C.c_longlong), P(C.c_longlong)]
    L.pvof_solver_kernel.argtypes = [V, C.c_int]
    L.pvof_set_particles.argtypes = [V, P(abi.Particle), C.c_int]
    L.pvof_Lagrangian_flag_points.argtypes = [V]
    L.pvof_particle_entries.argtypes = [V]
    L.pvof_particle_forces.argtypes = [V, P(C.c_double), P(C.c_double), C.c_int]
    L.pvof_particle_markers.argtypes = [V, C.c_int, P(C.c_double), P(C.c_double), P(C.c_double), P(C.c_int), C.c_int]
    L.pvof_VOF_DIFFUSE_compute_C_S.argtypes = [V]
    L.pvof_Velocity_solve_explicit.argtypes = [V, C.c_char]
    L.pvof_Lagrangian_force.argtypes = [V, C.c_int]
    L.pvof_Pressure_solve_fft.argtypes = [V]
    L.pvof_VOF_DIFFUSE_compute_solid_normals_MCL.argtypes = [V]
    L.pvof_VOF_DIFFUSE_apply_contact_angle.argtypes = [V]
    L.pvof_VOF_DIFFUSE_extend_psi_LG_contact_angle.argtypes = [V]
    L.pvof_Particle_initialize_velocities.argtypes = [V]
    L.pvof_Lagrangian_advect_particles.argtypes = [V]
    L.pvof_get_particles.argtypes = [V, P(abi.Particle), P(C.c_int), P(C.c_double), P(C.c_double), C.c_int]
    L.pvof_cnn_param_count.restype = C.c_size_t
    L.pvof_cnn_param_count.argtypes = []
    L.pvof_cnn_work_floats.restype = C.c_size_t
    L.pvof_cnn_work_floats.argtypes = [C.c_int, C.c_int]
    L.pvof_cnn_forward.argtypes = [V, V, V, V, C.c_int, C.c_int, V, V]
    L.pvof_cnn_backward.argtypes = [V, V, V, V, V, C.c_int, C.c_int, V, V]
    L.pvof_cnn_mse.argtypes = [V, V, V, C.c_size_t, V, V]
    L.pvof_cnn_status.argtypes = [V]
    L.pvof_cnn_conv32.argtypes = [V, V, V, V, C.c_int, C.c_int, C.c_int, V]
    L.pvof_cnn_adam.argtypes = [V, V, V, V, V, C.c_int, C.c_float, V]
    L.pvof_cnn_to_bf16.argtypes = [V, V, V]
    L.pvof_set_pressure_network.argtypes = [V, P(C.c_float), C.c_size_t]
    L.pvof_pressure_network_sample.argtypes = [V, C.c_int, V, V]
    L.pvof_run_steps_batched.argtypes = [P(V), C.c_int, C.c_int, C.c_double, P(abi.Stats)]
    L.pvof_solver_kernel.restype = C.c_char_p
    _lib = L
    return L


def check(rc, what=""):
    if rc < 0:
        msg = load().pvof_last_error().decode(errors="replace")
        raise PvofError("%s failed (%d): %s" % (what, rc, msg))
    return rc


class Solver:
    """One case on one GPU, driven through the C ABI."""

    def __init__(self, grid, params, device=0):
        L = load()
        self.grid, self.params = grid, params
        self.h = C.c_void_p()
        check(L.pvof_create(C.byref(grid), C.byref(params), device, C.byref(self.h)), "pvof_create")

    def close(self):
        if getattr(self, "h", None):
            load().pvof_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- fields ------------------------------------------------------------
    def block_count(self, name):
        return load().pvof_field_block_count(self.h, abi.FIELD[name])

    def upload(self, name, block):
        a = np.ascontiguousarray(block, dtype=np.float64).ravel()
        check(load().pvof_upload_field(self.h, abi.FIELD[name], a.ctypes.data_as(C.POINTER(C.c_double)), a.size),
              "upload " + name)

    def download(self, name, out=None):
        n = self.block_count(name)
        a = out if out is not None else np.empty(n, dtype=np.float64)
        check(load().pvof_download_field(self.h, abi.FIELD[name], a.ctypes.data_as(C.POINTER(C.c_double)), n),
              "download " + name)
        return a

    def get(self, name):
        """k = 0 plane of a field (ghost frame included for flow fields)."""
        f = abi.FIELD[name]
        return cases.block_plane(self.grid, self.download(name), ng=f in abi.NG_FIELDS)

    def set_fields(self, fields):
        """Upload G-range arrays: (NY, NX) planes copied to every k plane, or
        (NZ, NY, NX) boxes (the 3D mode)."""
        for name, arr in fields.items():
            ng = abi.FIELD[name] in abi.NG_FIELDS
            self.upload(name, cases.field_to_block(self.grid, arr, ng=ng))

    def get_block(self, name):
        """Whole host block of a field: (NZ+2G, NY+2G, NX+2G) for flow
        fields, (NZ, NY, NX) for no-ghost fields."""
        ng = abi.FIELD[name] in abi.NG_FIELDS
        return self.download(name).reshape(cases.block_shape(self.grid, ng))

    def get_g_range(self, name):
        """G-range part (NZ, NY, NX) of a field."""
        b = self.get_block(name)
        if abi.FIELD[name] in abi.NG_FIELDS:
            return b
        NX, NY, NZ = cases.dims(self.grid)
        G = cases.G
        return b[G:G + NZ, G:G + NY, G:G + NX]

    def set_planes(self, planes):
        for name, plane in planes.items():
            ng = abi.FIELD[name] in abi.NG_FIELDS
            self.upload(name, cases.plane_to_block(self.grid, plane, ng=ng))

    # -- routines ----------------------------------------------------------
    def set_stage(self, stage, dt):
        check(load().pvof_set_stage(self.h, stage, dt), "pvof_set_stage")

    def initialize(self):
        check(load().pvof_initialize(self.h), "pvof_initialize")

    def call(self, name, *args):
        fn = getattr(load(), "pvof_" + name)
        return check(fn(self.h, *args), name)

    def substep(self):
        st = abi.Stats()
        check(load().pvof_substep(self.h, C.byref(st)), "pvof_substep")
        return st

    def run_steps(self, n, dt):
        st = abi.Stats()
        check(load().pvof_run_steps(self.h, n, dt, C.byref(st)), "pvof_run_steps")
        return st

    # -- resolved solid particles -----------------------------------------
    def set_particles(self, particles):
        """particles: rows (mobile, x, y, R, u, v, omega_z, rho_s)."""
        arr = (abi.Particle * max(len(particles), 1))()
        for q, (mob, x, y, r, u, v, om, rs) in enumerate(particles):
            p = arr[q]
            p.mobile, p.R, p.Omega_z, p.rho_s = int(mob), float(r), float(om), float(rs)
            p.X[0], p.X[1], p.U[0], p.U[1] = float(x), float(y), float(u), float(v)
        check(load().pvof_set_particles(self.h, arr, len(particles)), "pvof_set_particles")

    def flag_points(self):
        check(load().pvof_Lagrangian_flag_points(self.h), "pvof_Lagrangian_flag_points")
        return check(load().pvof_particle_entries(self.h), "pvof_particle_entries")

    def particle_forces(self):
        n = check(load().pvof_particle_entries(self.h), "pvof_particle_entries")
        F = np.zeros(3 * max(n, 1))
        T = np.zeros(3 * max(n, 1))
        check(load().pvof_particle_forces(self.h, F.ctypes.data_as(C.POINTER(C.c_double)),
                                          T.ctypes.data_as(C.POINTER(C.c_double)), n), "pvof_particle_forces")
        return F[:3 * n].reshape(n, 3), T[:3 * n].reshape(n, 3)

    def get_particles(self, nmax=4096):
        """Owned particles in list order: dict of arrays id, mobile, X (n, 2),
        U (n, 2), Omega (n,), R, F (n, 3), T (n, 3)."""
        arr = (abi.Particle * nmax)()
        ids = (C.c_int * nmax)()
        F = np.zeros(3 * nmax)
        T = np.zeros(3 * nmax)
        dp = C.POINTER(C.c_double)
        n = check(load().pvof_get_particles(self.h, arr, ids, F.ctypes.data_as(dp), T.ctypes.data_as(dp), nmax),
                  "pvof_get_particles")
        return {"id": np.array(ids[:n], dtype=np.int64),
                "mobile": np.array([arr[q].mobile for q in range(n)], dtype=np.int64),
                "X": np.array([[arr[q].X[0], arr[q].X[1]] for q in range(n)]).reshape(n, 2),
                "U": np.array([[arr[q].U[0], arr[q].U[1]] for q in range(n)]).reshape(n, 2),
                "Omega": np.array([arr[q].Omega_z for q in range(n)]),
                "R": np.array([arr[q].R for q in range(n)]),
                "F": F[:3 * n].reshape(n, 3), "T": T[:3 * n].reshape(n, 3)}

    def particle_markers(self, entry, nmax=100000):
        x, y, vol = np.zeros(nmax), np.zeros(nmax), np.zeros(nmax)
        fl = np.zeros(nmax, dtype=np.int32)
        dp = C.POINTER(C.c_double)
        n = check(load().pvof_particle_markers(self.h, entry, x.ctypes.data_as(dp), y.ctypes.data_as(dp),
                                               vol.ctypes.data_as(dp), fl.ctypes.data_as(C.POINTER(C.c_int)), nmax),
                  "pvof_particle_markers")
        return x[:n], y[:n], vol[:n], fl[:n]

    def set_pressure_network(self, params):
        """The learned warm start's parameters (flat float32 array)."""
        a = np.ascontiguousarray(params, dtype=np.float32)
        check(load().pvof_set_pressure_network(self.h, a.ctypes.data_as(C.POINTER(C.c_float)), a.size),
              "pvof_set_pressure_network")

    def liquid_mass(self):
        m = C.c_double()
        check(load().pvof_liquid_mass(self.h, C.byref(m)), "pvof_liquid_mass")
        return m.value

    def synchronize(self):
        check(load().pvof_synchronize(self.h), "pvof_synchronize")

    def launch_count(self):
        return load().pvof_launch_count(self.h)

    # -- measurement ---------------------------------------------------------
    def timer_start(self):
        check(load().pvof_timer_start(self.h), "pvof_timer_start")

    def timer_stop(self):
        ms = C.c_double()
        check(load().pvof_timer_stop(self.h, C.byref(ms)), "pvof_timer_stop")
        return ms.value

    def flush_l2(self):
        check(load().pvof_flush_l2(self.h), "pvof_flush_l2")

    def set_solver_timing(self, on):
        check(load().pvof_set_solver_timing(self.h, 1 if on else 0), "pvof_set_solver_timing")

    def set_autotune(self, on):
        """Start (or stop) the stencil tile autotuner over the next substeps."""
        check(load().pvof_set_autotune(self.h, 1 if on else 0), "pvof_set_autotune")

    def autotune_active(self):
        return bool(load().pvof_autotune_active(self.h))

    def autotune_report(self):
        """[{kernel, tile, best_us, default_us, decided}] of the kernels the tuner met."""
        L = load()
        out = []
        for q in range(L.pvof_autotune_entries(self.h)):
            name, bx, by, best, dflt = C.c_char_p(), C.c_int(), C.c_int(), C.c_double(), C.c_double()
            rc = L.pvof_autotune_entry(self.h, q, C.byref(name), C.byref(bx), C.byref(by), C.byref(best), C.byref(dflt))
            check(min(rc, 0), "pvof_autotune_entry")
            out.append({"kernel": name.value.decode(), "tile": "%dx%d" % (bx.value, by.value),
                        "best_us": 1e3 * best.value, "default_us": 1e3 * dflt.value, "decided": rc == 1})
        return out

    def set_graphs(self, on):
        """Replay each substep's launches from captured CUDA graphs (default on)."""
        check(load().pvof_set_graphs(self.h, 1 if on else 0), "pvof_set_graphs")

    def graph_replays(self):
        return load().pvof_graph_replays(self.h)

    def clamp_mass_total(self):
        """The clamp's liquid mass change summed over the substeps since initialize()."""
        t = C.c_double()
        check(load().pvof_clamp_mass_total(self.h, C.byref(t)), "pvof_clamp_mass_total")
        return t.value

    def set_cluster_solvers(self, on):
        """Cluster-resident solvers where they fit (default), or the grid-wide ones."""
        check(load().pvof_set_cluster_solvers(self.h, 1 if on else 0), "pvof_set_cluster_solvers")

    def set_pressure_pairs(self, mode):
        """Grid-wide pressure solve over pairs of cells: -1 by size (default), 0 never, 1 always."""
        check(load().pvof_set_pressure_pairs(self.h, int(mode)), "pvof_set_pressure_pairs")

    def solver_kernel(self, solver):
        """Name of the kernel that runs solver abi.SOLVER_* in this context."""
        return load().pvof_solver_kernel(self.h, solver).decode()

    def solver_timing(self, solver):
        ms, nl, it, ci = C.c_double(), C.c_longlong(), C.c_longlong(), C.c_longlong()
        check(load().pvof_solver_timing(self.h, solver, C.byref(ms), C.byref(nl), C.byref(it), C.byref(ci)),
              "pvof_solver_timing")
        return {"ms": ms.value, "launches": nl.value, "iterations": it.value, "cell_iters": ci.value}


def run_steps_batched(solvers, nsteps, dt):
    """Advance independent Solver objects concurrently (pvof_run_steps_batched);
    returns their statistics."""
    n = len(solvers)
    handles = (C.c_void_p * max(n, 1))(*[s.h.value for s in solvers])
    stats = (abi.Stats * max(n, 1))()
    check(load().pvof_run_steps_batched(handles, n, nsteps, dt, stats), "pvof_run_steps_batched")
    return [stats[q] for q in range(n)]

