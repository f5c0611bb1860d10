"""ctypes mirror of include/pvof.h (structures, constants, field ids).

The structures and enumerations here must match include/pvof.h field for
field; tests/test_abi.py checks the exported symbols and the sizes.
"""
import ctypes as C

ABI_VERSION = 4

OK = 0
EINVAL = -1
ECUDA = -2
ENOMEM = -3
ENODEV = -4
EDIVERGED = -5

GEOM_3D = 0
GEOM_PLANAR = 1
GEOM_AXISYM = 2

WALL_NOSLIP = 0
WALL_FREESLIP = 1

LEFT, RIGHT, BOTTOM, TOP, BACK, FRONT = range(6)

FIELD_NAMES = [
    "C_L", "C_G", "C_S", "F",
    "RHO", "MU", "PSI_LG", "LAP_C",
    "CH_RHS_N", "CH_RHS_CUR",
    "U", "V", "W", "U_BC", "V_BC",
    "P", "DELTAP", "P_RHS",
    "U_EXPLICIT", "U_EXPLICIT_OLD", "U_IMPLICIT",
    "U_VISC_EXPLICIT", "U_VISC_EXPLICIT_OLD", "U_RHS",
    "V_EXPLICIT", "V_EXPLICIT_OLD", "V_IMPLICIT",
    "V_VISC_EXPLICIT", "V_VISC_EXPLICIT_OLD", "V_RHS",
    "FSIG_OLD_X", "FSIG_OLD_Y", "FSIG_NEW_X", "FSIG_NEW_Y",
    "NX_IBM", "NY_IBM",
    "W_EXPLICIT", "W_EXPLICIT_OLD", "W_IMPLICIT",
    "W_VISC_EXPLICIT", "W_VISC_EXPLICIT_OLD", "W_RHS",
    "FSIG_OLD_Z", "FSIG_NEW_Z",
]
FIELD = {name: idx for idx, name in enumerate(FIELD_NAMES)}
FIELD_COUNT = len(FIELD_NAMES)
# no-ghost ("ng_") fields: G-range blocks
NG_FIELDS = set(range(FIELD["U_EXPLICIT"], FIELD["FSIG_NEW_Y"] + 1)) | set(range(FIELD["W_EXPLICIT"], FIELD["FSIG_NEW_Z"] + 1))


class GridDesc(C.Structure):
    _fields_ = [
        ("NXM", C.c_int), ("NYM", C.c_int), ("NZM", C.c_int),
        ("ghost_nodes", C.c_int),
        ("geometry", C.c_int),
        ("periodic", C.c_int * 3),
        ("wall", C.c_int * 6),
        ("xmin", C.c_double), ("xmax", C.c_double),
        ("ymin", C.c_double), ("ymax", C.c_double),
        ("zmin", C.c_double), ("zmax", C.c_double),
        ("slab_thickness", C.c_double),
        ("theta_span", C.c_double),
    ]


class Params(C.Structure):
    _fields_ = [
        ("Re", C.c_double), ("We", C.c_double),
        ("rho1", C.c_double), ("rho2", C.c_double),
        ("mu1", C.c_double), ("mu2", C.c_double),
        ("Cn", C.c_double), ("Pe_CH", C.c_double),
        ("grav", C.c_double * 3),
        ("richardson", C.c_double),
        ("dp_dx", C.c_double),
        ("weno_order", C.c_int),
        ("ch_iter_max", C.c_int),
        ("ch_tol", C.c_double),
        ("CG_MAXIT", C.c_int),
        ("CG_ETOL", C.c_double),
        ("P_CG_MAXIT", C.c_int),
        ("P_CG_ETOL", C.c_double),
        ("surface_tension", C.c_int),
        ("gravity", C.c_int),
        ("contact_angle_deg", C.c_double),
        ("N_forcing_loops", C.c_int),
        ("stencil_fp32", C.c_int),
        ("pressure_warm_start", C.c_int),
        ("pressure_preconditioner", C.c_int),
        ("velocity_cg_unregularized", C.c_int),
    ]


class Stats(C.Structure):
    _fields_ = [
        ("ch_iters", C.c_int), ("ch_rel_res", C.c_double),
        ("u_iters", C.c_int), ("v_iters", C.c_int),
        ("u_rms", C.c_double), ("v_rms", C.c_double),
        ("p_iters", C.c_int), ("p_iters_total", C.c_int),
        ("p_res", C.c_double),
        ("poisson_passes", C.c_int),
        ("div_max", C.c_double),
        ("clamp_mass", C.c_double),
        ("w_iters", C.c_int), ("w_rms", C.c_double),
    ]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


class Particle(C.Structure):
    """pvof_particle: one resolved solid particle of the planar mode."""
    _fields_ = [
        ("mobile", C.c_int), ("X", C.c_double * 2), ("R", C.c_double),
        ("U", C.c_double * 2), ("Omega_z", C.c_double), ("rho_s", C.c_double),
    ]


# exported symbols of the C ABI (include/pvof.h), checked by the tests
EXPORTS = [
    "pvof_abi_version", "pvof_last_error", "pvof_device_count",
    "pvof_create", "pvof_destroy",
    "pvof_upload_field", "pvof_download_field", "pvof_field_block_count",
    "pvof_synchronize", "pvof_set_stage",
    "pvof_VOF_DIFFUSE_init", "pvof_VOF_DIFFUSE_step", "pvof_VOF_DIFFUSE_advect_WENO5",
    "pvof_VOF_update_density_viscosity", "pvof_VOF_DIFFUSE_compute_psi_LG",
    "pvof_VOF_DIFFUSE_compute_f_sigma", "pvof_VOF_apply_f_sigma_old", "pvof_VOF_swap_f_sigma",
    "pvof_Velocity_add_gravity_2_RHS", "pvof_Velocity_cell_center",
    "pvof_Velocity_set_implicit_explicit", "pvof_Velocity_set_RHS",
    "pvof_Velocity_solve_cg", "pvof_Velocity_update_boundaries",
    "pvof_Pressure_set_RHS", "pvof_Pressure_compute_preconditioner",
    "pvof_Pressure_solve_cg", "pvof_Pressure_project_velocity",
    "pvof_Pressure_compute_velocity_divergence",
    "pvof_substep", "pvof_run_steps", "pvof_liquid_mass",
    "pvof_initialize",
    "pvof_launch_count", "pvof_timer_start", "pvof_timer_stop", "pvof_flush_l2",
    "pvof_set_solver_timing", "pvof_solver_timing", "pvof_set_autotune", "pvof_autotune_active",
    "pvof_autotune_entries", "pvof_autotune_entry", "pvof_solver_kernel", "pvof_set_graphs", "pvof_graph_replays", "pvof_spectral_tables",
    "pvof_set_cluster_solvers", "pvof_set_pressure_pairs", "pvof_clamp_mass_total",
    "pvof_Pressure_solve_cg_noalloc", "pvof_noalloc_last_error",
    "pvof_set_particles", "pvof_Lagrangian_flag_points", "pvof_particle_entries", "pvof_particle_forces",
    "pvof_particle_markers", "pvof_VOF_DIFFUSE_compute_C_S", "pvof_Velocity_solve_explicit",
    "pvof_Lagrangian_force", "pvof_Pressure_solve_fft", "pvof_run_steps_batched",
    "pvof_VOF_DIFFUSE_compute_solid_normals_MCL", "pvof_VOF_DIFFUSE_apply_contact_angle",
    "pvof_VOF_DIFFUSE_extend_psi_LG_contact_angle",
    "pvof_Particle_initialize_velocities", "pvof_Lagrangian_advect_particles", "pvof_get_particles",
    "pvof_cnn_param_count", "pvof_cnn_work_floats", "pvof_cnn_forward", "pvof_cnn_backward", "pvof_cnn_mse",
    "pvof_cnn_adam", "pvof_cnn_to_bf16", "pvof_cnn_status", "pvof_cnn_conv32", "pvof_set_pressure_network", "pvof_pressure_network_sample",
]

SOLVER_BIHARMONIC = 0
SOLVER_VELOCITY = 1
SOLVER_PRESSURE = 2
