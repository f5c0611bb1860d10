/*
 * Oracle driver for the immersed-boundary routines of the reference, built
 * from the reference's own sources with the resolved-particle flags
 * (cfg/ibm2d.h: VOF_IBM, LAG_PARTICLE_RESOLVED).  It reuses the start-up of
 * ref_driver.c, reads the particle lists through the reference's
 * Particle_initialize (with the file reader below), and then calls, one by
 * one and in the order of Temporal_int_all_the_equations
 * (PARTIES/src/Temporal_int.c:948-1016), the routines of the IBM part of a
 * substep, dumping their inputs and outputs:
 *
 *   i0   after start-up: C_S (VOF_DIFFUSE_compute_C_S inside VOF_DIFFUSE_init),
 *        C_L, C_G, rho, mu, u, v
 *   markers.bin  Particle_MPI_update of both lists and Lagrangian_flag_points,
 *        as at the start of a substep: per particle (mobile list, then
 *        fixed list) N_L_local, X_L, Y_L, Vol_L_marker, flag_L as doubles
 *   r0   momentum RHS before the IBM (set_implicit_explicit, set_RHS, gravity)
 *   r1   Velocity_solve_explicit of u and v (+ boundary update)
 *   r2   Lagrangian_force(-1): RHS, particle F and T (particles_r2.txt)
 *   r3   Velocity_solve (Jacobi-PCG) of u and v (+ boundary update)
 *   r4   Lagrangian_force(N_forcing_loops) (+ boundary update): u, v, RHS,
 *        particle F and T (particles_r4.txt)
 *
 * Mode "mcl" instead dumps the contact-line routines of VOF_IBM_wetting.c
 * (Liu & Ding characteristic projection):
 *
 *   m1   C_L, C_G, C_S before VOF_DIFFUSE_apply_contact_angle: the state
 *        VOF_DIFFUSE_init has just before its own call of it (clamp of F,
 *        bound to 1 - C_S, boundary values, phase cache)
 *   m2   C_L right after VOF_DIFFUSE_apply_contact_angle (no boundary update)
 *        and the solid normals nx_IBM, ny_IBM it computed
 *   m3   psi_LG from VOF_DIFFUSE_compute_psi_LG after the boundary update and
 *        phase cache of m2, and the C_L, C_G it was computed from
 *   m4   psi_LG after VOF_DIFFUSE_extend_psi_LG_contact_angle
 *
 * Mode "steps" sets the particle velocities from the fluid
 * (Particle_initialize_velocities, as the reference's main does after the
 * primitive data), then runs <nsteps> whole time steps through the
 * reference's own substep routine Temporal_int_all_the_equations, as
 * ref_driver.c does, and dumps the state (dump_state of ref_driver.c) after
 * every step, plus per particle F, T, ID, X, U and Omega_z
 * (particles_s<n>.txt).
 *
 * The initial volume fraction goes into both F and C_L, as the reference's
 * initialisers do (IO/VoF_Init.c), before Particle_initialize and
 * VOF_DIFFUSE_init.
 *
 * Usage: ibm_driver <case_dir> <dt> <stage> [routines|mcl|steps] [nsteps]
 *   files of ref_driver.c, plus particles_fixed.txt and particles_mobile.txt:
 *   one particle per line, "X Y R U V Omega_z".
 * Test infrastructure only.
 */
#define main ref_driver_main
#include "ref_driver.c"
#undef main

#include "Lagrangian.h"
#include "Particle.h"
#include "ParticleInput.h"

/*
 * Particle file reader in place of the reference's ParticleInput_inp
 * (PARTIES/src/IO/ParticleInput.c:24-334, whose translation unit needs HDF5):
 * the same per-particle set-up -- in-plane position with z on the storage
 * plane, identity rotation, Particle_initialize_nonessential_data,
 * Particle_calc_derived_data, Particle_create_internal_arrays -- except that
 * the velocities come from the file instead of zero.
 */
void ParticleInput_inp(Particle_list *p_list, MAC_grid *grid, Parameters *params, Debug_trace *dtrace)
{
    (void)dtrace;
    const char *name = (p_list->type == FIXED) ? "particles_fixed.txt" : "particles_mobile.txt";
    p_list->start = NULL;
    p_list->Np = 0;
    p_list->state = LIST_STATE_LOCAL;
    FILE *f = fopen(name, "r");
    if (!f) return;
    Particle *last = NULL;
    double x, y, r, u, v, om;
    int n = 0;
    while (fscanf(f, "%lf %lf %lf %lf %lf %lf", &x, &y, &r, &u, &v, &om) == 6) {
        Particle *p = (Particle *)calloc(1, sizeof(Particle));
        p->X[0] = x;
        p->X[1] = y;
        p->X[2] = grid->zc[grid->G_Ks];
        p->R = r;
        p->ID = n + p_list->ID_start;
        p->U[0] = u;
        p->U[1] = v;
        p->Omega[2] = om;
        p->Rotn[0][0] = p->Rotn[1][1] = p->Rotn[2][2] = 1.0;
        p->particle_collision = NULL;
        p->wall_collision = NULL;
        Particle_initialize_nonessential_data(p);
        Particle_calc_derived_data(p, grid, params);
        Particle_create_internal_arrays(p);
        p->next = NULL;
        if (last) last->next = p;
        else p_list->start = p;
        last = p;
        n++;
    }
    fclose(f);
    p_list->Np = n;
}

static void dump_markers(Cart3d_bag *db)
{
    FILE *f = fopen("out/markers.bin", "wb");
    if (!f) die("cannot open markers.bin");
    Particle_list *lists[2] = {db->lag->p_mobile_list, db->lag->p_fixed_list};
    for (int l = 0; l < 2; l++) {
        for (Particle *p = lists[l]->start; p; p = p->next) {
            double n = (double)p->N_L_local;
            fwrite(&n, sizeof(double), 1, f);
            fwrite(p->X_L, sizeof(double), (size_t)p->N_L_local, f);
            fwrite(p->Y_L, sizeof(double), (size_t)p->N_L_local, f);
            fwrite(p->Vol_L_marker, sizeof(double), (size_t)p->N_L_local, f);
            for (int m = 0; m < p->N_L_local; m++) {
                double fl = (double)p->flag_L[m];
                fwrite(&fl, sizeof(double), 1, f);
            }
        }
    }
    fclose(f);
}

static void dump_particles(Cart3d_bag *db, const char *tag)
{
    char path[256];
    snprintf(path, sizeof(path), "out/particles_%s.txt", tag);
    FILE *f = fopen(path, "w");
    if (!f) die("cannot open a particle output file");
    Particle_list *lists[2] = {db->lag->p_mobile_list, db->lag->p_fixed_list};
    for (int l = 0; l < 2; l++)
        for (Particle *p = lists[l]->start; p; p = p->next)
            fprintf(f, "%.17g %.17g %.17g %.17g %.17g %.17g %d %.17g %.17g %.17g %.17g %.17g\n", p->F[0], p->F[1],
                    p->F[2], p->T[0], p->T[1], p->T[2], p->ID, p->X[0], p->X[1], p->U[0], p->U[1], p->Omega[2]);
    fclose(f);
}

static void dump_fields(Cart3d_bag *db, const char *tag, int rhs)
{
    MAC_grid *g = db->grid;
    char path[512];
#define D(arr, name) do { snprintf(path, sizeof(path), "out/%s_%s.bin", tag, name); dump(arr, g, path); } while (0)
#define DN(arr, name) do { snprintf(path, sizeof(path), "out/%s_%s.bin", tag, name); dump_ng(arr, g, path); } while (0)
    D(db->u->data, "u");
    D(db->v->data, "v");
    if (rhs) {
        DN(db->u->ng_rhs, "u_rhs");
        DN(db->v->ng_rhs, "v_rhs");
        DN(db->u->ng_implicit, "u_implicit");
        DN(db->v->ng_implicit, "v_implicit");
    }
#undef D
#undef DN
}

static void dump_tag(double ***a, MAC_grid *g, const char *tag, const char *name)
{
    char path[512];
    snprintf(path, sizeof(path), "out/%s_%s.bin", tag, name);
    dump(a, g, path);
}

/* the contact-line routines on the state VOF_DIFFUSE_init hands to its own
 * VOF_DIFFUSE_apply_contact_angle call (VOF_DIFFUSE.c:523-568) */
static void run_mcl(Cart3d_bag *db, const double *F0)
{
    MAC_grid *g = db->grid;
    VolumeFraction *vof = db->vof;
    inject(vof->F, F0, g);
    VOF_DIFFUSE_set_boundary_values(vof->F, db);
    for (int k = g->L_Ks; k < g->L_Ke; ++k)
        for (int j = g->L_Js; j < g->L_Je; ++j)
            for (int i = g->L_Is; i < g->L_Ie; ++i) {
                double f = vof->F[k][j][i];
                vof->C_L[k][j][i] = f < 0.0 ? 0.0 : (f > 1.0 ? 1.0 : f);
            }
    VOF_DIFFUSE_set_boundary_values(vof->C_L, db);
    VOF_DIFFUSE_update_phase_cache(db);
    /* diffuse_bound_liquid_fraction (VOF_DIFFUSE.c:1093-1127, static there) */
    for (int k = g->G_Ks; k < g->G_Ke; ++k)
        for (int j = g->G_Js; j < g->G_Je; ++j)
            for (int i = g->G_Is; i < g->G_Ie; ++i) {
                double cs = vof->C_S[k][j][i], cl = vof->C_L[k][j][i];
                double mx = 1.0 - cs;
                if (mx < 0.0) mx = 0.0;
                if (mx > 1.0) mx = 1.0;
                if (cl < 0.0) cl = 0.0;
                if (cl > mx) cl = mx;
                vof->C_L[k][j][i] = cl;
                double cg = 1.0 - cl - cs;
                vof->C_G[k][j][i] = cg < 0.0 ? 0.0 : (cg > 1.0 ? 1.0 : cg);
            }
    VOF_DIFFUSE_set_boundary_values(vof->C_L, db);
    VOF_DIFFUSE_update_phase_cache(db);
    dump_tag(vof->C_L, g, "m1", "C_L");
    dump_tag(vof->C_G, g, "m1", "C_G");
    dump_tag(vof->C_S, g, "m1", "C_S");
    VOF_DIFFUSE_apply_contact_angle(db);
    dump_tag(vof->C_L, g, "m2", "C_L");
    dump_tag(vof->nx_IBM, g, "m2", "nx");
    dump_tag(vof->ny_IBM, g, "m2", "ny");
    VOF_DIFFUSE_set_boundary_values(vof->C_L, db);
    VOF_DIFFUSE_update_phase_cache(db);
    VOF_DIFFUSE_compute_psi_LG(db);
    dump_tag(vof->psi_LG, g, "m3", "psi_LG");
    dump_tag(vof->C_L, g, "m3", "C_L");
    dump_tag(vof->C_G, g, "m3", "C_G");
    VOF_DIFFUSE_extend_psi_LG_contact_angle(db);
    dump_tag(vof->psi_LG, g, "m4", "psi_LG");
}

/* whole time steps as ref_driver.c takes them (Temporal_int.c:399-448) */
static void run_steps(Cart3d_bag *db, int nsteps, double dt, Debug_trace *dtrace)
{
    Parameters *params = db->params;
    const double BET2[] = {BETA2};
    double time = 0.0;
    params->time = 0.0;
#if defined(PVOF_BRIDGE_DRIVER) && PVOF_BRIDGE_DRIVER == 1
    /* the device takes the case from here: its start-up sets the particle
     * velocities and paints them (Particle_initialize_velocities) itself */
    (void)dtrace;
    bridge_check(pvof_bridge_start(db, 0), "pvof_bridge_start");
    bridge_check(pvof_bridge_download(db), "pvof_bridge_download");
#else
    /* Cart3d.c:505-515, then the cell-centred velocity of Temporal_int.c:194 */
    Particle_initialize_velocities(db, DTRACE("Particle_initialize_velocities"));
    Velocity_cell_center(db);
#endif
    dump_state(db, "s0");
    dump_particles(db, "s0");
    double t0 = MPI_Wtime(), t_io = 0.0;
    for (int n = 1; n <= nsteps; n++) {
        for (int rk = 0; rk < 3; rk++) {
            params->which_stage = rk;
            params->dt = dt;
#if defined(PVOF_BRIDGE_DRIVER) && PVOF_BRIDGE_DRIVER == 1
            bridge_check(pvof_bridge_substep(db), "pvof_bridge_substep");
#else
            if (time != 0 && rk == 0)
                Velocity_cell_center(db);
            Temporal_int_all_the_equations(db, DTRACE("Temporal_int_all_the_equations"));
#endif
            time += dt * BET2[rk];
            params->time = time;
        }
        params->ntime = n;
        double a = MPI_Wtime();
#if defined(PVOF_BRIDGE_DRIVER) && PVOF_BRIDGE_DRIVER == 1
        bridge_check(pvof_bridge_download(db), "pvof_bridge_download");
#endif
        char tag[64];
        snprintf(tag, sizeof(tag), "s%d", n);
        dump_state(db, tag);
        dump_particles(db, tag);
        t_io += MPI_Wtime() - a;
    }
    /* the step loop without the dumps, as ref_driver.c reports it */
    printf("REF_TIMING steps=%d cells=%ld seconds=%.6f\n", nsteps,
           (long)params->NXM * (long)params->NYM * (long)params->NZM, MPI_Wtime() - t0 - t_io);
}

int main(int argc, char **argv)
{
    if (argc < 4) die("usage: ibm_driver <case_dir> <dt> <stage> [routines|mcl|steps] [nsteps]");
    const char *case_dir = argv[1];
    double dt = atof(argv[2]);
    int stage = atoi(argv[3]);
    const char *mode = (argc > 4) ? argv[4] : "routines";
    int nsteps = (argc > 5) ? atoi(argv[5]) : 1;
    if (chdir(case_dir) != 0) die("cannot enter the case directory");
    mkdir("out", 0755);

    MPI_Init(&argc, &argv);
    Debug_trace dtrace_parent = {"", "", 0, NULL, NULL};
    Debug_trace *dtrace = &dtrace_parent;

    Cart3d_bag *db = (Cart3d_bag *)calloc(1, sizeof(Cart3d_bag));
    Parameters *params = (Parameters *)calloc(1, sizeof(Parameters));
    params->size = 1;
    params->rank = 0;
    Input_set_parameters(params, PARTIES_INPUT_FILE);
    db->params = params;

    MAC_grid *grid = Grid_create(params, DTRACE("Grid_create"));
    db->grid = grid;
    Communication_new_xyz_communicator(grid, params);
    db->timer = Timer_create(grid, params);
    db->u = Velocity_create(grid, params, 'u', DTRACE("Velocity_create"));
    db->v = Velocity_create(grid, params, 'v', DTRACE("Velocity_create"));
    db->w = Velocity_create(grid, params, 'w', DTRACE("Velocity_create"));
    db->p = Pressure_create(grid, params);
    db->vof = VoF_create(grid, params);
    db->lag = Lagrangian_create(grid, params);

    int NX = grid->NX, NY = grid->NY;
    double *plane;
    double *F0;
    if (!(F0 = read_plane("init_C.bin", NX * NY))) die("missing init_C.bin");
    inject(db->vof->F, F0, grid);
    inject(db->vof->C_L, F0, grid);
    if ((plane = read_plane("init_u.bin", NX * NY))) { inject(db->u->data, plane, grid); free(plane); }
    if ((plane = read_plane("init_v.bin", NX * NY))) { inject(db->v->data, plane, grid); free(plane); }
    if ((plane = read_plane("init_p.bin", NX * NY))) { inject(db->p->p_data, plane, grid); free(plane); }

    Velocity_update_boundaries(db->u->data, 'u', VEL_TYPE_NORMAL, db);
    Velocity_update_boundaries(db->v->data, 'v', VEL_TYPE_NORMAL, db);
    Velocity_update_boundaries(db->w->data, 'w', VEL_TYPE_NORMAL, db);
    Pressure_apply_BCs(db->p->p_data, grid, params);
    Communication_update_ghost_nodes_flow_variable(db->p->p_data, CONCENTRATION_PERTURBATION, 3, db);

    /* particles before VOF_DIFFUSE_init, as Cart3d.c:488-496 does */
    params->which_stage = 0;
    params->dt = dt;
    Particle_initialize(db, DTRACE("Particle_initialize"));
    VOF_DIFFUSE_set_boundary_values(db->vof->F, db);
    VOF_DIFFUSE_init(db);
    VOF_update_density_viscosity(db);
#ifdef SURFACE_TENSION
    /* Cart3d.c:1110-1125 */
    VOF_DIFFUSE_compute_psi_LG(db);
    VOF_DIFFUSE_extend_psi_LG_contact_angle(db);
    VOF_DIFFUSE_compute_f_sigma(db);
    Array_copy_noghost(db->vof->f_sigma_new_x, db->vof->f_sigma_old_x, grid, params);
    Array_copy_noghost(db->vof->f_sigma_new_y, db->vof->f_sigma_old_y, grid, params);
    Array_copy_noghost(db->vof->f_sigma_new_z, db->vof->f_sigma_old_z, grid, params);
#endif
    Velocity_cell_center(db);

    {
        char path[512];
#define D(arr, name) do { snprintf(path, sizeof(path), "out/i0_%s.bin", name); dump(arr, grid, path); } while (0)
        D(db->vof->C_S, "C_S");
        D(db->vof->C_L, "C_L");
        D(db->vof->C_G, "C_G");
        D(db->vof->rho, "rho");
        D(db->vof->mu, "mu");
        D(db->u->data, "u");
        D(db->v->data, "v");
#undef D
    }

    if (!strcmp(mode, "mcl")) {
        run_mcl(db, F0);
        printf("IBM_DONE mcl\n");
        return 0;
    }
    if (!strcmp(mode, "steps")) {
        run_steps(db, nsteps, dt, dtrace);
        printf("IBM_DONE steps=%d\n", nsteps);
        return 0;
    }
    if (strcmp(mode, "routines")) die("unknown mode");

    params->which_stage = stage;
    params->dt = dt;
    /* the list updates and marker flags at the start of a substep (Temporal_int.c:678-681) */
    Particle_MPI_update(db->lag->p_mobile_list, db, DTRACE("Particle_MPI_update"));
    Particle_MPI_update(db->lag->p_fixed_list, db, DTRACE("Particle_MPI_update"));
    Lagrangian_flag_points(db, DTRACE("Lagrangian_flag_points"));
    dump_markers(db);

    Velocity_u_set_implicit_explicit(db);
    Velocity_v_set_implicit_explicit(db);
    Velocity_u_set_RHS(db);
    Velocity_v_set_RHS(db);
    Velocity_w_set_RHS(db);
#ifdef VOF_GRAVITY
    Velocity_add_gravity_2_RHS(db);
#endif
    dump_fields(db, "r0", 1);

    Velocity_solve_explicit(db->u, db);
    Velocity_solve_explicit(db->v, db);
    Velocity_solve_explicit(db->w, db);
    Velocity_update_boundaries(db->u->data, 'u', VEL_TYPE_NORMAL, db);
    Velocity_update_boundaries(db->v->data, 'v', VEL_TYPE_NORMAL, db);
    Velocity_update_boundaries(db->w->data, 'w', VEL_TYPE_NORMAL, db);
    dump_fields(db, "r1", 0);

    Lagrangian_force(-1, db, DTRACE("Lagrangian_force"));
    dump_fields(db, "r2", 1);
    dump_particles(db, "r2");

    Velocity_solve(db->u, db);
    Velocity_solve(db->v, db);
    Velocity_solve(db->w, db);
    Velocity_update_boundaries(db->u->data, 'u', VEL_TYPE_NORMAL, db);
    Velocity_update_boundaries(db->v->data, 'v', VEL_TYPE_NORMAL, db);
    Velocity_update_boundaries(db->w->data, 'w', VEL_TYPE_NORMAL, db);
    dump_fields(db, "r3", 0);

    Lagrangian_force(params->N_forcing_loops, db, DTRACE("Lagrangian_force"));
    Velocity_update_boundaries(db->u->data, 'u', VEL_TYPE_NORMAL, db);
    Velocity_update_boundaries(db->v->data, 'v', VEL_TYPE_NORMAL, db);
    Velocity_update_boundaries(db->w->data, 'w', VEL_TYPE_NORMAL, db);
    dump_fields(db, "r4", 1);
    dump_particles(db, "r4");
    printf("IBM_DONE N_forcing_loops=%d\n", params->N_forcing_loops);
    return 0;
}
