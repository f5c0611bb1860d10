/*
 * Oracle driver around the reference's own time-step code.
 *
 * This program is linked against the reference's C sources, compiled
 * unchanged from their location with the single-rank shims in shim/ and one
 * case header from cfg/ (see Makefile).  It performs the start-up sequence of
 * the reference's main() that the diffuse-interface path needs
 * (PARTIES/src/Cart3d.c:252-520 and the VOF part of
 * Cart3d_initialize_primitive_data, Cart3d.c:1096-1130), but injects the
 * initial fields from raw files instead of the reference's VoF_init_*
 * initialisers, then advances with the reference's own substep routine
 * Temporal_int_all_the_equations (PARTIES/src/Temporal_int.c:563) exactly as
 * Temporal_int_rk3 calls it (Temporal_int.c:399-448) with a constant dt.
 *
 * Usage: ref_driver <case_dir> <nsteps> <dt> <dump_every> [substeps] [warmup]
 *   <case_dir>/parties.inp            INI parameters (reference format)
 *   <case_dir>/init_{C,u,v,w,p}.bin   doubles on the G range of one plane,
 *                                     [j][i] order, i fastest, NX*NY values
 *                                     (NX = NXM+1, NY = NYM+1), replicated
 *                                     over every k plane (2D cases); or on the
 *                                     whole G range, [k][j][i], NX*NY*NZ
 *                                     values (3D cases)
 *   outputs in <case_dir>/out/: s<step>_<field>.bin, each the full ghosted
 *   block of the field (L ranges, [k][j][i], i fastest); "substeps" > 0 also
 *   dumps after every RK substep as s<step>_<rk>_<field>.bin.
 * The timing line "REF_TIMING steps=<n> cells=<c> seconds=<t>" covers the
 * step loop only, after the first <warmup> steps (default 0).
 *
 * Built with -DPVOF_BRIDGE_DRIVER (oracle/ref/Makefile, BRIDGE=substep or
 * BRIDGE=routines) the same program drives the B200 library through the
 * PARTIES-side bridge (parties-vof-ibm_b200/bridge/pvof_bridge.c):
 *   PVOF_BRIDGE_DRIVER == 1: after the reference's start-up, pvof_bridge_start
 *     hands the case to the device, and every substep is pvof_bridge_substep
 *     in place of Velocity_cell_center + Temporal_int_all_the_equations (the
 *     drop-in of the whole substep); the fields are brought back with
 *     pvof_bridge_download before every dump;
 *   PVOF_BRIDGE_DRIVER == 2: the reference's routines that the bridge
 *     defines under their own names (PVOF_BRIDGE_ROUTINES) replace the
 *     reference's CPU definitions (made weak in this build), and the
 *     reference's own start-up and Temporal_int_all_the_equations run
 *     unchanged around them.
 * Test infrastructure only.
 */
#include "DataTypes.h"
#include "definitions.h"
#include "Grid.h"
#include "Communication.h"
#include "Timer.h"
#include "Velocity.h"
#include "Pressure.h"
#include "VolumeFraction.h"
#include "VOF_DIFFUSE.h"
#include "Temporal.h"
#include "Input.h"
#include "Array.h"
#include "Memory.h"
#include "Display.h"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>
#include <sys/stat.h>

#ifdef PVOF_BRIDGE_DRIVER
#include "pvof_bridge.h"
static void bridge_check(int rc, const char *what)
{
    if (rc < 0) {
        fprintf(stderr, "ref_driver: %s: %s\n", what, pvof_last_error());
        exit(3);
    }
}
#endif

static void die(const char *msg)
{
    fprintf(stderr, "ref_driver: %s\n", msg);
    exit(2);
}

static double *read_plane(const char *name, int n)
{
    FILE *f = fopen(name, "rb");
    if (!f) return NULL;
    double *buf = (double *)malloc(sizeof(double) * (size_t)n);
    if (fread(buf, sizeof(double), (size_t)n, f) != (size_t)n) die("short read of an init file");
    fclose(f);
    return buf;
}

/* Copy a [j][i] plane over the G range of every k plane of a flow variable. */
static void inject(double ***a, const double *plane, MAC_grid *g)
{
    int NX = g->NX, NY = g->NY;
    for (int k = g->G_Ks; k < g->G_Ke; k++)
        for (int j = 0; j < NY; j++)
            for (int i = 0; i < NX; i++)
                a[k][j][i] = plane[(size_t)j * NX + i];
}

/* An init file of NX*NY values (one plane, copied to every k plane) or of
 * NX*NY*NZ values ([k][j][i] over the whole G range); returns 0 if absent. */
static int inject_file(double ***a, const char *name, MAC_grid *g)
{
    FILE *f = fopen(name, "rb");
    if (!f) return 0;
    fseek(f, 0, SEEK_END);
    long bytes = ftell(f);
    fclose(f);
    size_t n2 = (size_t)g->NX * (size_t)g->NY, n3 = n2 * (size_t)g->NZ;
    if ((size_t)bytes != n3 * sizeof(double) || n3 == n2) {
        double *plane = read_plane(name, (int)n2);
        inject(a, plane, g);
        free(plane);
        return 1;
    }
    double *buf = read_plane(name, (int)n3);
    for (int k = g->G_Ks; k < g->G_Ke; k++)
        for (int j = 0; j < g->NY; j++)
            for (int i = 0; i < g->NX; i++)
                a[k][j][i] = buf[((size_t)(k - g->G_Ks) * g->NY + j) * g->NX + i];
    free(buf);
    return 1;
}

static void dump(double ***a, MAC_grid *g, const char *path)
{
    size_t n = (size_t)(g->L_Ie - g->L_Is) * (size_t)(g->L_Je - g->L_Js) * (size_t)(g->L_Ke - g->L_Ks);
    FILE *f = fopen(path, "wb");
    if (!f) die("cannot open an output file");
    fwrite(&a[g->L_Ks][g->L_Js][g->L_Is], sizeof(double), n, f);
    fclose(f);
}

/* no-ghost (G range) arrays */
static void dump_ng(double ***a, MAC_grid *g, const char *path)
{
    size_t n = (size_t)(g->G_Ie - g->G_Is) * (size_t)(g->G_Je - g->G_Js) * (size_t)(g->G_Ke - g->G_Ks);
    FILE *f = fopen(path, "wb");
    if (!f) die("cannot open an output file");
    fwrite(&a[g->G_Ks][g->G_Js][g->G_Is], sizeof(double), n, f);
    fclose(f);
}

static void dump_state(Cart3d_bag *db, const char *tag)
{
    MAC_grid *g = db->grid;
    VolumeFraction *vof = db->vof;
    char path[512];
#define DUMP(arr, name) do { snprintf(path, sizeof(path), "out/%s_%s.bin", tag, name); dump(arr, g, path); } while (0)
#define DUMPNG(arr, name) do { snprintf(path, sizeof(path), "out/%s_%s.bin", tag, name); dump_ng(arr, g, path); } while (0)
    DUMP(vof->C_L, "C_L");
    DUMP(vof->C_G, "C_G");
    DUMP(vof->rho, "rho");
    DUMP(vof->mu, "mu");
    DUMP(vof->ch_rhs_n, "ch_rhs_n");
    DUMP(db->u->data, "u");
    DUMP(db->v->data, "v");
    DUMP(db->p->p_data, "p");
    DUMPNG(db->u->ng_explicit_old, "u_explicit_old");
    DUMPNG(db->v->ng_explicit_old, "v_explicit_old");
    DUMPNG(db->u->ng_visc_explicit_old, "u_visc_explicit_old");
    DUMPNG(db->v->ng_visc_explicit_old, "v_visc_explicit_old");
#ifndef TWOD_MODE
    DUMP(db->w->data, "w");
    DUMPNG(db->w->ng_explicit_old, "w_explicit_old");
    DUMPNG(db->w->ng_visc_explicit_old, "w_visc_explicit_old");
#endif
#ifdef SURFACE_TENSION
    DUMP(vof->psi_LG, "psi_LG");
    DUMPNG(vof->f_sigma_old_x, "f_sigma_old_x");
    DUMPNG(vof->f_sigma_old_y, "f_sigma_old_y");
#ifndef TWOD_MODE
    DUMPNG(vof->f_sigma_old_z, "f_sigma_old_z");
#endif
#endif
#undef DUMP
#undef DUMPNG
}

int main(int argc, char **argv)
{
    if (argc < 5) die("usage: ref_driver <case_dir> <nsteps> <dt> <dump_every> [substeps]");
    const char *case_dir = argv[1];
    int nsteps = atoi(argv[2]);
    double dt = atof(argv[3]);
    int dump_every = atoi(argv[4]);
    int dump_substeps = (argc > 5) ? atoi(argv[5]) : 0;
    int warm = (argc > 6) ? atoi(argv[6]) : 0;   /* leading steps left out of REF_TIMING */
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
    db->lag = NULL;

    if (!inject_file(db->vof->F, "init_C.bin", grid)) die("missing init_C.bin");
    inject_file(db->u->data, "init_u.bin", grid);
    inject_file(db->v->data, "init_v.bin", grid);
    inject_file(db->w->data, "init_w.bin", grid);
    inject_file(db->p->p_data, "init_p.bin", grid);
#if defined(PVOF_BRIDGE_DRIVER) && PVOF_BRIDGE_DRIVER == 2
    /* the bridged routines below work on the device copy from here on */
    params->dt = dt;
    bridge_check(pvof_bridge_start(db, 0), "pvof_bridge_start");
#endif

    Velocity_update_boundaries(db->u->data, 'u', VEL_TYPE_NORMAL, db);
    Velocity_update_boundaries(db->v->data, 'v', VEL_TYPE_NORMAL, db);
    Velocity_update_boundaries(db->w->data, 'w', VEL_TYPE_NORMAL, db);
    Pressure_apply_BCs(db->p->p_data, grid, params);
    Communication_update_ghost_nodes_flow_variable(db->p->p_data, CONCENTRATION_PERTURBATION, 3, db);

    /* VOF part of Cart3d_initialize_primitive_data (Cart3d.c:1096-1130) */
    params->which_stage = 0;
    params->dt = dt;
    VOF_DIFFUSE_set_boundary_values(db->vof->F, db);
    VOF_DIFFUSE_init(db);
    VOF_update_density_viscosity(db);
#ifdef SURFACE_TENSION
    VOF_DIFFUSE_compute_psi_LG(db);
    VOF_DIFFUSE_compute_f_sigma(db);
    Array_copy_noghost(db->vof->f_sigma_new_x, db->vof->f_sigma_old_x, grid, params);
    Array_copy_noghost(db->vof->f_sigma_new_y, db->vof->f_sigma_old_y, grid, params);
    Array_copy_noghost(db->vof->f_sigma_new_z, db->vof->f_sigma_old_z, grid, params);
#endif
    /* cell-centred velocity for the first substep (Temporal_int.c:420-424) */
    Velocity_cell_center(db);
#if defined(PVOF_BRIDGE_DRIVER) && PVOF_BRIDGE_DRIVER == 1
    bridge_check(pvof_bridge_start(db, 0), "pvof_bridge_start");
    bridge_check(pvof_bridge_download(db), "pvof_bridge_download");
#endif

    dump_state(db, "s0");

    const double BET2[] = {BETA2};
    double time = 0.0;
    params->time = 0.0;
    double t0 = MPI_Wtime();
    double t_io = 0.0;
    for (int n = 1; n <= nsteps; n++) {
        if (n == warm + 1) {
            t0 = MPI_Wtime();
            t_io = 0.0;
        }
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
            if (dump_substeps > 0 && dump_every > 0 && n % dump_every == 0) {
                double a = MPI_Wtime();
#if defined(PVOF_BRIDGE_DRIVER) && PVOF_BRIDGE_DRIVER == 1
                bridge_check(pvof_bridge_download(db), "pvof_bridge_download");
#endif
                char tag[64];
                snprintf(tag, sizeof(tag), "s%d_%d", n, rk);
                dump_state(db, tag);
                t_io += MPI_Wtime() - a;
            }
        }
        params->ntime = n;
        if (dump_every > 0 && n % dump_every == 0) {
            double a = MPI_Wtime();
#if defined(PVOF_BRIDGE_DRIVER) && PVOF_BRIDGE_DRIVER == 1
            bridge_check(pvof_bridge_download(db), "pvof_bridge_download");
#endif
            char tag[64];
            snprintf(tag, sizeof(tag), "s%d", n);
            dump_state(db, tag);
            t_io += MPI_Wtime() - a;
        }
    }
    double secs = MPI_Wtime() - t0 - t_io;
    printf("REF_TIMING steps=%d cells=%ld seconds=%.6f\n", nsteps - (warm < nsteps ? warm : 0),
           (long)params->NXM * (long)params->NYM * (long)params->NZM, secs);
    return 0;
}
