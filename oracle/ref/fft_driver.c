/*
 * Oracle driver for the reference's constant-density FFT Poisson solver
 * (PARTIES/src/Eulerian/lsolver/psolve_fft.c): builds the grid and pressure
 * objects as ref_driver.c does, sets the solver up with the reference's
 * Pressure_setup_lsys_accounting_geometry (FFT plans through the
 * single-rank FFTW shim in shim/, transposes, tridiagonal coefficients), puts
 * the right-hand side from <case_dir>/rhs.bin ([j][i] plane over the G
 * range, replicated over k) into p->rhs and calls Pressure_solve_xz_period.
 * Output: out/fft_deltap.bin (the ghosted block of p->deltap).
 *
 * Usage: fft_driver <case_dir>
 * Test infrastructure only.
 */
#define main ref_driver_main
#include "ref_driver.c"
#undef main

int Pressure_solve_xz_period(Pressure *p, MAC_grid *grid, Parameters *params);
void Pressure_setup_lsys_accounting_geometry(Pressure *p, MAC_grid *grid, Parameters *params);

int main(int argc, char **argv)
{
    if (argc < 2) die("usage: fft_driver <case_dir>");
    if (chdir(argv[1]) != 0) die("cannot enter the case directory");
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
    db->p = Pressure_create(grid, params);
    Pressure_setup_lsys_accounting_geometry(db->p, grid, params);
    double *plane = read_plane("rhs.bin", grid->NX * grid->NY);
    if (!plane) die("missing rhs.bin");
    inject(db->p->rhs, plane, grid);
    free(plane);
    Pressure_solve_xz_period(db->p, grid, params);
    dump(db->p->deltap, grid, "out/fft_deltap.bin");
    printf("FFT_DONE\n");
    return 0;
}
