/*
 * CPU restatement (oracle) of PARTIES' diffuse-interface RK3 substep.
 *
 * TEST INFRASTRUCTURE ONLY: the parity tests, the smoke check and the CPU
 * baseline leg of bench.py use this library as the checker.  The product
 * path (the CUDA library behind include/pvof.h) never links or calls it.
 *
 * The oracle keeps one k plane of every field (the 2D modes of the
 * reference keep all planes identical) with the reference's ghosted index
 * space, and restates each reference routine loop by loop on the same index
 * ranges, in the same floating-point operation order.  It is pinned against
 * the reference compiled from its own sources (oracle/ref, golden fixtures in
 * tests/golden).
 */
#ifndef PVOF_ORACLE_H
#define PVOF_ORACLE_H

#include "../include/pvof.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc orc_t;

/* routine identifiers for orc_routine() */
enum orc_routine_id {
    ORC_VOF_DIFFUSE_INIT = 0,
    ORC_VOF_DIFFUSE_STEP,
    ORC_ADVECT_WENO5,
    ORC_UPDATE_DENSITY_VISCOSITY,
    ORC_COMPUTE_PSI_LG,
    ORC_COMPUTE_F_SIGMA,
    ORC_APPLY_F_SIGMA_OLD,
    ORC_SWAP_F_SIGMA,
    ORC_ADD_GRAVITY,
    ORC_CELL_CENTER,
    ORC_U_IMPLICIT_EXPLICIT,
    ORC_V_IMPLICIT_EXPLICIT,
    ORC_U_SET_RHS,
    ORC_V_SET_RHS,
    ORC_U_SOLVE_CG,
    ORC_V_SOLVE_CG,
    ORC_U_UPDATE_BOUNDARIES,
    ORC_V_UPDATE_BOUNDARIES,
    ORC_PRESSURE_SET_RHS,
    ORC_PRESSURE_PRECONDITIONER,
    ORC_PRESSURE_SOLVE_CG,
    ORC_PRESSURE_PROJECT,
    ORC_PRESSURE_DIVERGENCE,
    ORC_ROUTINE_COUNT
};

int orc_create(const pvof_grid_desc *grid, const pvof_params *params, orc_t **out);
void orc_destroy(orc_t *o);
/* fields are exchanged in the same host block layout as pvof_upload_field */
size_t orc_field_block_count(const orc_t *o, int field);
int orc_set_field(orc_t *o, int field, const double *block, size_t count);
int orc_get_field(const orc_t *o, int field, double *block, size_t count);
int orc_set_stage(orc_t *o, int which_stage, double dt);
int orc_routine(orc_t *o, int routine, pvof_stats *stats);
int orc_substep(orc_t *o, pvof_stats *stats);
int orc_run_steps(orc_t *o, int nsteps, double dt, pvof_stats *stats);
double orc_liquid_mass(const orc_t *o);

#ifdef __cplusplus
}
#endif

#endif
