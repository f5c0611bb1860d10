/*
 * Row-weighted pressure right-hand side for the axisymmetric oracle builds.
 * Test infrastructure only.
 *
 * In the axisymmetric mode the reference multiplies every row of its pressure
 * operator by the cell radius r_c so that the matrix is symmetric
 * (TwodOps_pressure_row_weight, PARTIES/src/Eulerian/TwodOps.c:144-157;
 * psolve_cg.c:90, :336).  Its HYPRE solver multiplies the right-hand side by
 * the same weight (psolve_hypre.c:184-200, b = -row_w * rhs), but its in-tree
 * Jacobi-PCG (psolve_cg.c:130-293), the solver the oracle builds use because
 * HYPRE is not available, solves r_c L phi = rhs with the unweighted
 * divergence from Pressure_set_RHS (Pressure.c:100-196).  That system is not
 * the projection's: the divergence after the projection grows over the outer
 * Poisson passes and the run aborts.
 *
 * Linked with -Wl,--wrap=Pressure_solve_cg, every call of the reference's
 * Pressure_solve_cg (Temporal_int.c:1071) comes here: the right-hand side is
 * multiplied by r_c over the solve range (the reference's own index ranges),
 * the reference's solver runs unchanged, and the unweighted right-hand side is
 * put back.  Planar builds do not link this file.
 */
#include "DataTypes.h"
#include "TwodOps.h"
#include "definitions.h"

#include <stdlib.h>
#include <string.h>

int __real_Pressure_solve_cg(Cart3d_bag *data_bag);

int __wrap_Pressure_solve_cg(Cart3d_bag *data_bag)
{
    MAC_grid *g = data_bag->grid;
    Parameters *params = data_bag->params;
    double ***rhs = data_bag->p->rhs;
    int Is = g->G_Is, Js = g->G_Js, Ks = g->G_Ks;
    int Ie = min(g->G_Ie, g->NX - 1);
    int Je = min(g->G_Je, g->NY - 1);
    int Ke = min(g->G_Ke, g->NZ - 1);
    size_t n = (size_t)(Ke - Ks) * (size_t)(Je - Js) * (size_t)(Ie - Is);
    double *saved = (double *)malloc(sizeof(double) * (n ? n : 1));
    size_t q = 0;
    for (int k = Ks; k < Ke; k++)
        for (int j = Js; j < Je; j++)
            for (int i = Is; i < Ie; i++) {
                saved[q++] = rhs[k][j][i];
                rhs[k][j][i] *= TwodOps_pressure_row_weight(g, params, i);
            }
    int iters = __real_Pressure_solve_cg(data_bag);
    q = 0;
    for (int k = Ks; k < Ke; k++)
        for (int j = Js; j < Je; j++)
            for (int i = Is; i < Ie; i++)
                rhs[k][j][i] = saved[q++];
    free(saved);
    return iters;
}
