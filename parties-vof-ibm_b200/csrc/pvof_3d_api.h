// Entry points of the 3D mode (pvof_3d.cu), called by the C ABI in
// pvof_api.cu for contexts created with PVOF_GEOM_3D.  Errors return the
// negative PVOF_E* codes with the message in last_error().
#pragma once

#include <cstddef>

#include "../../include/pvof.h"

namespace pvof3 {

struct Handle;

const char *last_error();
int create(const pvof_grid_desc *grid, const pvof_params *params, int device, Handle **out);
int destroy(Handle *h);
size_t block_count(const Handle *h, int field);
int upload(Handle *h, int field, const double *host, size_t count);
int download(Handle *h, int field, double *host, size_t count);
int synchronize(Handle *h);
int set_stage(Handle *h, int stage, double dt);
int initialize(Handle *h);
int substep(Handle *h, pvof_stats *st);
int run_steps(Handle *h, int nsteps, double dt, pvof_stats *st);
int liquid_mass(Handle *h, double *mass);
long long launch_count(const Handle *h);
int set_solver_timing(Handle *h, int on);
int solver_timing(const Handle *h, int solver, double *ms, long long *launches, long long *iters, long long *cell_iters);
double clamp_total(const Handle *h);
int timer_start(Handle *h);
int timer_stop(Handle *h, double *ms);
int flush_l2(Handle *h);

}  // namespace pvof3
