/*
 * Link stubs for the reference entry points whose sources the oracle build
 * leaves out (HDF5 output/resume, particle output and particle-file input).  The oracle
 * driver never calls them; each aborts if it is reached.
 * Test infrastructure only.
 */
#include "DataTypes.h"
#include <stdio.h>
#include <stdlib.h>

static void ref_stub_abort(const char *name)
{
    fprintf(stderr, "oracle build: %s is not part of the single-rank oracle\n", name);
    abort();
}

void Output_h5_resume(Cart3d_bag *data_bag, Debug_trace *dtrace) { (void)data_bag; (void)dtrace; ref_stub_abort("Output_h5_resume"); }
void Output_h5_data(Cart3d_bag *data_bag, Debug_trace *dtrace) { (void)data_bag; (void)dtrace; ref_stub_abort("Output_h5_data"); }
void Resume_h5_resume(Cart3d_bag *data_bag, Debug_trace *dtrace) { (void)data_bag; (void)dtrace; ref_stub_abort("Resume_h5_resume"); }
void Resume_h5_data(Cart3d_bag *data_bag, Debug_trace *dtrace) { (void)data_bag; (void)dtrace; ref_stub_abort("Resume_h5_data"); }
void ParticleInput_h5(Cart3d_bag *data_bag, Debug_trace *dtrace) { (void)data_bag; (void)dtrace; ref_stub_abort("ParticleInput_h5"); }
#ifndef LAG_PARTICLE_RESOLVED
/* builds with resolved particles read their particle lists in ibm_driver.c */
void ParticleInput_inp(Particle_list *p_list, MAC_grid *grid, Parameters *params, Debug_trace *dtrace)
{ (void)p_list; (void)grid; (void)params; (void)dtrace; ref_stub_abort("ParticleInput_inp"); }
#endif
void ParticleOutput_dat(Particle_list *p_list, MAC_grid *grid, Parameters *params, Debug_trace *dtrace)
{ (void)p_list; (void)grid; (void)params; (void)dtrace; ref_stub_abort("ParticleOutput_dat"); }
void ParticleOutput_h5(Cart3d_bag *data_bag, int counter, Debug_trace *dtrace)
{ (void)data_bag; (void)counter; (void)dtrace; ref_stub_abort("ParticleOutput_h5"); }
