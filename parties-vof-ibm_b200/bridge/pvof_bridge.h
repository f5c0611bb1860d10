/*
 * pvof_bridge.h -- the PARTIES side of the B200 substep: a C file a PARTIES
 * build compiles (with the reference's own headers on its include path and
 * -DPVOF_GPU) and links against libpvof.so.  It maps the reference's
 * Cart3d_bag (PARTIES/src/Include/DataTypes.h:1616-1635) onto the C ABI of
 * include/pvof.h.
 *
 * Whole-substep use (the fast path): after the reference's start-up
 * (Cart3d_initialize_primitive_data and Particle_initialize), call
 * pvof_bridge_start once; in Temporal_int_rk3 (PARTIES/src/Temporal_int.c:
 * 399-448) call pvof_bridge_substep where the reference calls
 * Temporal_int_all_the_equations (:443), and drop the host
 * Velocity_cell_center just before it (:420-424; the bridge refreshes the
 * device copy itself); call pvof_bridge_download before anything on the host
 * reads the fields (output, statistics, restart) and pvof_bridge_upload after
 * anything on the host writes them.
 *
 * Routine-by-routine use: compiled with -DPVOF_BRIDGE_ROUTINES the file also
 * defines the reference's own routine names and signatures
 * (Include/VOF_DIFFUSE.h:7-30, VolumeFraction.h:52-84, Pressure.h:6-65,
 * Velocity.h), each a call of the matching pvof_ entry point on the device
 * copy of the state; the reference's CPU definitions of those routines must
 * then be left out of the link (or made weak).  Each of these routines copies
 * every state field to the device before the call and back after it, so the
 * reference's own orchestration (Temporal_int_all_the_equations) runs
 * unchanged around them, host operations between the calls included; that
 * copying makes this form a porting and checking aid, not the fast path.
 *
 * Every function returns 0 or a negative PVOF_E* code; with
 * -DPVOF_BRIDGE_ABORT a failure prints pvof_last_error() and aborts through
 * MPI_Abort instead, as the reference's Display_throw_error does
 * (PARTIES/src/IO/Display.c:910-941).
 */
#ifndef PVOF_BRIDGE_H
#define PVOF_BRIDGE_H

#include "DataTypes.h"
#include "pvof.h"

/* create the device context from the reference's parameters and compile-time
 * flags, copy F, u, v, p (and the particle lists) and run the library's
 * start-up (pvof_initialize); `device` is the CUDA device */
int pvof_bridge_start(Cart3d_bag *b, int device);
/* one RK substep at params->which_stage and params->dt: the device's
 * cell-centred velocity at stage 0 after t = 0, then pvof_substep */
int pvof_bridge_substep(Cart3d_bag *b);
/* device -> host: every state field of include/pvof.h's field list that the
 * reference keeps, and the particles' position, velocity, spin, force and
 * torque */
int pvof_bridge_download(Cart3d_bag *b);
/* host -> device: the same fields */
int pvof_bridge_upload(Cart3d_bag *b);
/* the last substep's statistics (iteration counts, residuals) */
const pvof_stats *pvof_bridge_stats(void);
pvof_ctx *pvof_bridge_context(void);
void pvof_bridge_stop(void);

#endif
