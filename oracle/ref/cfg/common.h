/*
 * Compile-time feature set shared by every oracle build of the reference
 * sources.  Each per-case header defines the include guard of the
 * reference's Boundary.h (H_BOUNDARY) so that the reference's own flag file
 * is skipped, then sets the flags of that case and includes this file.
 * The flag names are the reference's (src/Include/Boundary.h); only the
 * subset that the two-phase diffuse-interface path reads is set here.
 */
#ifndef PVOF_REFCFG_COMMON_H
#define PVOF_REFCFG_COMMON_H

/* solver and discretisation (Boundary.h:230-236, logic checks :410-420) */
#define CG_SOLVE
#define FULLY_IMPLICIT
#define GRID_UNIFORM

/* diffuse-interface two-phase model (Boundary.h:251-262); HYPRE is not
 * linked, so the in-tree Jacobi-PCG pressure solver is selected */
#define VOF
#define VOF_DIFFUSE
#define VOF_GRAVITY
#undef USE_HYPRE
#undef GPU_PRESSURE_SOLVER

/* collision model selection required by the logic checks (Boundary.h:480-500) */
#define ACTM
#define LIN_TAN
#define STORE_COLLISION
#define LAG_MARKER_FLAG
#define SUBSTEP
#define LUBRICATION_NORMAL

#if defined TWOD_CARTESIAN || defined AXISYM_RZ
#define TWOD_MODE
#endif

#endif
