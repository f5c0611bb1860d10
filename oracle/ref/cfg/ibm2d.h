/* Planar 2D two-phase case with resolved solid particles: as rt2d, plus the
 * diffuse-interface immersed-boundary coupling (VOF_IBM) and the resolved
 * Lagrangian particles (LAG_PARTICLE_RESOLVED).  Flags as in the reference's
 * Boundary.h. */
#define H_BOUNDARY
#define TWOD_CARTESIAN
#define XPERIODIC
#define ZPERIODIC
#define BOTTOM_WALL_VELOCITY_NOSLIP
#define TOP_WALL_VELOCITY_NOSLIP
#define VOF_IBM
#define LAG_PARTICLE_RESOLVED
#include "common.h"
