/* Planar 2D two-phase case: x periodic, no-slip walls in y, gravity, no
 * surface tension, no solids.  Flags as in the reference's Boundary.h. */
#define H_BOUNDARY
#define TWOD_CARTESIAN
#define XPERIODIC
#define ZPERIODIC
#define BOTTOM_WALL_VELOCITY_NOSLIP
#define TOP_WALL_VELOCITY_NOSLIP
#include "common.h"
