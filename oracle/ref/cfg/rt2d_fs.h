/* Planar 2D two-phase case with free-slip walls in y: x periodic, gravity,
 * no surface tension, no solids.  Flags as in the reference's Boundary.h. */
#define H_BOUNDARY
#define TWOD_CARTESIAN
#define XPERIODIC
#define ZPERIODIC
#define BOTTOM_WALL_VELOCITY_FREESLIP
#define TOP_WALL_VELOCITY_FREESLIP
#include "common.h"
