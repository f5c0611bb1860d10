/* Planar 2D two-phase case with the potential-form surface tension force:
 * x periodic, no-slip walls in y, gravity, no solids. */
#define H_BOUNDARY
#define TWOD_CARTESIAN
#define XPERIODIC
#define ZPERIODIC
#define BOTTOM_WALL_VELOCITY_NOSLIP
#define TOP_WALL_VELOCITY_NOSLIP
#define SURFACE_TENSION
#include "common.h"
