/* Axisymmetric (r, z) two-phase case with surface tension: the symmetry axis
 * on the left, no-slip walls elsewhere, gravity, no solids.  Flags as in the
 * reference's Boundary.h (AXISYM_RZ reserves the left boundary for the axis;
 * the collapsed third direction is periodic, as in the reference's own
 * default branch). */
#define H_BOUNDARY
#define AXISYM_RZ
#define AXISYM_NO_SWIRL
#define ZPERIODIC
#define RIGHT_WALL_VELOCITY_NOSLIP
#define BOTTOM_WALL_VELOCITY_NOSLIP
#define TOP_WALL_VELOCITY_NOSLIP
#define SURFACE_TENSION
#include "common.h"
