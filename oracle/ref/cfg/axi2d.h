/* Axisymmetric (r, z) two-phase case: the symmetry axis on the left, no-slip
 * walls elsewhere, gravity, no surface tension, no solids.  Flags as in the
 * reference's Boundary.h (AXISYM_RZ reserves the left boundary for the axis). */
#define H_BOUNDARY
#define AXISYM_RZ
#define AXISYM_NO_SWIRL
#define ZPERIODIC
#define RIGHT_WALL_VELOCITY_NOSLIP
#define BOTTOM_WALL_VELOCITY_NOSLIP
#define TOP_WALL_VELOCITY_NOSLIP
#include "common.h"
