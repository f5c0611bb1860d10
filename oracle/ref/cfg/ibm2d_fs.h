/* As ibm2d, with free-slip walls in y.  Flags as in the reference's
 * Boundary.h. */
#define H_BOUNDARY
#define TWOD_CARTESIAN
#define XPERIODIC
#define ZPERIODIC
#define BOTTOM_WALL_VELOCITY_FREESLIP
#define TOP_WALL_VELOCITY_FREESLIP
#define VOF_IBM
#define LAG_PARTICLE_RESOLVED
#include "common.h"
