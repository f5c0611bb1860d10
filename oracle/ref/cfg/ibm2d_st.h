/* As ibm2d, with surface tension (SURFACE_TENSION): the contact-line
 * extension of psi_LG runs at every third substep.  Flags as in the
 * reference's Boundary.h. */
#define H_BOUNDARY
#define TWOD_CARTESIAN
#define XPERIODIC
#define ZPERIODIC
#define BOTTOM_WALL_VELOCITY_NOSLIP
#define TOP_WALL_VELOCITY_NOSLIP
#define VOF_IBM
#define LAG_PARTICLE_RESOLVED
#define SURFACE_TENSION
#include "common.h"
