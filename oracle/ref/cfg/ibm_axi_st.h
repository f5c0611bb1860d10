/* Axisymmetric (r, z) two-phase case with resolved solid spheres on the
 * symmetry axis (VOF_IBM, LAG_PARTICLE_RESOLVED) and surface tension: the
 * axis on the left, no-slip walls elsewhere, gravity.  Flags as in the
 * reference's Boundary.h (AXISYM_RZ reserves the left boundary for the axis;
 * the collapsed third direction is periodic, as in its default branch). */
#define H_BOUNDARY
#define AXISYM_RZ
#define AXISYM_NO_SWIRL
#define ZPERIODIC
#define RIGHT_WALL_VELOCITY_NOSLIP
#define BOTTOM_WALL_VELOCITY_NOSLIP
#define TOP_WALL_VELOCITY_NOSLIP
#define VOF_IBM
#define LAG_PARTICLE_RESOLVED
#define SURFACE_TENSION
#include "common.h"
