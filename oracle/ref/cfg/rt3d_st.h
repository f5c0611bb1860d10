/* 3D two-phase box with the potential-form surface tension force: x and z
 * periodic, no-slip walls in y, gravity, no solids (the precision form's
 * configuration). */
#define H_BOUNDARY
#define XPERIODIC
#define ZPERIODIC
#define BOTTOM_WALL_VELOCITY_NOSLIP
#define TOP_WALL_VELOCITY_NOSLIP
#define SURFACE_TENSION
#include "common.h"
