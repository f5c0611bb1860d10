/* 3D two-phase box: x and z periodic, no-slip walls in y, gravity, no solids,
 * no surface tension. */
#define H_BOUNDARY
#define XPERIODIC
#define ZPERIODIC
#define BOTTOM_WALL_VELOCITY_NOSLIP
#define TOP_WALL_VELOCITY_NOSLIP
#include "common.h"
