/* Case of the constant-density FFT Poisson solver routine driver (fft_driver.c).
 * The reference's FFT solver needs an even number of cells in z
 * (Pressure_transpose_setup), so the driver runs it in 3D (NZM = 2, x and z
 * periodic, walls in y) on a right-hand side that does not depend on z; its
 * solution is then the 2D one on every z plane. */
#define H_BOUNDARY
#define XPERIODIC
#define ZPERIODIC
#define BOTTOM_WALL_VELOCITY_NOSLIP
#define TOP_WALL_VELOCITY_NOSLIP
#include "common.h"
