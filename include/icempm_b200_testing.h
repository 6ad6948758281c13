/*
 * Test hooks of icempm_b200 (no reference counterpart). They select kernel
 * variants and run single device routines so that tests can compare them
 * with the CPU oracle; they are not needed to run a simulation.
 */
#ifndef ICEMPM_B200_TESTING_H
#define ICEMPM_B200_TESTING_H

#include "icempm_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* P2G kernel of the phase API and of mpm_step: 0 = shared-memory tile with
 * one flush per tile node (default), 1 = one thread per particle with 27x4
 * global atomics, 2 = as 1 with a warp reduction over particles sharing a
 * base cell, 3 = as 0 with that warp reduction. */
int mpm_testing_set_p2g_variant(mpm_handle* h, int variant);

/* Runs the device 3x3 SVD on `count` row-major matrices A (9 doubles each)
 * on `device`: mode 0 = FP32 arithmetic of the reference, mode 1 = FP64.
 * U, V receive 9 doubles per matrix, S 3. Allocates its own scratch. */
int mpm_testing_svd3x3(int mode, const double* A, int count, double* U, double* S, double* V, int device);

/* Copies the grid to the host as 4 rows [m, mvx|vx, mvy|vy, mvz|vz] of
 * (GridXTotal + 2*GridHaloSize)*GridY*GridZ doubles, node order
 * ((x + halo)*GridY + y)*GridZ + z (the reference's one-partition buffer). */
int mpm_testing_download_grid(mpm_handle* h, double* out);

/* sizeof(SimParams3D) as compiled into the library (layout check). */
size_t mpm_testing_sizeof_params(void);

#ifdef __cplusplus
}
#endif

#endif
