/*
 * Test hooks of icempm_b200 (no reference counterpart). They run single
 * device routines and read intermediate device state so that tests can
 * compare them with the CPU oracle; they are not needed to run a simulation.
 */
#ifndef ICEMPM_B200_TESTING_H
#define ICEMPM_B200_TESTING_H

#include "icempm_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Runs the device 3x3 SVD on `count` row-major matrices A (9 doubles each)
 * on `device`: mode 0 = FP32 arithmetic of the reference, mode 1 = FP64.
 * U, V receive 9 doubles per matrix, S 3. Allocates its own scratch. */
int mpm_testing_svd3x3(int mode, const double* A, int count, double* U, double* S, double* V, int device);

/* Copies the grid to the host as 4 rows [m, mvx|vx, mvy|vy, mvz|vz] of
 * (GridXTotal + 2*GridHaloSize)*GridY*GridZ doubles, node order
 * ((x + halo)*GridY + y)*GridZ + z (the reference's one-partition buffer).
 * FP64 modes keep one grid (which is ignored); the mixed mode keeps the
 * accumulator (which = 0: m, m v) and the updated velocities (which = 1:
 * 0, v) apart. */
int mpm_testing_download_grid(mpm_handle* h, double* out, int which);

/* Runs nsteps substeps like mpm_step (without the force history) with CUDA
 * events recorded on the handle's stream around each kernel; ms[0..3]
 * receive the summed durations of [grid clear, P2G, node update, G2P] (FP64
 * modes) or [-, return map of crushed points, node update, fused
 * G2P->P2G] (mixed mode). */
int mpm_testing_step_timed(mpm_handle* h, int nsteps, float* ms);

/* Number of grid nodes with non-zero mass in the current P2G result (the
 * accumulator in mixed mode; the grid after P2G in FP64 modes). */
int mpm_testing_active_nodes(mpm_handle* h, long long* count);

/* sizeof(SimParams3D) as compiled into the library (layout check). */
size_t mpm_testing_sizeof_params(void);

#ifdef __cplusplus
}
#endif

#endif
