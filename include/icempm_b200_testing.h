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

/* P2G kernel of the phase API and of mpm_step: 0 = shared-memory FP64 tile
 * with one flush per tile node, 1 = one thread per particle with 27x4
 * global atomics, 2 = as 1 with a warp reduction over particles sharing a
 * base cell, 3 = as 0 with that warp reduction, 4 = shared-memory tile in
 * 64-bit block fixed point over 1024-particle chunks, 5 (default) and 6 =
 * as 1 with same-cell particle pairs merged by one shuffle round
 * (128-thread blocks, 6 and 4 per SM). In the mixed mode (where 0..4 give MPM_ERR_ARG) 5..9
 * select the fused kernel's scatter: 5 = warp-reduced float4 atomics,
 * 6 = float4 atomics per particle, 7 = FP32 shared-memory tile,
 * 8 = int32 block fixed-point shared-memory tile, 9 = float4 atomics with
 * same-cell particle pairs merged in registers (default), 10 = split
 * scatter: a same-cell pair exchanges its payloads once and each lane adds
 * both particles' contributions over half of the stencil. 10 needs G2P
 * variant 5 (the default); with the other gathers it runs as 9. */
int mpm_testing_set_p2g_variant(mpm_handle* h, int variant);

/* G2P kernel occupancy target (FP64 modes): 0 = 4 blocks of 128 threads per
 * SM (default), 1 = 3 blocks, 2 = 6 blocks (fewer registers per thread). In
 * the mixed mode the fused kernel's target: 0 = 4, 1 = 5, 2 = 6 blocks;
 * 3 = 6, 4 = 5 and 5 = 8 blocks (default) with each warp's velocity box
 * staged in shared memory for the gather by the warp's loads, 6 = 8 blocks
 * with the box brought in by one TMA tensor copy per warp (mixed mode only;
 * MPM_ERR_ARG where the driver cannot encode the tensor map). */
int mpm_testing_set_g2p_variant(mpm_handle* h, int variant);

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

/* The bounded wait of the kernels' asynchronous (TMA) copies, run on an
 * mbarrier armed for bytes that no copy delivers (nothing is in flight):
 * *status receives MPM_ERR_COPY_TIMEOUT after `polls` polls (0 would mean the
 * phase completed). Returns 0, or MPM_ERR_CUDA if the launch failed. */
int mpm_testing_copy_wait_timeout(int device, int polls, int* status);

/* Number of grid nodes with non-zero mass in the current P2G result (the
 * accumulator in mixed mode; the grid after P2G in FP64 modes). */
int mpm_testing_active_nodes(mpm_handle* h, long long* count);

/* sizeof(SimParams3D) as compiled into the library (layout check). */
size_t mpm_testing_sizeof_params(void);

#ifdef __cplusplus
}
#endif

#endif
