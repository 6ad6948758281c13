/*
 * CPU ORACLE — test infrastructure, not product code.
 *
 * A plain-C restatement of the reference's single-partition MLS-MPM step
 * (simulation/mpm_kernels.cuh and simulation/helper_math.cuh of
 * igorg520b/iceMPM_3Dm), used only by tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py, as the checker. Nothing in the product
 * (icempm_3dm_b200/) links, imports or calls it.
 *
 * Parity pinning:
 *   - the step (P2G, node update, G2P, the constitutive functions) is pinned
 *     against the reference's own simulation/mpm_kernels.cuh, compiled
 *     unmodified as host C++ from the reference tree (oracle/ref_kernels.cpp
 *     over the Eigen-API stand-in of oracle/refshim/; oracle/Makefile target
 *     `ref`): tests/test_oracle_vs_reference.py requires agreement to 1e-13
 *     phase by phase and 1e-11 over 30 substeps on inputs that reach every
 *     branch;
 *   - the 3x3 SVD restatement (or_svd3x3_f32) is pinned bit-for-bit against
 *     the reference's own helper_math.cuh svd<T>, compiled the same way, and
 *     against golden vectors generated from it (tests/golden/svd_ref.npz).
 *
 * Data layouts are the reference's:
 *   particles: host SoA, 28 rows of `pitch` doubles (parameters_sim_3d.h:29-38)
 *   grid: 4 arrays [m, mvx, mvy, mvz], each of (GridXTotal + 2*GridHaloSize)
 *         * GridY * GridZ doubles, node (x*GridY + y)*GridZ + z where buffer
 *         slab x holds grid column x - GridHaloSize (one partition,
 *         gpu_partition_3d.cu:88-95, mpm_kernels.cuh:92-93,163-166).
 */
#ifndef ICEMPM_ORACLE_H
#define ICEMPM_ORACLE_H

#include <stdint.h>
#include "../include/sim_params_3d.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Number of doubles per grid array for one partition. */
long long or_grid_nodes(const SimParams3D* prms);

/* 3x3 SVD as helper_math.cuh:24-1120 + svd3x3 (mpm_kernels.cuh:585-601):
 * A row-major, inputs narrowed to float; U, V row-major; S singular values. */
void or_svd3x3_f32(const double A[9], double U[9], double S[3], double V[9]);
/* The same algorithm carried out in double with `sweeps` Jacobi sweeps (the
 * "FP64 SVD" variant used as the high-accuracy reference). */
void or_svd3x3_f64(const double A[9], double U[9], double S[3], double V[9], int sweeps);
/* Forward-mode derivative of or_svd3x3_f64 in FP64 dual numbers: the tangent
 * (dU, dS, dV) of the factors along the direction dA. */
void or_svd3x3_dual(const double A[9], const double dA[9], double U[9], double dU[9], double S[3],
                    double dS[3], double V[9], double dV[9], int sweeps);

/* Cell key of ProxyPoint3D::getCellIndex (proxypoint3d.cpp:158-163). */
int or_cell_key(const SimParams3D* prms, double x, double y, double z);

/* HostSideSOA::RemoveDisabledAndSort (host_side_soa.cpp:56-67) as a stable
 * sort: perm[k] = source index of the k-th particle after the sort; returns
 * the new count (disabled particles removed). */
unsigned or_sort_permutation(const SimParams3D* prms, const double* soa, unsigned pitch,
                             unsigned n, unsigned* perm);

/* partition_kernel_p2g (mpm_kernels.cuh:20-100). grid must be zeroed by the
 * caller (4 * or_grid_nodes doubles). nthreads <= 1: serial, deterministic
 * particle order; > 1: OpenMP over slab windows. Returns 0 or 70..75. */
int or_p2g(const SimParams3D* prms, const double* soa, unsigned pitch, unsigned n,
           double* grid, int nthreads);

/* partition_kernel_update_nodes (mpm_kernels.cuh:138-232). sensor has
 * 3*IndenterSubdivisions*GridZ doubles and is accumulated into; force3
 * (may be NULL) receives the summed force of this call. */
void or_update_nodes(const SimParams3D* prms, double* grid, double ind_x, double ind_y,
                     double* sensor, double force3[3], int nthreads);

/* partition_kernel_g2p without migration (mpm_kernels.cuh:237-351) with the
 * constitutive functions of :434-581. p0 (may be NULL) = per-particle
 * Drucker-Prager apex shift replacing DP_threshold_p. svd_mode 0: FP32 SVD of
 * the reference; 1: FP64 SVD. Returns 0 or 70..75 (stencil outside grid). */
int or_g2p(const SimParams3D* prms, double* soa, unsigned pitch, unsigned n,
           const double* grid, int record_pq, const double* p0, int svd_mode, int nthreads);

/* One substep of Model3D::Step (model_3d.cpp:35-51): advances
 * prms->SimulationTime / indenter_x / SimulationStep like the reference.
 * grid: scratch of 4*or_grid_nodes doubles. force3: this substep's force. */
int or_step(SimParams3D* prms, double* soa, unsigned pitch, unsigned n, double* grid,
            double* sensor, double force3[3], const double* p0, int svd_mode, int nthreads);

/* FP64 dual-number forward-mode derivative of nsteps substeps of or_step
 * (serial, FP64 SVD): soa/dsoa are the initial state and its tangent (rows
 * and pitch as for soa), p0/dp0 (may be NULL) the per-particle apex shift
 * and its tangent, dE the tangent of YoungsModulus (carried into mu and
 * kappa). On return soa/dsoa hold the final state and its tangent and
 * force_hist/dforce_hist[3*nsteps] the indenter force of every substep and
 * its tangent. prms advances like or_step. Returns 0 or 70..75. */
int or_dual_steps(SimParams3D* prms, double* soa, double* dsoa, unsigned pitch, unsigned n,
                  const double* p0, const double* dp0, double dE, int nsteps,
                  double* force_hist, double* dforce_hist);

#ifdef __cplusplus
}
#endif

#endif
