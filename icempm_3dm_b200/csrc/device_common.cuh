// Device-side parameter block, status word and small helpers shared by the
// kernels of the single-partition step.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/icempm_b200.h"

namespace icempm {

// The subset of SimParams3D the kernels read, with derived constants, passed
// by value as a kernel argument (the reference copies the whole struct to a
// __constant__ symbol, gpu_partition_3d.cu:140; a by-value argument lives in
// the same constant bank and keeps handles independent).
struct DevParams {
    int Gx, Gy, Gz, halo;          // GridXTotal, GridY, GridZ, GridHaloSize
    int setup_type;
    int subdiv;                    // IndenterSubdivisions
    long long nodes;               // (Gx + 2 halo) * Gy * Gz
    long long gstride;             // doubles between the 4 grid arrays
    long long slab;                // Gy * Gz
    double h, h_inv, dt;
    double particle_mass, liquid_mass;
    double dt_vol_Dpinv;
    double dt_gravity, vmax, vmax_sq;
    double ind_rsq, ind_velocity;
    double mu, kappa;
    double pmax, tensile, shear, tensile2, beta, grain_var;
    double tan_phi, p0;            // DP_tan_phi, DP_threshold_p
    double drag;
    // failure-surface constants for GrainVariability = 0 (FP32 fast path)
    float fs_pmin2, fs_k, fs_msq, fs_1p2b, fs_bpmax, fs_pmax;
    // FP32 copies for the mixed kernels, rounded once on the host (constant-
    // bank operands there, instead of a double multiply and a conversion in
    // every thread): h, 1/h, 4/h, dt, dt/h 2^20 (fixed-point advection), mu,
    // kappa, kappa/2, sqrt(3/2) mu, particle and liquid mass, dt V Dp^-1
    float f_h, f_h_inv, f_s4, f_dt, f_adv, f_mu, f_kappa, f_hkappa, f_qmu, f_pmass, f_lmass, f_dvd;
    // scales of the fixed-point grid accumulator (AccQ) and their inverses
    float f_qm, f_qp;
    double q_inv_m, q_inv_p;
    double inv_gz, inv_gy;         // 1 / Gz, 1 / Gy for node index -> (x, y, z)
    // x-slab window of a partition (GPU_Partition_3D::GridX_offset and
    // GridX_partition; one partition: the whole grid):
    int win_lo, win_hi;            // allowed base-node x of a particle: [x0 - halo, x0 + gxp + halo - 3]
    int own_lo, own_hi;            // grid columns x whose contact force this partition counts
    int node_lo, node_hi;          // node indices the update covers: slabs x0 - halo .. x0 + gxp + halo
};

// q = n / d and r = n % d for 0 <= n < 2^31 with the double reciprocal of d:
// the product is within 2^-22 of n/d, so one correction step makes it exact.
__device__ __forceinline__ long long div_by64(long long n, int d, double inv_d, int& r) {
    // as div_by for 0 <= n < 2^50: the quotient estimate is off by at most 1
    long long q = (long long)((double)n * inv_d);
    long long rr = n - q * d;
    if (rr < 0) { q--; rr += d; }
    else if (rr >= d) { q++; rr -= d; }
    r = (int)rr;
    return q;
}

__device__ __forceinline__ int div_by(int n, int d, double inv_d, int& r) {
    int q = __double2int_rz((double)n * inv_d);
    r = n - q * d;
    if (r < 0) { q--; r += d; }
    else if (r >= d) { q++; r -= d; }
    return q;
}

constexpr double kCoeff1 = 1.224744871391589;      // sqrt(3/2)
constexpr double kCoeff1Inv = 0.8164965809277260;  // 1/sqrt(3/2)
constexpr long long kCrushed = MPM_STATUS_CRUSHED;
constexpr long long kDisabled = MPM_STATUS_DISABLED;
constexpr long long kLiquid = MPM_STATUS_LIQUID;

// First error wins (the reference's byte is overwritten by any failing
// thread; with one failing particle the outcome is the same).
__device__ __forceinline__ void raise_error(int* err, int code) {
    if (*(volatile int*)err == 0) atomicCAS(err, 0, code);
}

// Bounds test of mpm_kernels.cuh:70-75 against the partition's window
// (base_x - GridX_offset outside [-halo, GridX_partition + halo - 3]): the
// last failing test of the sequence determines the code.
__device__ __forceinline__ int stencil_error(const DevParams& P, int bx, int by, int bz) {
    int e = 0;
    if (bx < P.win_lo) e = 70;
    if (by < 0) e = 71;
    if (bz < 0) e = 72;
    if (bx > P.win_hi) e = 73;
    if (by > P.Gy - 3) e = 74;
    if (bz > P.Gz - 3) e = 75;
    return e;
}

__device__ __forceinline__ bool node_inside(const DevParams& P, int x, int y, int z) {
    return x >= -P.halo && x < P.Gx + P.halo && y >= 0 && y < P.Gy && z >= 0 && z < P.Gz;
}

__device__ __forceinline__ long long node_index(const DevParams& P, int x, int y, int z) {
    return ((long long)(x + P.halo) * P.Gy + y) * P.Gz + z;
}

template <typename T>
__device__ __forceinline__ void quad_weights(const T fx[3], T ww[3][3]) {
    // quadratic B-spline weights, mpm_kernels.cuh:78-81
#pragma unroll
    for (int d = 0; d < 3; d++) {
        T v0 = (T)1.5 - fx[d], v1 = fx[d] - (T)1.0, v2 = fx[d] - (T)0.5;
        ww[0][d] = (T)0.5 * v0 * v0;
        ww[1][d] = (T)0.75 - v1 * v1;
        ww[2][d] = (T)0.5 * v2 * v2;
    }
}

}  // namespace icempm
