// FP64 transfer kernels of the single-partition step.
//
// Device layouts
//   particles: SoA, row r of the reference's 28-row layout at pts + r*pitch
//              (parameters_sim_3d.h:29-38); pitch a multiple of 32 doubles
//   grid:      SoA, 4 arrays [m, m vx, m vy, m vz] gstride doubles apart (as
//              the reference's 4 pitched arrays, gpu_partition_3d.cu:88-95);
//              after the node update [m, vx, vy, vz]. Node (x, y, z), x in
//              [-halo, GridX + halo), at ((x + halo) * GridY + y) * GridZ + z.
#pragma once

#include "device_common.cuh"
#include "physics_f64.cuh"

namespace icempm {

// ------------------------------------------------------------------ P2G

// Per-particle data of partition_kernel_p2g (mpm_kernels.cuh:24-81): node
// contributions are  m w  and  w (m v + S (x_node - x_p)),
// S = m C - dt V Dp^-1 tau.
struct P2GPoint {
    int base[3];
    double fx[3];
    double mass;
    double mv[3];
    double S[3][3];
};

// Loads particle i and forms its P2G payload; false if disabled.
__device__ __forceinline__ bool p2g_prepare(const DevParams& P, const double* __restrict__ pts, size_t pitch, int i,
                                            P2GPoint& q, int* err) {
    const long long util = __double_as_longlong(pts[i]);
    if (util & kDisabled) return false;
    const bool liquid = (util & kLiquid) != 0;
    q.mass = liquid ? P.liquid_mass : P.particle_mass;
    double pos[3], vel[3], F[3][3], C[3][3];
#pragma unroll
    for (int d = 0; d < 3; d++) {
        pos[d] = pts[(MPM_POSX + d) * pitch + i];
        vel[d] = pts[(MPM_VELX + d) * pitch + i];
    }
#pragma unroll
    for (int r = 0; r < 3; r++)
#pragma unroll
        for (int c = 0; c < 3; c++) {
            F[r][c] = pts[(MPM_FE00 + 3 * r + c) * pitch + i];
            C[r][c] = pts[(MPM_BP00 + 3 * r + c) * pitch + i];
        }
    double tau[3][3];
    if (liquid) {
        const double pw = water_pressure(P, pts[MPM_IDX_JP_INV * pitch + i]);
#pragma unroll
        for (int r = 0; r < 3; r++)
#pragma unroll
            for (int c = 0; c < 3; c++) tau[r][c] = (r == c) ? pw : 0.0;
    } else {
        kirchhoff_wolper(P, F, tau);
    }
#pragma unroll
    for (int r = 0; r < 3; r++)
#pragma unroll
        for (int c = 0; c < 3; c++) q.S[r][c] = q.mass * C[r][c] - P.dt_vol_Dpinv * tau[r][c];
#pragma unroll
    for (int d = 0; d < 3; d++) {
        q.mv[d] = vel[d] * q.mass;
        q.base[d] = (int)(pos[d] * P.h_inv - 0.5);
        q.fx[d] = pos[d] * P.h_inv - (double)q.base[d];
    }
    const int e = stencil_error(P, q.base[0], q.base[1], q.base[2]);
    if (e) raise_error(err, e);
    return true;
}

// Calls emit(a, b, c, incM, incV) for the 27 stencil nodes (base + (a,b,c)).
template <class Emit>
__device__ __forceinline__ void p2g_scatter(const DevParams& P, const P2GPoint& q, Emit&& emit) {
    double ww[3][3];
    quad_weights<double>(q.fx, ww);
    const double h = P.h;
#pragma unroll
    for (int a = 0; a < 3; a++) {
        const double dx = (a - q.fx[0]) * h;
#pragma unroll
        for (int b = 0; b < 3; b++) {
            const double dy = (b - q.fx[1]) * h;
            const double wab = ww[a][0] * ww[b][1];
            double part[3];
#pragma unroll
            for (int m = 0; m < 3; m++) part[m] = q.S[m][0] * dx + q.S[m][1] * dy;
#pragma unroll
            for (int c = 0; c < 3; c++) {
                const double dz = (c - q.fx[2]) * h;
                const double W = wab * ww[c][2];
                double incV[3];
#pragma unroll
                for (int m = 0; m < 3; m++) incV[m] = W * (q.mv[m] + (part[m] + q.S[m][2] * dz));
                emit(a, b, c, W * q.mass, incV);
            }
        }
    }
}

// Adds one node contribution to the SoA grid (4 arrays, gs doubles apart).
__device__ __forceinline__ void grid_atomic_add(double* __restrict__ grid, long long gs, long long idx, double m,
                                                const double v[3]) {
    atomicAdd(grid + idx, m);
    atomicAdd(grid + gs + idx, v[0]);
    atomicAdd(grid + 2 * gs + idx, v[1]);
    atomicAdd(grid + 3 * gs + idx, v[2]);
}

// Pair key of a particle: its base-cell index, or a lane-unique negative
// value for lanes that must act alone (inactive, or a stencil reaching
// outside the grid).
__device__ __forceinline__ long long base_key(const DevParams& P, const P2GPoint& q, bool ok, int lane) {
    if (!ok) return -1 - lane;
    return node_index(P, q.base[0], q.base[1], q.base[2]);
}

// P2G with lanes that share a base cell merged in pairs by one shuffle round
// per node (cell-sorted order puts them in neighbouring lanes; the
// odd-ranked partner's four sums go to the even-ranked lane, which issues the
// FP64 atomics for both), 128-thread blocks at 6 blocks per SM.
__global__ void __launch_bounds__(128, 6) k_p2g_pairs_f64(DevParams P, const double* __restrict__ pts, size_t pitch,
                                                             int n, double* __restrict__ grid, int* err) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31;
    P2GPoint q;
    bool active = (i < n) && p2g_prepare(P, pts, pitch, i, q, err);
    const bool inside = active && !stencil_error(P, q.base[0], q.base[1], q.base[2]);
    if (!inside) {
        q.mass = 0;
        if (!active) {
#pragma unroll
            for (int d = 0; d < 3; d++) { q.base[d] = 0; q.fx[d] = 1.0; q.mv[d] = 0; }
#pragma unroll
            for (int r = 0; r < 3; r++)
#pragma unroll
                for (int c = 0; c < 3; c++) q.S[r][c] = 0;
        }
    }
    const long long key = base_key(P, q, inside, lane);
    const unsigned peers = __match_any_sync(0xffffffffu, key);
    const int rank = __popc(peers & ((1u << lane) - 1u));
    const long long next_key = __shfl_down_sync(0xffffffffu, key, 1);
    const bool absorb = lane < 31 && next_key == key && (rank & 1) == 0;
    const bool absorbed = __shfl_up_sync(0xffffffffu, (int)absorb, 1) != 0 && lane > 0;
    p2g_scatter(P, q, [&](int a, int b, int c, double incM, const double incV[3]) {
        double v[4] = {incM, incV[0], incV[1], incV[2]};
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const double o = __shfl_down_sync(0xffffffffu, v[k], 1);
            if (absorb) v[k] += o;
        }
        if (!active || absorbed) return;
        const int x = q.base[0] + a, y = q.base[1] + b, z = q.base[2] + c;
        if (!inside && !node_inside(P, x, y, z)) return;
        const double vv[3] = {v[1], v[2], v[3]};
        grid_atomic_add(grid, P.gstride, node_index(P, x, y, z), v[0], vv);
    });
}

// ----------------------------------------------------------- grid update

// partition_kernel_update_nodes (mpm_kernels.cuh:138-232) for one partition:
// v = mv/m, gravity, speed clamp, cylindrical indenter contact with its force
// added to the angle x z sensor and to this substep's total, wall conditions.
// force3 receives the block-reduced force of this substep (3 doubles).
// One node with mass of partition_kernel_update_nodes: v (the node's momentum
// on entry) becomes its velocity; the contact force goes to f and the sensor.
__device__ __forceinline__ void update_node_f64(const DevParams& P, double* __restrict__ grid, long long idx,
                                                double mass, double v[3], double ind_x, double ind_y,
                                                double* __restrict__ sensor, double f[3]) {
    int idx_z, idx_y;
    const long long col = div_by64(idx, P.Gz, P.inv_gz, idx_z);
    const int idx_x = (int)div_by64(col, P.Gy, P.inv_gy, idx_y);
    const int gx = idx_x - P.halo, gy = idx_y, gz = idx_z;
#pragma unroll
    for (int k = 0; k < 3; k++) v[k] /= mass;
    v[1] -= P.dt_gravity;
    const double vsq = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
    if (vsq > P.vmax_sq) {
        const double nv = sqrt(vsq);
#pragma unroll
        for (int k = 0; k < 3; k++) v[k] = v[k] / nv * P.vmax;
    }
    if (P.setup_type != 2) {
        double n0 = gx * P.h - ind_x, n1 = gy * P.h - ind_y;
        const double nsq = n0 * n0 + n1 * n1;
        if (nsq < P.ind_rsq) {
            const double vrel[3] = {v[0] - P.ind_velocity, v[1], v[2]};
            if (nsq > 0) { const double nn = sqrt(nsq); n0 /= nn; n1 /= nn; }
            const double vn = vrel[0] * n0 + vrel[1] * n1;
            if (vn < 0) {
                const double vt[3] = {vrel[0] - n0 * vn, vrel[1] - n1 * vn, vrel[2]};
                const double prev[3] = {v[0], v[1], v[2]};
                v[0] = P.ind_velocity + vt[0];
                v[1] = vt[1];
                v[2] = vt[2];
                // a node in the overlap of two partitions is updated
                // by both; its force is counted by its owner only
                if (gx >= P.own_lo && gx < P.own_hi) {
                    double fn[3];
#pragma unroll
                    for (int k = 0; k < 3; k++) { fn[k] = (prev[k] - v[k]) * mass / P.dt; f[k] += fn[k]; }
                    float angle = atan2f((float)n0, (float)n1);
                    angle = (float)((double)angle + MPM_PI);
                    angle = (float)((double)angle * (P.subdiv / (2 * MPM_PI)));
                    const int ia = min(max((int)angle, 0), P.subdiv - 1);
                    const int iz = min(max(idx_z, 0), P.Gz - 1);
                    double* s = sensor + 3 * (iz + ia * P.Gz);
                    atomicAdd(s + 0, fn[0]);
                    atomicAdd(s + 1, fn[1]);
                    atomicAdd(s + 2, fn[2]);
                }
            }
        }
    }
    if (P.setup_type != 2) {
        if (gy <= 2) { v[0] = v[1] = v[2] = 0; }
    } else {
        if (gy <= 2 && v[1] < 0) v[1] = 0;
    }
    if (gy >= P.Gy - 3 && v[1] > 0) v[1] = 0;
    if (gx <= 2 && v[0] < 0) v[0] = 0;
    else if (gx >= P.Gx - 3 && v[0] > 0) v[0] = 0;
    if (gz <= 2 && v[2] < 0) v[2] = 0;
    else if (gz >= P.Gz - 3 && v[2] > 0) v[2] = 0;
    if (P.setup_type == 2 && P.drag != 0) {
#pragma unroll
        for (int k = 0; k < 3; k++) v[k] *= (1 - P.drag);
    }
    grid[P.gstride + idx] = v[0];
    grid[2 * P.gstride + idx] = v[1];
    grid[3 * P.gstride + idx] = v[2];
}

// partition_kernel_update_nodes (mpm_kernels.cuh:138-232) for one partition:
// v = mv/m, gravity, speed clamp, cylindrical indenter contact with its force
// added to the angle x z sensor and to this substep's total, wall conditions.
// force3 receives the block-reduced force of this substep (3 doubles). Two
// nodes per thread, BLOCK apart, with all eight of their sums loaded before
// either is used (8 M block: 0.053 ms against 0.073 ms for one node per thread
// that read a node's momentum only after its mass).
constexpr int kUpdateF64NodesPerThread = 2;
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_update_f64(DevParams P, double* __restrict__ grid, double ind_x, double ind_y,
                                                      double* __restrict__ sensor, double* __restrict__ force3) {
    constexpr int NPT = kUpdateF64NodesPerThread;
    const long long idx0 = (long long)P.node_lo + (long long)blockIdx.x * (BLOCK * NPT) + threadIdx.x;
    double f[3] = {0, 0, 0};
    double m[NPT], v[NPT][3];
#pragma unroll
    for (int j = 0; j < NPT; j++) {
        const long long idx = idx0 + j * BLOCK;
        m[j] = 0;
        if (idx < P.node_hi) {
            m[j] = grid[idx];
#pragma unroll
            for (int k = 0; k < 3; k++) v[j][k] = grid[(k + 1) * P.gstride + idx];
        }
    }
#pragma unroll
    for (int j = 0; j < NPT; j++)
        if (m[j] != 0) update_node_f64(P, grid, idx0 + j * BLOCK, m[j], v[j], ind_x, ind_y, sensor, f);
    // block reduction of the substep force (only blocks that touch the
    // indenter contribute non-zero values)
    __shared__ double red[3][BLOCK / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    bool any = (f[0] != 0) | (f[1] != 0) | (f[2] != 0);
    if (!__syncthreads_or(any)) return;
#pragma unroll
    for (int k = 0; k < 3; k++) {
        double x = f[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        if (lane == 0) red[k][warp] = x;
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        double x = 0;
        for (int w = 0; w < BLOCK / 32; w++) x += red[threadIdx.x][w];
        atomicAdd(force3 + threadIdx.x, x);
    }
}

// ------------------------------------------------------------------ G2P

// Gathers v and C (APIC "Bp") of one particle from the updated grid
// (mpm_kernels.cuh:278-305). Out-of-grid nodes contribute nothing.
__device__ __forceinline__ void g2p_gather(const DevParams& P, const double* __restrict__ grid, const double pos[3],
                                           double vel[3], double C[3][3], int* err) {
    int base[3];
    double fx[3];
#pragma unroll
    for (int d = 0; d < 3; d++) {
        base[d] = (int)(pos[d] * P.h_inv - 0.5);
        fx[d] = pos[d] * P.h_inv - (double)base[d];
    }
    const int e = stencil_error(P, base[0], base[1], base[2]);
    if (e) raise_error(err, e);
    double ww[3][3];
    quad_weights<double>(fx, ww);
    // v = sum w v_i and the first moments M_k = sum w v_i o_k over the node
    // offsets o = (a, b, c); C = 4/h sum w v_i (o - f) = 4/h (M - f v)
    double Mx[3], My[3], Mz[3];
#pragma unroll
    for (int d = 0; d < 3; d++) { vel[d] = 0; Mx[d] = 0; My[d] = 0; Mz[d] = 0; }
    const long long i0 = node_index(P, base[0], base[1], base[2]);
    const double* gx = grid + P.gstride;
    const double* gy = grid + 2 * P.gstride;
    const double* gz = grid + 3 * P.gstride;
#pragma unroll 1
    for (int a = 0; a < 3; a++) {
        const double wa = a == 0 ? ww[0][0] : (a == 1 ? ww[1][0] : ww[2][0]);
        double ra[3] = {0, 0, 0};
#pragma unroll
        for (int b = 0; b < 3; b++) {
            const long long ib = i0 + a * P.slab + b * P.Gz;
            const double wab = wa * ww[b][1];
            double rb[3] = {0, 0, 0};
#pragma unroll
            for (int c = 0; c < 3; c++) {
                const int x = base[0] + a, y = base[1] + b, z = base[2] + c;
                if (e && !node_inside(P, x, y, z)) continue;
                const long long ni = ib + c;
                const double w = wab * ww[c][2];
                const double wn[3] = {w * __ldg(gx + ni), w * __ldg(gy + ni), w * __ldg(gz + ni)};
#pragma unroll
                for (int r = 0; r < 3; r++) {
                    rb[r] += wn[r];
                    if (c == 1) Mz[r] += wn[r];
                    if (c == 2) Mz[r] += 2.0 * wn[r];
                }
            }
#pragma unroll
            for (int r = 0; r < 3; r++) {
                ra[r] += rb[r];
                if (b == 1) My[r] += rb[r];
                if (b == 2) My[r] += 2.0 * rb[r];
            }
        }
#pragma unroll
        for (int r = 0; r < 3; r++) {
            vel[r] += ra[r];
            Mx[r] += (double)a * ra[r];
        }
    }
    const double s4 = 4. * P.h_inv;
#pragma unroll
    for (int r = 0; r < 3; r++) {
        C[r][0] = s4 * (Mx[r] - fx[0] * vel[r]);
        C[r][1] = s4 * (My[r] - fx[1] * vel[r]);
        C[r][2] = s4 * (Mz[r] - fx[2] * vel[r]);
    }
}

// The particle update after the gather (mpm_kernels.cuh:307-327) up to the
// failure test: returns true for a crushed solid point, whose return map (on
// the trial F) is left to k_return_map_f64.
__device__ __forceinline__ bool g2p_advance_trial(const DevParams& P, double pos[3], const double vel[3],
                                                  const double C[3][3], double F[3][3], double& Jp_inv,
                                                  long long& util, double& p_tr, double& q_tr) {
    const double dt = P.dt;
#pragma unroll
    for (int d = 0; d < 3; d++) pos[d] += vel[d] * dt;
    double A[3][3];
#pragma unroll
    for (int r = 0; r < 3; r++)
#pragma unroll
        for (int c = 0; c < 3; c++) A[r][c] = (r == c ? 1.0 : 0.0) + dt * C[r][c];
    double Fn[3][3];
#pragma unroll
    for (int r = 0; r < 3; r++)
#pragma unroll
        for (int c = 0; c < 3; c++) Fn[r][c] = A[r][0] * F[0][c] + A[r][1] * F[1][c] + A[r][2] * F[2][c];
#pragma unroll
    for (int r = 0; r < 3; r++)
#pragma unroll
        for (int c = 0; c < 3; c++) F[r][c] = Fn[r][c];
    p_tr = 0;
    q_tr = 0;
    if (util & kLiquid) {
        Jp_inv *= det3(A);
        return false;
    }
    double Je;
    trial_pq(P, F, Je, p_tr, q_tr);
    if (!(util & kCrushed)) {
        if (outside_failure_surface(P, (short)util, p_tr, q_tr)) util |= kCrushed;
    }
    return (util & kCrushed) != 0;
}

// partition_kernel_g2p without migration (mpm_kernels.cuh:237-351), up to
// the failure test; a crushed point is appended to rm_list and its return map
// runs in k_return_map_f64 (it needs the SVD, whose registers would hold every
// thread of this kernel). 7 blocks of 128 per SM at 72 registers: 0.80 ms per
// launch on the 8 M block against 0.90 ms with the return map inline at 128
// registers (5 blocks: 0.90, 6: 0.85, 8 at 64 registers: 0.83 ms).
constexpr int kG2PF64Blocks = 7;
template <class K>
__global__ void __launch_bounds__(128, kG2PF64Blocks) k_g2p_f64(DevParams P, double* __restrict__ pts, size_t pitch,
                                                 int n, const double* __restrict__ grid, int record_pq,
                                                 int* err, int* __restrict__ rm_list, int* __restrict__ rm_count) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    long long util = __double_as_longlong(pts[i]);
    if (util & kDisabled) return;
    double pos[3], F[3][3];
#pragma unroll
    for (int d = 0; d < 3; d++) pos[d] = pts[(MPM_POSX + d) * pitch + i];
#pragma unroll
    for (int r = 0; r < 3; r++)
#pragma unroll
        for (int c = 0; c < 3; c++) F[r][c] = pts[(MPM_FE00 + 3 * r + c) * pitch + i];
    double Jp_inv = pts[MPM_IDX_JP_INV * pitch + i];

    double vel[3], C[3][3];
    g2p_gather(P, grid, pos, vel, C, err);
    double p_tr, q_tr;
    if (g2p_advance_trial(P, pos, vel, C, F, Jp_inv, util, p_tr, q_tr)) rm_list[atomicAdd(rm_count, 1)] = i;

#pragma unroll
    for (int d = 0; d < 3; d++) {
        pts[(MPM_POSX + d) * pitch + i] = pos[d];
        pts[(MPM_VELX + d) * pitch + i] = vel[d];
    }
#pragma unroll
    for (int r = 0; r < 3; r++)
#pragma unroll
        for (int c = 0; c < 3; c++) {
            pts[(MPM_FE00 + 3 * r + c) * pitch + i] = F[r][c];
            pts[(MPM_BP00 + 3 * r + c) * pitch + i] = C[r][c];
        }
    pts[MPM_IDX_JP_INV * pitch + i] = Jp_inv;
    pts[i] = __longlong_as_double(util);
    if (record_pq) {
        pts[MPM_IDX_P * pitch + i] = p_tr;
        pts[MPM_IDX_Q * pitch + i] = q_tr;
    }
}

// The return map (mpm_kernels.cuh:494-544) of the points k_g2p_f64 listed:
// the trial p, q again from the stored trial F (the same arithmetic), then
// F and Jp_inv projected. The list holds *count indices; the kernel also
// clears next_count, the counter the next k_g2p_f64 appends to.
template <class K>
__global__ void __launch_bounds__(128) k_return_map_f64(DevParams P, double* __restrict__ pts, size_t pitch,
                                                        const double* __restrict__ p0_arr,
                                                        const int* __restrict__ rm_list, const int* __restrict__ count,
                                                        int* __restrict__ next_count) {
    if (blockIdx.x == 0 && threadIdx.x == 0) *next_count = 0;
    const int m = *count;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < m; k += gridDim.x * blockDim.x) {
        const int i = rm_list[k];
        double F[3][3];
#pragma unroll
        for (int r = 0; r < 3; r++)
#pragma unroll
            for (int c = 0; c < 3; c++) F[r][c] = pts[(MPM_FE00 + 3 * r + c) * pitch + i];
        double Jp_inv = pts[MPM_IDX_JP_INV * pitch + i];
        const double p0 = p0_arr ? p0_arr[i] : P.p0;
        double Je, p_tr, q_tr;
        trial_pq(P, F, Je, p_tr, q_tr);
        drucker_prager_return<K>(P, F, Jp_inv, Je, p_tr, q_tr, p0);
#pragma unroll
        for (int r = 0; r < 3; r++)
#pragma unroll
            for (int c = 0; c < 3; c++) pts[(MPM_FE00 + 3 * r + c) * pitch + i] = F[r][c];
        pts[MPM_IDX_JP_INV * pitch + i] = Jp_inv;
    }
}

}  // namespace icempm
