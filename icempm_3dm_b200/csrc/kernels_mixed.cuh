// Mixed-precision step: FP32 particle state and transfers, FP64 where
// precision needs it (3x3 SVD and return map of crushed particles, the
// indenter force reduction).
//
// Particle state (SoA, 26 words = 104 B per particle):
//   int32   X[3]   position in fixed point, x / h * 2^kFixBits
//   float   v[3]   velocity
//   float   E[9]   F - I (deviation of the elastic deformation gradient from
//                  the identity, so that J - 1 and dev(F F^T) keep their
//                  relative precision near the undeformed state)
//   float   C[9]   APIC affine matrix ("Bp")
//   float   Jp_inv - 1
//   int32   status (low 32 bits of the reference's utility word)
// optional float p0 (apex shift from cohesion), and float P, Q rows written
// on record steps.
//
// Grid: acc = float4 {m, m vx, m vy, m vz} per node, accumulated with
// float4 vector atomics (same-cell particle pairs merged in registers first);
// vel = float4 {vx, vy, vz, 0} per node, written by the node update (which
// also clears acc for the next P2G).
// One step is three kernels: node update, the fused G2P->P2G kernel (G2P of
// this step and P2G of the next read each particle once), and the FP64
// return map of the points that crushed (k_return_map_mixed, over a list).
#pragma once

#include "device_common.cuh"
#include "physics_f64.cuh"

namespace icempm {

constexpr int kFixBits = 20;
constexpr float kFixScale = 1048576.0f;           // 2^20
constexpr float kFixInv = 9.5367431640625e-07f;   // 2^-20

struct MixedState {
    int* X;          // 3 rows
    float* v;        // 3 rows
    float* E;        // 9 rows
    float* C;        // 9 rows
    float* Jpm1;     // Jp_inv - 1 (1 row): keeps the precision of Jp_inv near 1
    int* status;     // 1 row
    float* p0;       // 1 row or null
    float* PQ;       // 2 rows (P, Q)
    size_t pitch;
};

// base = (int)(x/h - 0.5) with C truncation, fx = x/h - base, from the
// fixed-point coordinate (exact: fx has 21 significant bits)
__device__ __forceinline__ void fix_base(int X, int& base, float& fx) {
    const int num = X - (1 << (kFixBits - 1));
    base = num / (1 << kFixBits);
    fx = (float)(X - base * (1 << kFixBits)) * kFixInv;
}

// J - 1 = det(I + E) - 1 without cancellation
__device__ __forceinline__ float detm1(const float E[3][3]) {
    const float tr = E[0][0] + E[1][1] + E[2][2];
    const float m2 = (E[0][0] * E[1][1] - E[0][1] * E[1][0]) + (E[0][0] * E[2][2] - E[0][2] * E[2][0]) +
                     (E[1][1] * E[2][2] - E[1][2] * E[2][1]);
    const float d = E[0][0] * (E[1][1] * E[2][2] - E[2][1] * E[1][2]) -
                    E[1][0] * (E[0][1] * E[2][2] - E[2][1] * E[0][2]) +
                    E[2][0] * (E[0][1] * E[1][2] - E[1][1] * E[0][2]);
    return tr + m2 + d;
}

// dev(F F^T) with F = I + E: dev(E + E^T + E E^T), symmetric (upper triangle mirrored)
__device__ __forceinline__ void dev_b(const float E[3][3], float D[3][3]) {
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = i; j < 3; j++) {
            D[i][j] = E[i][j] + E[j][i] + (E[i][0] * E[j][0] + E[i][1] * E[j][1] + E[i][2] * E[j][2]);
            D[j][i] = D[i][j];
        }
    const float t = (D[0][0] + D[1][1] + D[2][2]) * (1.0f / 3.0f);
    D[0][0] -= t; D[1][1] -= t; D[2][2] -= t;
}

// J - 1, J, J^(-2/3) and dev(F F^T) of F = I + E: shared by the trial p, q
// (mpm_kernels.cuh:477-484) and the Kirchhoff stress (:547-557)
struct ElasticInv {
    float jm1, J, jm23;
    float D[3][3];
};

__device__ __forceinline__ ElasticInv elastic_invariants(const float E[3][3]) {
    ElasticInv e;
    e.jm1 = detm1(E);
    e.J = 1.0f + e.jm1;
    e.jm23 = exp2f(-(2.0f / 3.0f) * log2f(e.J));
    dev_b(E, e.D);
    return e;
}

__device__ __forceinline__ void trial_pq_inv(const DevParams& P, const ElasticInv& e, float& p_tr, float& q_tr) {
    p_tr = -P.f_hkappa * (e.jm1 * (e.J + 1.0f));
    const float off = e.D[0][1] * e.D[0][1] + e.D[0][2] * e.D[0][2] + e.D[1][2] * e.D[1][2];
    const float sq = e.D[0][0] * e.D[0][0] + e.D[1][1] * e.D[1][1] + e.D[2][2] * e.D[2][2] + 2.0f * off;
    q_tr = P.f_qmu * e.jm23 * sqrtf(sq);
}

__device__ __forceinline__ void tau_inv(const DevParams& P, const ElasticInv& e, float tau[3][3]) {
    const float s = P.f_mu * e.jm23;
    const float hyd = P.f_hkappa * (e.jm1 * (e.J + 1.0f));
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) tau[i][j] = s * e.D[i][j] + (i == j ? hyd : 0.0f);
}

// CheckIfPointIsInsideFailureSurface (mpm_kernels.cuh:453-474) in FP32; the
// grain-independent constants come precomputed when GrainVariability = 0.
__device__ __forceinline__ bool outside_failure_surface_f32(const DevParams& P, short grain, float p_tr, float q_tr) {
    if (P.grain_var != 0.0) return outside_failure_surface(P, grain, (double)p_tr, (double)q_tr);
    if (p_tr < 0.f) {
        if (p_tr < P.fs_pmin2) return true;
        return q_tr > P.fs_k * (p_tr - P.fs_pmin2);
    }
    const float y = P.fs_1p2b * q_tr * q_tr + P.fs_msq * (p_tr + P.fs_bpmax) * (p_tr - P.fs_pmax);
    return y > 0.f;
}

// Kirchhoff stress (mpm_kernels.cuh:547-557) from E
__device__ __forceinline__ void kirchhoff_mixed(const DevParams& P, const float E[3][3], float tau[3][3]) {
    const float jm1 = detm1(E);
    const float J = 1.0f + jm1;
    float D[3][3];
    dev_b(E, D);
    const float s = P.f_mu * exp2f(-(2.0f / 3.0f) * log2f(J));
    const float hyd = P.f_hkappa * (jm1 * (J + 1.0f));
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) tau[i][j] = s * D[i][j] + (i == j ? hyd : 0.0f);
}

// Trial p, q (mpm_kernels.cuh:477-484) from E
__device__ __forceinline__ void trial_pq_mixed(const DevParams& P, const float E[3][3], float& jm1, float& p_tr,
                                               float& q_tr) {
    jm1 = detm1(E);
    const float J = 1.0f + jm1;
    p_tr = -P.f_hkappa * (jm1 * (J + 1.0f));
    float D[3][3];
    dev_b(E, D);
    float sq = 0.f;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) sq += D[i][j] * D[i][j];
    q_tr = P.f_qmu * exp2f(-(2.0f / 3.0f) * log2f(J)) * sqrtf(sq);
}

// w[a] of a 3-entry weight column with a loop counter that is not unrolled:
// selects keep the column in registers (an indexed load would place the
// whole weight array in local memory).
__device__ __forceinline__ float pick3(int a, float w0, float w1, float w2) {
    return a == 0 ? w0 : (a == 1 ? w1 : w2);
}

// The x-column of the weights in a per-thread shared-memory slot (stride
// 128 floats): read with the loop counter of a loop that is not unrolled, it
// costs one shared load per iteration and no register (local memory would
// also send its stores on to L2).
struct WxSlot {
    float* p;
    __device__ __forceinline__ void put(const float ww[3][3]) {
        p[0] = ww[0][0];
        p[128] = ww[1][0];
        p[256] = ww[2][0];
    }
    __device__ __forceinline__ float get(int a) const { return *(volatile const float*)(p + 128 * a); }
};

// ------------------------------------------------------------- G2P part

// Gathers v and C from the float4 velocity grid (mpm_kernels.cuh:278-305).
// Node indices step from the base node by constant offsets (32-bit: the
// handle checks that the grid has fewer than 2^31 nodes).
__device__ __forceinline__ void g2p_gather_mixed(const DevParams& P, const float4* __restrict__ vel, const int base[3],
                                                 const float fx[3], float v[3], float C[3][3], bool check, WxSlot wx) {
    float ww[3][3];
    quad_weights<float>(fx, ww);
    wx.put(ww);
#pragma unroll
    for (int d = 0; d < 3; d++) {
        v[d] = 0.f;
#pragma unroll
        for (int k = 0; k < 3; k++) C[d][k] = 0.f;
    }
    const float s4 = P.f_s4;
    const int slab = (int)P.slab, gz = P.Gz;
    const int i0 = ((base[0] + P.halo) * P.Gy + base[1]) * gz + base[2];
#pragma unroll 1
    for (int a = 0; a < 3; a++) {
        const float wa = wx.get(a);
        const float dpa = a - fx[0];
#pragma unroll
        for (int b = 0; b < 3; b++) {
            const float wab = wa * ww[b][1];
            const float dpb = b - fx[1];
            const int ib = i0 + a * slab + b * gz;
#pragma unroll
            for (int c = 0; c < 3; c++) {
                if (check && !node_inside(P, base[0] + a, base[1] + b, base[2] + c)) continue;
                const float4 nd = __ldg(vel + ib + c);
                const float w = wab * ww[c][2];
                const float nv[3] = {nd.x, nd.y, nd.z};
                const float dp[3] = {dpa, dpb, c - fx[2]};
                const float sw = s4 * w;
#pragma unroll
                for (int r = 0; r < 3; r++) {
                    v[r] += w * nv[r];
                    const float swv = sw * nv[r];
#pragma unroll
                    for (int k = 0; k < 3; k++) C[r][k] += swv * dp[k];
                }
            }
        }
    }
}

// Gather with the warp's velocity box staged in shared memory. The warp's
// lanes with an in-grid stencil (part) span a box of base cells; the box's
// nodes (base .. base+2 per axis) are copied from the grid once, row by row
// along z (coalesced, 16-byte cp.async), into this warp's slice vbox[VCAP], and each lane then
// gathers its 27 nodes from shared memory. A box larger than VCAP, or lanes
// whose stencil leaves the grid, take the global gather. Called by the whole
// warp (the box, the loads and __syncwarp are warp-wide).
template <int VCAP>
__device__ __forceinline__ void g2p_gather_staged(const DevParams& P, const float4* __restrict__ vel,
                                                  float4* __restrict__ vbox, bool part, bool active,
                                                  const int base[3], const float fx[3], float v[3], float C[3][3],
                                                  int lane, WxSlot wx) {
    const int lo0 = __reduce_min_sync(0xffffffffu, part ? base[0] : INT_MAX);
    const int lo1 = __reduce_min_sync(0xffffffffu, part ? base[1] : INT_MAX);
    const int lo2 = __reduce_min_sync(0xffffffffu, part ? base[2] : INT_MAX);
    const int hi0 = __reduce_max_sync(0xffffffffu, part ? base[0] : INT_MIN);
    const int hi1 = __reduce_max_sync(0xffffffffu, part ? base[1] : INT_MIN);
    const int hi2 = __reduce_max_sync(0xffffffffu, part ? base[2] : INT_MIN);
    int ey = 0, ez = 0;
    bool staged = false;
    if (lo0 <= hi0) {
        const int ex = hi0 - lo0 + 3;
        ey = hi1 - lo1 + 3;
        ez = hi2 - lo2 + 3;
        staged = (long long)ex * ey * ez <= VCAP;
        if (staged) {
            const int vol = ex * ey * ez;
            const int slab = (int)P.slab, gz = P.Gz;
            const int g0 = ((lo0 + P.halo) * P.Gy + lo1) * gz + lo2;
            const float inv_ez = 1.0f / (float)ez, inv_ey = 1.0f / (float)ey;
            for (int k = lane; k < vol; k += 32) {
                const int row = (int)(((float)k + 0.5f) * inv_ez);   // k / ez (k, ez <= VCAP)
                const int tz = k - row * ez;
                const int tx = (int)(((float)row + 0.5f) * inv_ey);
                const int ty = row - tx * ey;
                // global -> shared without a round trip through registers: the
                // lane issues all its copies before it waits for any of them
                const unsigned dst = (unsigned)__cvta_generic_to_shared(vbox + k);
                asm volatile("cp.async.ca.shared.global [%0], [%1], 16;"
                             :: "r"(dst), "l"(vel + (g0 + tx * slab + ty * gz + tz)) : "memory");
            }
            asm volatile("cp.async.wait_all;" ::: "memory");
            __syncwarp();
        }
    }
    if (part && staged) {
        // v = sum w nv and the first moments M_k = sum w nv o_k over the node
        // offsets o = (a, b, c); C = 4/h sum w nv (o - f) = 4/h (M - f v)
        // (mpm_kernels.cuh:278-305). The weights factor, w = wx_a wy_b wz_c, so
        // each stencil row first sums T = sum_c wz_c nv and Z = sum_c c wz_c nv.
        float ww[3][3];
        quad_weights<float>(fx, ww);
        wx.put(ww);
        float Mx[3], My[3], Mz[3];
#pragma unroll
        for (int r = 0; r < 3; r++) { v[r] = 0.f; Mx[r] = 0.f; My[r] = 0.f; Mz[r] = 0.f; }
        const int t0 = ((base[0] - lo0) * ey + (base[1] - lo1)) * ez + (base[2] - lo2);
        const float wz0 = ww[0][2], wz1 = ww[1][2], wz2 = ww[2][2], wz2d = 2.0f * ww[2][2];
#pragma unroll 1
        for (int a = 0; a < 3; a++) {
            const float wa = wx.get(a);
            float ra[3];
#pragma unroll
            for (int b = 0; b < 3; b++) {
                const float wab = wa * ww[b][1];
                const float bwab = (float)b * wab;
                const float4* row = vbox + (t0 + a * ey * ez + b * ez);
                float T[3], Z[3];
                {
                    const float4 nd = row[0];
                    T[0] = wz0 * nd.x; T[1] = wz0 * nd.y; T[2] = wz0 * nd.z;
                }
                {
                    const float4 nd = row[1];
                    T[0] = fmaf(wz1, nd.x, T[0]); T[1] = fmaf(wz1, nd.y, T[1]); T[2] = fmaf(wz1, nd.z, T[2]);
                    Z[0] = wz1 * nd.x; Z[1] = wz1 * nd.y; Z[2] = wz1 * nd.z;
                }
                {
                    const float4 nd = row[2];
                    T[0] = fmaf(wz2, nd.x, T[0]); T[1] = fmaf(wz2, nd.y, T[1]); T[2] = fmaf(wz2, nd.z, T[2]);
                    Z[0] = fmaf(wz2d, nd.x, Z[0]); Z[1] = fmaf(wz2d, nd.y, Z[1]); Z[2] = fmaf(wz2d, nd.z, Z[2]);
                }
#pragma unroll
                for (int r = 0; r < 3; r++) {
                    ra[r] = b == 0 ? wab * T[r] : fmaf(wab, T[r], ra[r]);
                    if (b > 0) My[r] = fmaf(bwab, T[r], My[r]);
                    Mz[r] = fmaf(wab, Z[r], Mz[r]);
                }
            }
            const float fa = (float)a;
#pragma unroll
            for (int r = 0; r < 3; r++) {
                v[r] += ra[r];
                Mx[r] = fmaf(fa, ra[r], Mx[r]);
            }
        }
        const float s4 = P.f_s4;
#pragma unroll
        for (int r = 0; r < 3; r++) {
            C[r][0] = s4 * (Mx[r] - fx[0] * v[r]);
            C[r][1] = s4 * (My[r] - fx[1] * v[r]);
            C[r][2] = s4 * (Mz[r] - fx[2] * v[r]);
        }
    } else if (active) {
        g2p_gather_mixed(P, vel, base, fx, v, C, !part, wx);
    }
    __syncwarp();
}

// Return map of a crushed point in FP64 (mpm_kernels.cuh:486-544). Out of
// line (it is rare and register-hungry); arguments and result travel by
// value so that nothing of the caller is forced into local memory.
struct ElasticState {
    float e[9];   // F - I, row-major
    float jp;     // Jp_inv - 1
};

__device__ __noinline__ ElasticState return_map_f64(const DPParams P, const ElasticState in, const double p0) {
    double F[3][3];
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) F[i][j] = (i == j ? 1.0 : 0.0) + (double)in.e[3 * i + j];
    double Je, p_tr, q_tr;
    trial_pq(P, F, Je, p_tr, q_tr);
    double jp = 1.0 + (double)in.jp;
    drucker_prager_return<SvdF64>(P, F, jp, Je, p_tr, q_tr, p0);
    ElasticState out;
    out.jp = (float)(jp - 1.0);
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) out.e[3 * i + j] = (float)(F[i][j] - (i == j ? 1.0 : 0.0));
    return out;
}

// ------------------------------------------------------------- P2G part

// The grid accumulator of the mixed P2G (and of the halo exchange):
//   AccF4: float4 {m, m v} per node, added with FP32 vector atomics (the
//          default): the sum's rounding depends on the order of the adds;
//   AccQ:  4 int64 per node, each contribution converted to fixed point with
//          the per-quantity scales q_m = 2^44 / m_ref and q_p = 2^44 /
//          (m_ref vmax) (m_ref = the larger particle mass) and added as an
//          integer: the sum is exact and independent of the order, so a run
//          repeats bit for bit. Resolution 2^-44 m_ref in mass and
//          2^-44 m_ref vmax in momentum; a node holds 2^19 such full-scale
//          contributions before the 2^63 range (each conversion saturates).
struct AccF4 {
    float4* a;
    __device__ __forceinline__ void add(const DevParams&, int node, float m, float x, float y, float z) const {
        atomicAdd(a + node, make_float4(m, x, y, z));
    }
};
struct AccQ {
    unsigned long long* a;   // 4 per node: m, m vx, m vy, m vz in units of 1 / scale
    __device__ __forceinline__ static unsigned long long q(float v, float scale) {
        const float t = fminf(fmaxf(v * scale, -4.0e18f), 4.0e18f);
        return (unsigned long long)__float2ll_rn(t);
    }
    __device__ __forceinline__ void add(const DevParams& P, int node, float m, float x, float y, float z) const {
        unsigned long long* p = a + 4 * (size_t)node;
        atomicAdd(p + 0, q(m, P.f_qm));
        atomicAdd(p + 1, q(x, P.f_qp));
        atomicAdd(p + 2, q(y, P.f_qp));
        atomicAdd(p + 3, q(z, P.f_qp));
    }
};

// Scatter of one particle (base, fx, m, mv, S): float4 {m, mv} atomics per
// node, no merging (the return map's list of crushed points, whose lanes
// rarely share a cell). Out-of-grid nodes of a lane that is not inside are
// skipped.
template <class Acc>
__device__ __forceinline__ void p2g_scatter_mixed(const DevParams& P, Acc acc, bool active, bool inside,
                                                  const int base[3], const float fx[3], float mass, const float mv[3],
                                                  const float S[3][3]) {
    const int i0 = ((base[0] + P.halo) * P.Gy + base[1]) * P.Gz + base[2];
    float ww[3][3];
    quad_weights<float>(fx, ww);
    const float h = P.f_h;
    const int slab = (int)P.slab, gz = P.Gz;
#pragma unroll 1
    for (int a = 0; a < 3; a++) {
        const float dx = (a - fx[0]) * h;
#pragma unroll
        for (int b = 0; b < 3; b++) {
            const float dy = (b - fx[1]) * h;
            const float wab = pick3(a, ww[0][0], ww[1][0], ww[2][0]) * ww[b][1];
            const int ib = i0 + a * slab + b * gz;
            float part[3];
#pragma unroll
            for (int m = 0; m < 3; m++) part[m] = mv[m] + S[m][0] * dx + S[m][1] * dy;
#pragma unroll
            for (int c = 0; c < 3; c++) {
                const float dz = (c - fx[2]) * h;
                const float W = wab * ww[c][2];
                float val[4] = {W * mass, W * (part[0] + S[0][2] * dz), W * (part[1] + S[1][2] * dz),
                                W * (part[2] + S[2][2] * dz)};
                if (!active) continue;
                if (!inside && !node_inside(P, base[0] + a, base[1] + b, base[2] + c)) continue;
                acc.add(P, ib + c, val[0], val[1], val[2], val[3]);
            }
        }
    }
}

// Scatter with pairs of particles that share a base cell merged in
// registers: in cell-sorted order they sit in neighbouring lanes, so one
// shuffle round per node moves the odd-ranked partner's four values to the
// even-ranked lane, which issues the single float4 atomic for both. A third
// particle of a cell (rank 2) pairs with a fourth or adds alone. Halves the
// atomic traffic to L2 at ppc ~2 for 8 shuffles and adds per node.
template <class Acc>
__device__ __forceinline__ void p2g_scatter_pairs(const DevParams& P, Acc acc, bool active,
                                                  bool inside, const int base[3], const float fx[3], float mass,
                                                  const float mv[3], const float S[3][3], int lane, WxSlot wx) {
    const int i0 = ((base[0] + P.halo) * P.Gy + base[1]) * P.Gz + base[2];
    const int key = (active && inside) ? i0 : -1 - lane;
    const unsigned peers = __match_any_sync(0xffffffffu, key);
    const int rank = __popc(peers & ((1u << lane) - 1u));
    const int next_key = __shfl_down_sync(0xffffffffu, key, 1);
    const bool absorb = lane < 31 && next_key == key && (rank & 1) == 0;
    const bool absorbed = __shfl_up_sync(0xffffffffu, (int)absorb, 1) != 0 && lane > 0;
    float ww[3][3];
    quad_weights<float>(fx, ww);
    wx.put(ww);
    const bool emit = active && !absorbed;
    if (__all_sync(0xffffffffu, inside || !active)) {
        // every stencil of the warp lies in the grid: no per-node checks
        const float h = P.f_h;
        const int slab = (int)P.slab, gz = P.Gz;
#pragma unroll 1
        for (int a = 0; a < 3; a++) {
            const float dx = (a - fx[0]) * h;
            const float wa = wx.get(a);
#pragma unroll
            for (int b = 0; b < 3; b++) {
                const float dy = (b - fx[1]) * h;
                const float wab = wa * ww[b][1];
                const int ib = i0 + a * slab + b * gz;
                float part[3];
#pragma unroll
                for (int m = 0; m < 3; m++) part[m] = mv[m] + S[m][0] * dx + S[m][1] * dy;
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    const float dz = (c - fx[2]) * h;
                    const float W = wab * ww[c][2];
                    float val[4] = {W * mass, W * (part[0] + S[0][2] * dz), W * (part[1] + S[1][2] * dz),
                                    W * (part[2] + S[2][2] * dz)};
#pragma unroll
                    for (int q = 0; q < 4; q++) {
                        const float o = __shfl_down_sync(0xffffffffu, val[q], 1);
                        if (absorb) val[q] += o;
                    }
                    if (emit) acc.add(P, ib + c, val[0], val[1], val[2], val[3]);
                }
            }
        }
        return;
    }
    const float h = P.f_h;
    const int slab = (int)P.slab, gz = P.Gz;
#pragma unroll 1
    for (int a = 0; a < 3; a++) {
        const float dx = (a - fx[0]) * h;
        const float wa = wx.get(a);
#pragma unroll
        for (int b = 0; b < 3; b++) {
            const float dy = (b - fx[1]) * h;
            const float wab = wa * ww[b][1];
            const int ib = i0 + a * slab + b * gz;
            float part[3];
#pragma unroll
            for (int m = 0; m < 3; m++) part[m] = mv[m] + S[m][0] * dx + S[m][1] * dy;
#pragma unroll
            for (int c = 0; c < 3; c++) {
                const float dz = (c - fx[2]) * h;
                const float W = wab * ww[c][2];
                float val[4] = {W * mass, W * (part[0] + S[0][2] * dz), W * (part[1] + S[1][2] * dz),
                                W * (part[2] + S[2][2] * dz)};
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    const float o = __shfl_down_sync(0xffffffffu, val[q], 1);
                    if (absorb) val[q] += o;
                }
                if (!active || absorbed) continue;
                if (!inside && !node_inside(P, base[0] + a, base[1] + b, base[2] + c)) continue;
                acc.add(P, ib + c, val[0], val[1], val[2], val[3]);
            }
        }
    }
}

// P2G payload of a particle: S = m C - dt V Dp^-1 tau (mpm_kernels.cuh:63)
__device__ __forceinline__ void p2g_payload_mixed(const DevParams& P, const float E[3][3], const float C[3][3],
                                                  const float v[3], bool liquid, float Jpm1, float& mass, float mv[3],
                                                  float S[3][3]) {
    mass = liquid ? P.f_lmass : P.f_pmass;
    float tau[3][3];
    if (liquid) {
        // kappa (1 - J^-3) with J = 1 + d: (J^3 - 1) / J^3 = d (3 + 3d + d^2) / J^3, free of cancellation
        const float J = 1.0f + Jpm1;
        const float pw = P.f_kappa * (Jpm1 * (3.0f + Jpm1 * (3.0f + Jpm1)) / (J * J * J));
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = 0; j < 3; j++) tau[i][j] = (i == j) ? pw : 0.f;
    } else {
        kirchhoff_mixed(P, E, tau);
    }
    const float dvd = P.f_dvd;
#pragma unroll
    for (int i = 0; i < 3; i++) {
        mv[i] = v[i] * mass;
#pragma unroll
        for (int j = 0; j < 3; j++) S[i][j] = mass * C[i][j] - dvd * tau[i][j];
    }
}

__device__ __forceinline__ void load_mixed(const MixedState& s, int i, int X[3], float E[3][3], float& Jpm1, int& st) {
#pragma unroll
    for (int d = 0; d < 3; d++) X[d] = s.X[d * s.pitch + i];
#pragma unroll
    for (int r = 0; r < 3; r++)
#pragma unroll
        for (int c = 0; c < 3; c++) E[r][c] = s.E[(3 * r + c) * s.pitch + i];
    Jpm1 = s.Jpm1[i];
    st = s.status[i];
}

// Standalone P2G from the stored state (first step, phase API), with the
// fused kernel's same-cell pair merge (128-thread blocks: the x-weight slots).
// 8 M block: 0.47 ms against 1.24 ms for a general warp-group reduction.
template <class Acc>
__global__ void __launch_bounds__(128) k_p2g_mixed(DevParams P, MixedState s, int n, Acc acc,
                                                   int* err) {
    __shared__ float wx_slots[3 * 128];
    const WxSlot wx{wx_slots + threadIdx.x};
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31;
    bool active = i < n;
    int X[3] = {0, 0, 0}, st = (int)kDisabled;
    float E[3][3], Jpm1 = 0.f;
    if (active) load_mixed(s, i, X, E, Jpm1, st);
    active = active && !(st & (int)kDisabled);
    int base[3];
    float fx[3], mass = 0.f, mv[3] = {0, 0, 0}, S[3][3];
#pragma unroll
    for (int d = 0; d < 3; d++) fix_base(X[d], base[d], fx[d]);
    bool inside = false;
    if (active) {
        float v[3], C[3][3];
#pragma unroll
        for (int d = 0; d < 3; d++) v[d] = s.v[d * s.pitch + i];
#pragma unroll
        for (int r = 0; r < 3; r++)
#pragma unroll
            for (int c = 0; c < 3; c++) C[r][c] = s.C[(3 * r + c) * s.pitch + i];
        p2g_payload_mixed(P, E, C, v, (st & (int)kLiquid) != 0, Jpm1, mass, mv, S);
        const int e = stencil_error(P, base[0], base[1], base[2]);
        if (e) raise_error(err, e);
        inside = e == 0;
    } else {
#pragma unroll
        for (int r = 0; r < 3; r++)
#pragma unroll
            for (int c = 0; c < 3; c++) S[r][c] = 0.f;
    }
    p2g_scatter_pairs(P, acc, active, inside, base, fx, mass, mv, S, lane, wx);
}

// G2P tail of the fused kernels for one particle (whole warp): fixed-point
// advection, E <- E + dt C (I + E), trial p and q, the failure test, the P/Q
// record; a newly crushed point is appended to rm_list (its return map and
// P2G run in k_return_map_mixed) and returns true. Stores X and E; v and C
// only when store_vc or crushed (the next G2P recomputes them from the grid);
// Jp_inv and status only when they changed.
__device__ __forceinline__ bool fused_update_state(const DevParams& P, const MixedState& s, int i, bool active,
                                                   int X[3], int& st, int st_in, float jpm1_in, float E[3][3],
                                                   float& Jpm1, const float v[3], const float C[3][3],
                                                   ElasticInv& inv, int record_pq, int store_vc,
                                                   int* __restrict__ rm_list, int* __restrict__ rm_count, int lane) {
    bool need_rm = false;
    if (active) {
        const float dt = P.f_dt;
        const float adv = P.f_adv;
#pragma unroll
        for (int d = 0; d < 3; d++) X[d] += __float2int_rn(v[d] * adv);
        float En[3][3];
#pragma unroll
        for (int r = 0; r < 3; r++)
#pragma unroll
            for (int c = 0; c < 3; c++)
                En[r][c] = E[r][c] + dt * (C[r][c] + (C[r][0] * E[0][c] + C[r][1] * E[1][c] + C[r][2] * E[2][c]));
        float p_tr = 0.f, q_tr = 0.f;
        if (st & (int)kLiquid) {
            float A[3][3];
#pragma unroll
            for (int r = 0; r < 3; r++)
#pragma unroll
                for (int c = 0; c < 3; c++) A[r][c] = dt * C[r][c];
            const float dA = detm1(A);   // det(I + dt C) - 1
            Jpm1 = Jpm1 + dA + Jpm1 * dA;     // Jp_inv <- Jp_inv det(I + dt C), as Jp_inv - 1
#pragma unroll
            for (int r = 0; r < 3; r++)
#pragma unroll
                for (int c = 0; c < 3; c++) E[r][c] = En[r][c];
        } else {
#pragma unroll
            for (int r = 0; r < 3; r++)
#pragma unroll
                for (int c = 0; c < 3; c++) E[r][c] = En[r][c];
            inv = elastic_invariants(E);
            trial_pq_inv(P, inv, p_tr, q_tr);
            if (!(st & (int)kCrushed) && outside_failure_surface_f32(P, (short)st, p_tr, q_tr)) st |= (int)kCrushed;
            need_rm = (st & (int)kCrushed) != 0;
        }
        if (record_pq) {
            s.PQ[i] = p_tr;
            s.PQ[s.pitch + i] = q_tr;
        }
    }
    const unsigned rm_mask = __ballot_sync(0xffffffffu, need_rm);
    if (rm_mask) {
        const int first = __ffs(rm_mask) - 1;
        int slot0 = 0;
        if (lane == first) slot0 = atomicAdd(rm_count, __popc(rm_mask));
        slot0 = __shfl_sync(0xffffffffu, slot0, first);
        if (need_rm) rm_list[slot0 + __popc(rm_mask & ((1u << lane) - 1u))] = i;
    }
    if (active) {
#pragma unroll
        for (int d = 0; d < 3; d++) s.X[d * s.pitch + i] = X[d];
#pragma unroll
        for (int r = 0; r < 3; r++)
#pragma unroll
            for (int c = 0; c < 3; c++) s.E[(3 * r + c) * s.pitch + i] = E[r][c];
        if (store_vc || need_rm) {
#pragma unroll
            for (int d = 0; d < 3; d++) s.v[d * s.pitch + i] = v[d];
#pragma unroll
            for (int r = 0; r < 3; r++)
#pragma unroll
                for (int c = 0; c < 3; c++) s.C[(3 * r + c) * s.pitch + i] = C[r][c];
        }
        if (__float_as_int(Jpm1) != __float_as_int(jpm1_in)) s.Jpm1[i] = Jpm1;
        if (st != st_in) s.status[i] = st;
    }
    return need_rm;
}

// P2G payload of the fused kernels (S = m C - dt V Dp^-1 tau, mpm_kernels.cuh:63)
// at the advected position; inactive lanes get a zero payload.
__device__ __forceinline__ void fused_payload(const DevParams& P, bool active, const int X[3], int st,
                                              const float E[3][3], const float C[3][3], const float v[3], float Jpm1,
                                              const ElasticInv& inv, int base[3], float fx[3], float& mass,
                                              float mv[3], float S[3][3], bool& inside, int* err) {
    mass = 0.f;
    inside = false;
    if (active) {
#pragma unroll
        for (int d = 0; d < 3; d++) fix_base(X[d], base[d], fx[d]);
        if (st & (int)kLiquid) {
            p2g_payload_mixed(P, E, C, v, true, Jpm1, mass, mv, S);
        } else {
            mass = P.f_pmass;
            float tau[3][3];
            tau_inv(P, inv, tau);
            const float dvd = P.f_dvd;
#pragma unroll
            for (int r = 0; r < 3; r++) {
                mv[r] = v[r] * mass;
#pragma unroll
                for (int c = 0; c < 3; c++) S[r][c] = mass * C[r][c] - dvd * tau[r][c];
            }
        }
        const int e = stencil_error(P, base[0], base[1], base[2]);
        if (e) raise_error(err, e);
        inside = e == 0;
    } else {
#pragma unroll
        for (int d = 0; d < 3; d++) { base[d] = 0; fx[d] = 1.0f; mv[d] = 0.f; }
#pragma unroll
        for (int r = 0; r < 3; r++)
#pragma unroll
            for (int c = 0; c < 3; c++) S[r][c] = 0.f;
    }
}

// Fused G2P (this step) -> P2G (next step) of particle i (whole warp; lanes
// past n or disabled are inactive). do_p2g = 0 gives a plain G2P. The gather
// reads the warp's velocity box staged in shared memory by the warp's own
// coalesced loads (vbox: kVBoxNodes float4 of this warp); the scatter adds
// float4 atomics with same-cell particle pairs merged in registers.
constexpr int kVBoxNodes = 256;
template <class Acc>
__device__ __forceinline__ void fused_particle(const DevParams& P, const MixedState& s, int i, int n,
                                               const float4* __restrict__ vel, Acc acc,
                                               int do_p2g, int record_pq, int store_vc, int* err,
                                               int* __restrict__ rm_list, int* __restrict__ rm_count,
                                               float4* __restrict__ vbox, WxSlot wx, int lane) {
    bool active = i < n;
    int X[3] = {0, 0, 0}, st = (int)kDisabled;
    float E[3][3], Jpm1 = 0.f;
    // positions and status first: the gather box depends on them
    if (active) {
        st = s.status[i];
#pragma unroll
        for (int d = 0; d < 3; d++) X[d] = s.X[d * s.pitch + i];
    }
    active = active && !(st & (int)kDisabled);

    int base[3] = {0, 0, 0};
    float fx[3] = {1.f, 1.f, 1.f}, v[3] = {0, 0, 0}, C[3][3];
    bool inside = false;
    ElasticInv inv;
    int e0 = 0;
    if (active) {
#pragma unroll
        for (int d = 0; d < 3; d++) fix_base(X[d], base[d], fx[d]);
        e0 = stencil_error(P, base[0], base[1], base[2]);
        if (e0) raise_error(err, e0);
    }
    if (active) {
#pragma unroll
        for (int r = 0; r < 3; r++)
#pragma unroll
            for (int c = 0; c < 3; c++) E[r][c] = s.E[(3 * r + c) * s.pitch + i];
        Jpm1 = s.Jpm1[i];
    }
    const int st_in = st;
    const float jpm1_in = Jpm1;
    g2p_gather_staged<kVBoxNodes>(P, vel, vbox, active && e0 == 0, active, base, fx, v, C, lane, wx);
    const bool need_rm = fused_update_state(P, s, i, active, X, st, st_in, jpm1_in, E, Jpm1, v, C, inv, record_pq,
                                            store_vc, rm_list, rm_count, lane);
    active = active && !need_rm;   // crushed points scatter in k_return_map_mixed
    if (!do_p2g) return;   // uniform across the launch
    float mass, mv[3], S[3][3];
    fused_payload(P, active, X, st, E, C, v, Jpm1, inv, base, fx, mass, mv, S, inside, err);
    p2g_scatter_pairs(P, acc, active, inside, base, fx, mass, mv, S, lane, wx);
}

// The fused kernel: 64-thread blocks at 16 per SM (64 registers, 32 warps
// per SM), kVBoxNodes float4 of dynamic shared memory per warp. Measured on
// the 8 M block: 0.598 ms per launch against 0.627 ms with 128-thread blocks
// at 8 per SM (a finished warp's slot frees sooner), 0.602 ms with 32-thread
// blocks; a persistent grid of warps looping over 32-particle chunks (static
// or counter-scheduled) spills at 64 registers and takes 0.79-0.92 ms.
constexpr int kFusedBlock = 64;
template <class Acc>
__global__ void __launch_bounds__(kFusedBlock, 1024 / kFusedBlock) k_g2p2g_mixed(
    DevParams P, MixedState s, int n, const float4* __restrict__ vel, Acc acc, int do_p2g,
    int record_pq, int store_vc, int* err, int* __restrict__ rm_list, int* __restrict__ rm_count) {
    extern __shared__ __align__(128) float mixed_tile[];
    __shared__ float wx_slots[3 * 128];
    const WxSlot wx{wx_slots + threadIdx.x};
    const int lane = threadIdx.x & 31;
    float4* vbox = reinterpret_cast<float4*>(mixed_tile) + (threadIdx.x >> 5) * kVBoxNodes;
    fused_particle(P, s, blockIdx.x * kFusedBlock + threadIdx.x, n, vel, acc, do_p2g, record_pq, store_vc, err,
                   rm_list, rm_count, vbox, wx, lane);
}

// Return map (FP64, mpm_kernels.cuh:486-544) of the crushed points listed by
// k_g2p2g_mixed, then their P2G (direct float4 atomics) when do_p2g. The
// list holds *count indices; the kernel also clears next_count, the counter
// the next fused launch appends to. Grid-stride over the list.
template <class Acc>
__global__ void __launch_bounds__(128) k_return_map_mixed(DevParams P, MixedState s, const int* __restrict__ rm_list,
                                                          const int* __restrict__ count, int* __restrict__ next_count,
                                                          Acc acc, int do_p2g, int* err) {
    if (blockIdx.x == 0 && threadIdx.x == 0) *next_count = 0;
    const int m = *count;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < m; k += gridDim.x * blockDim.x) {
        const int i = rm_list[k];
        int X[3], st;
        float E[3][3], Jpm1;
        load_mixed(s, i, X, E, Jpm1, st);
        const double p0 = s.p0 ? (double)s.p0[i] : P.p0;
        ElasticState es;
#pragma unroll
        for (int q = 0; q < 9; q++) es.e[q] = E[q / 3][q % 3];
        es.jp = Jpm1;
        es = return_map_f64(dp_params(P), es, p0);
#pragma unroll
        for (int q = 0; q < 9; q++) {
            E[q / 3][q % 3] = es.e[q];
            s.E[q * s.pitch + i] = es.e[q];
        }
        if (__float_as_int(es.jp) != __float_as_int(Jpm1)) s.Jpm1[i] = es.jp;
        if (!do_p2g) continue;
        float v[3], C[3][3], mass, mv[3], S[3][3], fx[3];
        int base[3];
#pragma unroll
        for (int d = 0; d < 3; d++) v[d] = s.v[d * s.pitch + i];
#pragma unroll
        for (int q = 0; q < 9; q++) C[q / 3][q % 3] = s.C[q * s.pitch + i];
#pragma unroll
        for (int d = 0; d < 3; d++) fix_base(X[d], base[d], fx[d]);
        p2g_payload_mixed(P, E, C, v, false, es.jp, mass, mv, S);
        const int e = stencil_error(P, base[0], base[1], base[2]);
        if (e) raise_error(err, e);
        p2g_scatter_mixed(P, acc, true, e == 0, base, fx, mass, mv, S);
    }
}

// Node update for the mixed grid: FP64 arithmetic on the FP32 sums (one
// reciprocal of the mass), contact force in FP64 (sensor and per-substep
// total), velocities written as float4, the accumulator cleared for the next
// P2G. Node coordinates by reciprocal multiplication (no integer division).
// The node's sums {m, m vx, m vy, m vz} as loaded, in double, and the
// accumulator cleared for the next P2G (when the node has mass).
struct NodeF4 { float4 a; };
__device__ __forceinline__ NodeF4 load_node(AccF4 acc, int idx) { return {acc.a[idx]}; }
__device__ __forceinline__ void node_sums(const NodeF4& r, const DevParams&, double& m, double mv[3]) {
    m = r.a.x; mv[0] = r.a.y; mv[1] = r.a.z; mv[2] = r.a.w;
}
__device__ __forceinline__ void clear_node(AccF4 acc, int idx) { acc.a[idx] = make_float4(0.f, 0.f, 0.f, 0.f); }
struct NodeQ { ulonglong2 q0, q1; };
__device__ __forceinline__ NodeQ load_node(AccQ acc, int idx) {
    const ulonglong2* p = reinterpret_cast<const ulonglong2*>(acc.a + 4 * (size_t)idx);
    return {p[0], p[1]};
}
__device__ __forceinline__ void node_sums(const NodeQ& r, const DevParams& P, double& m, double mv[3]) {
    m = (double)(long long)r.q0.x * P.q_inv_m;
    mv[0] = (double)(long long)r.q0.y * P.q_inv_p;
    mv[1] = (double)(long long)r.q1.x * P.q_inv_p;
    mv[2] = (double)(long long)r.q1.y * P.q_inv_p;
}
__device__ __forceinline__ void clear_node(AccQ acc, int idx) {
    ulonglong2* p = reinterpret_cast<ulonglong2*>(acc.a + 4 * (size_t)idx);
    p[0] = make_ulonglong2(0ull, 0ull);
    p[1] = make_ulonglong2(0ull, 0ull);
}

// One node with mass: velocity, gravity, indenter contact (force into f and
// the sensor), walls; writes vel[idx].
__device__ __forceinline__ void update_node(const DevParams& P, int idx, double mass, const double amv[3],
                                            float4* __restrict__ vel, double ind_x, double ind_y,
                                            double* __restrict__ sensor, double f[3]) {
    int idx_z, idx_y;
    const int col = div_by(idx, P.Gz, P.inv_gz, idx_z);
    const int idx_x = div_by(col, P.Gy, P.inv_gy, idx_y);
    const int gx = idx_x - P.halo, gy = idx_y, gz = idx_z;
    const double inv_m = 1.0 / mass;
    double v[3] = {amv[0] * inv_m, amv[1] * inv_m, amv[2] * inv_m};
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
    vel[idx] = make_float4((float)v[0], (float)v[1], (float)v[2], 0.f);
}

// NPT nodes per thread, BLOCK apart: both loads are in flight before the
// first is used (8 M block: 0.049 ms per update against 0.059 ms with one
// node per thread; four per thread need 80 registers and gain nothing more).
constexpr int kUpdateNodesPerThread = 2;
template <int BLOCK, class Acc, int NPT = kUpdateNodesPerThread>
__global__ void __launch_bounds__(BLOCK) k_update_mixed(DevParams P, Acc acc, float4* __restrict__ vel,
                                                        double ind_x, double ind_y, double* __restrict__ sensor,
                                                        double* __restrict__ force3) {
    const int idx0 = P.node_lo + blockIdx.x * (BLOCK * NPT) + threadIdx.x;   // the handle keeps nodes < 2^31
    double f[3] = {0, 0, 0};
    decltype(load_node(acc, 0)) r[NPT];
#pragma unroll
    for (int j = 0; j < NPT; j++) {
        const int idx = idx0 + j * BLOCK;
        if (idx < P.node_hi) r[j] = load_node(acc, idx);
    }
#pragma unroll
    for (int j = 0; j < NPT; j++) {
        const int idx = idx0 + j * BLOCK;
        if (idx < P.node_hi) {
            double mass, amv[3];
            node_sums(r[j], P, mass, amv);
            if (mass != 0) {
                clear_node(acc, idx);
                update_node(P, idx, mass, amv, vel, ind_x, ind_y, sensor, f);
            }
        }
    }
    __shared__ double red[3][BLOCK / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const bool any = (f[0] != 0) | (f[1] != 0) | (f[2] != 0);
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

// ------------------------------------------- conversion from / to FP64 SoA

__global__ void k_mixed_from_f64(const double* __restrict__ src, size_t spitch, int n, MixedState s, double h_inv) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
#pragma unroll
    for (int d = 0; d < 3; d++) {
        s.X[d * s.pitch + i] = __double2int_rn(src[(MPM_POSX + d) * spitch + i] * h_inv * (double)(1 << kFixBits));
        s.v[d * s.pitch + i] = (float)src[(MPM_VELX + d) * spitch + i];
    }
#pragma unroll
    for (int r = 0; r < 3; r++)
#pragma unroll
        for (int c = 0; c < 3; c++) {
            s.E[(3 * r + c) * s.pitch + i] = (float)(src[(MPM_FE00 + 3 * r + c) * spitch + i] - (r == c ? 1.0 : 0.0));
            s.C[(3 * r + c) * s.pitch + i] = (float)src[(MPM_BP00 + 3 * r + c) * spitch + i];
        }
    s.Jpm1[i] = (float)(src[MPM_IDX_JP_INV * spitch + i] - 1.0);
    s.status[i] = (int)__double_as_longlong(src[i]);
    s.PQ[i] = (float)src[MPM_IDX_P * spitch + i];
    s.PQ[s.pitch + i] = (float)src[MPM_IDX_Q * spitch + i];
}

// The upper 32 bits of the utility word are kept from the uploaded copy
// (the step only changes the low status bits).
__global__ void k_mixed_to_f64(MixedState s, int n, double* __restrict__ dst, size_t dpitch, double h) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
#pragma unroll
    for (int d = 0; d < 3; d++) {
        dst[(MPM_POSX + d) * dpitch + i] = (double)s.X[d * s.pitch + i] * (1.0 / (double)(1 << kFixBits)) * h;
        dst[(MPM_VELX + d) * dpitch + i] = (double)s.v[d * s.pitch + i];
    }
#pragma unroll
    for (int r = 0; r < 3; r++)
#pragma unroll
        for (int c = 0; c < 3; c++) {
            dst[(MPM_FE00 + 3 * r + c) * dpitch + i] = (double)s.E[(3 * r + c) * s.pitch + i] + (r == c ? 1.0 : 0.0);
            dst[(MPM_BP00 + 3 * r + c) * dpitch + i] = (double)s.C[(3 * r + c) * s.pitch + i];
        }
    dst[MPM_IDX_JP_INV * dpitch + i] = 1.0 + (double)s.Jpm1[i];
    const long long hi = __double_as_longlong(dst[i]) & (long long)0xffffffff00000000LL;
    dst[i] = __longlong_as_double(hi | (long long)(unsigned)s.status[i]);
    dst[MPM_IDX_P * dpitch + i] = (double)s.PQ[i];
    dst[MPM_IDX_Q * dpitch + i] = (double)s.PQ[s.pitch + i];
}

}  // namespace icempm
