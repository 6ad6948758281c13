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

// dev(F F^T) with F = I + E: dev(E + E^T + E E^T)
__device__ __forceinline__ void dev_b(const float E[3][3], float D[3][3]) {
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++)
            D[i][j] = E[i][j] + E[j][i] + (E[i][0] * E[j][0] + E[i][1] * E[j][1] + E[i][2] * E[j][2]);
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
    p_tr = -(float)(0.5 * P.kappa) * (e.jm1 * (e.J + 1.0f));
    float sq = 0.f;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) sq += e.D[i][j] * e.D[i][j];
    q_tr = (float)(kCoeff1 * P.mu) * e.jm23 * sqrtf(sq);
}

__device__ __forceinline__ void tau_inv(const DevParams& P, const ElasticInv& e, float tau[3][3]) {
    const float s = (float)P.mu * e.jm23;
    const float hyd = (float)(P.kappa * 0.5) * (e.jm1 * (e.J + 1.0f));
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
    const float s = (float)P.mu * exp2f(-(2.0f / 3.0f) * log2f(J));
    const float hyd = (float)(P.kappa * 0.5) * (jm1 * (J + 1.0f));
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
    p_tr = -(float)(0.5 * P.kappa) * (jm1 * (J + 1.0f));
    float D[3][3];
    dev_b(E, D);
    float sq = 0.f;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) sq += D[i][j] * D[i][j];
    q_tr = (float)(kCoeff1 * P.mu) * exp2f(-(2.0f / 3.0f) * log2f(J)) * sqrtf(sq);
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
    const float s4 = 4.0f * (float)P.h_inv;
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
// nodes (base .. base+2 per axis) are read from the grid once, row by row
// along z (coalesced), into this warp's slice vbox[VCAP], and each lane then
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
                vbox[k] = __ldg(vel + (g0 + tx * slab + ty * gz + tz));
            }
            __syncwarp();
        }
    }
    if (part && staged) {
        // v = sum w nv and the first moments M_k = sum w nv o_k over the node
        // offsets o = (a, b, c); C = 4/h sum w nv (o - f) = 4/h (M - f v)
        // (mpm_kernels.cuh:278-305 summed in this order).
        float ww[3][3];
        quad_weights<float>(fx, ww);
        wx.put(ww);
        float Mx[3], My[3], Mz[3];
#pragma unroll
        for (int r = 0; r < 3; r++) { v[r] = 0.f; Mx[r] = 0.f; My[r] = 0.f; Mz[r] = 0.f; }
        const int t0 = ((base[0] - lo0) * ey + (base[1] - lo1)) * ez + (base[2] - lo2);
#pragma unroll 1
        for (int a = 0; a < 3; a++) {
            const float wa = wx.get(a);
            float ra[3] = {0.f, 0.f, 0.f};
#pragma unroll
            for (int b = 0; b < 3; b++) {
                const float wab = wa * ww[b][1];
                const float4* row = vbox + (t0 + a * ey * ez + b * ez);
                float rb[3] = {0.f, 0.f, 0.f};
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    const float4 nd = row[c];
                    const float w = wab * ww[c][2];
                    const float wn[3] = {w * nd.x, w * nd.y, w * nd.z};
#pragma unroll
                    for (int r = 0; r < 3; r++) {
                        rb[r] += wn[r];
                        if (c == 1) Mz[r] += wn[r];
                        if (c == 2) Mz[r] += 2.0f * wn[r];
                    }
                }
#pragma unroll
                for (int r = 0; r < 3; r++) {
                    ra[r] += rb[r];
                    if (b == 1) My[r] += rb[r];
                    if (b == 2) My[r] += 2.0f * rb[r];
                }
            }
            const float fa = (float)a;
#pragma unroll
            for (int r = 0; r < 3; r++) {
                v[r] += ra[r];
                Mx[r] += fa * ra[r];
            }
        }
        const float s4 = 4.0f * (float)P.h_inv;
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

// ------------------------------------------------- TMA-staged gather box
// The velocity grid as a 4-D tensor (float components, z, y, x): one tensor
// copy brings a fixed box of kTmaBoxX x kTmaBoxY x kTmaBoxZ nodes (4,608 B,
// innermost coordinate 0, so always 16-byte aligned) into the warp's shared
// slice, completed on a per-warp mbarrier. Plain (non-multicast) loads.
constexpr int kTmaBoxX = 3, kTmaBoxY = 3, kTmaBoxZ = 20;
constexpr int kTmaBoxNodes = kTmaBoxX * kTmaBoxY * kTmaBoxZ;
constexpr unsigned kTmaBoxBytes = kTmaBoxNodes * 16u;
constexpr int kTmaSliceNodes = 184;   // per-warp slice: >= kTmaBoxNodes, a multiple of 128 B
constexpr int kTmaWaitPolls = 1 << 22;   // polls of one bounded wait (a copy takes ~1 us)

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init_one(unsigned long long* bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait for phase `parity` of bar: false when `polls` polls passed.
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long* bar, unsigned parity,
                                                  int polls = kTmaWaitPolls) {
    for (int k = 0; k < polls; k++)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

// Test of the bounded wait's error path: one warp arms an mbarrier for 16
// bytes that no copy delivers (nothing is in flight), waits at most `polls`
// polls and records MPM_ERR_COPY_TIMEOUT, or 0 if the phase completed.
__global__ void k_wait_timeout_probe(int polls, int* status) {
    __shared__ unsigned long long bar;
    if (threadIdx.x == 0) {
        mbar_init_one(&bar);
        mbar_expect_tx(&bar, 16u);
    }
    __syncwarp();
    const bool done = mbar_wait_bounded(&bar, 0, polls);
    if (threadIdx.x == 0) *status = done ? 0 : MPM_ERR_COPY_TIMEOUT;
}

__device__ __forceinline__ void tma_load_box(void* dst, const CUtensorMap* map, int z0, int y0, int x0,
                                             unsigned long long* bar) {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
        "[%6];" ::"r"(smem_u32(dst)),
        "l"(map), "r"(0), "r"(z0), "r"(y0), "r"(x0), "r"(smem_u32(bar))
        : "memory");
}

// Box of base cells of the warp's lanes with an in-grid stencil, and the
// TMA copy of its velocity nodes when it fits the fixed box (issued by lane
// 0 as soon as the bases are known, so that it overlaps the particles' other
// loads). Called by the whole warp.
struct WarpBox {
    int lo0, lo1, lo2;
    int dims;   // ex | ey << 8 | ez << 16 | any << 24 | tma << 25 (extents <= 255 when used)
    __device__ __forceinline__ int ex() const { return dims & 255; }
    __device__ __forceinline__ int ey() const { return (dims >> 8) & 255; }
    __device__ __forceinline__ int ez() const { return (dims >> 16) & 255; }
    __device__ __forceinline__ bool any() const { return (dims >> 24) & 1; }
    __device__ __forceinline__ bool tma() const { return (dims >> 25) & 1; }
};

// Computes the box and, when it fits, initialises the warp's mbarrier (one
// use per launch) and issues the tensor copy (lane 0).
__device__ __forceinline__ WarpBox warp_box_issue(const DevParams& P, const CUtensorMap* map, float4* vbox,
                                                  unsigned long long* bar, bool part, const int base[3], int lane) {
    WarpBox B;
    B.lo0 = __reduce_min_sync(0xffffffffu, part ? base[0] : INT_MAX);
    B.lo1 = __reduce_min_sync(0xffffffffu, part ? base[1] : INT_MAX);
    B.lo2 = __reduce_min_sync(0xffffffffu, part ? base[2] : INT_MAX);
    const int hi0 = __reduce_max_sync(0xffffffffu, part ? base[0] : INT_MIN);
    const int hi1 = __reduce_max_sync(0xffffffffu, part ? base[1] : INT_MIN);
    const int hi2 = __reduce_max_sync(0xffffffffu, part ? base[2] : INT_MIN);
    const bool any = B.lo0 <= hi0;
    const int ex = any ? hi0 - B.lo0 + 3 : 0, ey = any ? hi1 - B.lo1 + 3 : 0, ez = any ? hi2 - B.lo2 + 3 : 0;
    const bool tma = any && ex <= kTmaBoxX && ey <= kTmaBoxY && ez <= kTmaBoxZ;
    const bool small = any && ex <= 255 && ey <= 255 && ez <= 255;
    B.dims = small ? (ex | (ey << 8) | (ez << 16) | (1 << 24) | ((int)tma << 25)) : 0;
    if (tma && lane == 0) {
        mbar_init_one(bar);
        mbar_expect_tx(bar, kTmaBoxBytes);
        tma_load_box(vbox, map, B.lo2, B.lo1, B.lo0 + P.halo, bar);
    }
    return B;
}

// Gather from the warp's box: the TMA copy issued by warp_box_issue when it
// fit, else the warp's own coalesced loads (boxes up to VCAP nodes), else the
// grid through L1. A copy that does not complete within the bounded wait
// raises MPM_ERR_COPY_TIMEOUT, is waited for once more, and the warp gathers
// through L1. Called by the whole warp.
template <int VCAP>
__device__ __forceinline__ void g2p_gather_tma(const DevParams& P, const WarpBox& B, const float4* __restrict__ vel,
                                               float4* __restrict__ vbox, unsigned long long* bar, bool part,
                                               bool active, const int base[3], const float fx[3], float v[3],
                                               float C[3][3], int lane, WxSlot wx, int* err) {
    const int lo0 = B.lo0, lo1 = B.lo1, lo2 = B.lo2;
    int ey = B.ey(), ez = B.ez();
    bool staged = false;
    if (B.tma()) {
        __syncwarp();
        staged = mbar_wait_bounded(bar, 0);
        if (!staged) {
            if (lane == 0) raise_error(err, MPM_ERR_COPY_TIMEOUT);
            mbar_wait_bounded(bar, 0);   // let the copy in flight land before the slice is left
        }
        ey = kTmaBoxY;
        ez = kTmaBoxZ;
    } else if (B.any() && B.ex() * ey * ez <= VCAP) {
        const int vol = B.ex() * ey * ez;
        const int slab = (int)P.slab, gz = P.Gz;
        const int g0 = ((lo0 + P.halo) * P.Gy + lo1) * gz + lo2;
        const float inv_ez = 1.0f / (float)ez, inv_ey = 1.0f / (float)ey;
        for (int k = lane; k < vol; k += 32) {
            const int row = (int)(((float)k + 0.5f) * inv_ez);   // k / ez (k, ez <= VCAP)
            const int tz = k - row * ez;
            const int tx = (int)(((float)row + 0.5f) * inv_ey);
            const int ty = row - tx * ey;
            vbox[k] = __ldg(vel + (g0 + tx * slab + ty * gz + tz));
        }
        __syncwarp();
        staged = true;
    }
    if (part && staged) {
        // v = sum w nv and the first moments M_k = sum w nv o_k over the node
        // offsets o = (a, b, c); C = 4/h sum w nv (o - f) = 4/h (M - f v)
        float ww[3][3];
        quad_weights<float>(fx, ww);
        wx.put(ww);
        float Mx[3], My[3], Mz[3];
#pragma unroll
        for (int r = 0; r < 3; r++) { v[r] = 0.f; Mx[r] = 0.f; My[r] = 0.f; Mz[r] = 0.f; }
        const int t0 = ((base[0] - lo0) * ey + (base[1] - lo1)) * ez + (base[2] - lo2);
#pragma unroll 1
        for (int a = 0; a < 3; a++) {
            const float wa = wx.get(a);
            float ra[3] = {0.f, 0.f, 0.f};
#pragma unroll
            for (int b = 0; b < 3; b++) {
                const float wab = wa * ww[b][1];
                const float4* row = vbox + (t0 + a * ey * ez + b * ez);
                float rb[3] = {0.f, 0.f, 0.f};
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    const float4 nd = row[c];
                    const float w = wab * ww[c][2];
                    const float wn[3] = {w * nd.x, w * nd.y, w * nd.z};
#pragma unroll
                    for (int r = 0; r < 3; r++) {
                        rb[r] += wn[r];
                        if (c == 1) Mz[r] += wn[r];
                        if (c == 2) Mz[r] += 2.0f * wn[r];
                    }
                }
#pragma unroll
                for (int r = 0; r < 3; r++) {
                    ra[r] += rb[r];
                    if (b == 1) My[r] += rb[r];
                    if (b == 2) My[r] += 2.0f * rb[r];
                }
            }
            const float fa = (float)a;
#pragma unroll
            for (int r = 0; r < 3; r++) {
                v[r] += ra[r];
                Mx[r] += fa * ra[r];
            }
        }
        const float s4 = 4.0f * (float)P.h_inv;
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

// Scatter of one particle (base, fx, m, mv, S) with the warp reduction over
// lanes sharing a base cell; leaders add float4 {m, mv} to acc.
template <bool AGG = true>
__device__ __forceinline__ void p2g_scatter_mixed(const DevParams& P, float4* __restrict__ acc, bool active, bool inside,
                                                  const int base[3], const float fx[3], float mass, const float mv[3],
                                                  const float S[3][3], int lane) {
    const int i0 = ((base[0] + P.halo) * P.Gy + base[1]) * P.Gz + base[2];
    const int key = inside ? i0 : -1 - lane;
    const unsigned peers = AGG ? __match_any_sync(0xffffffffu, key) : (1u << lane);
    const int leader = __ffs(peers) - 1;
    const int rounds = AGG ? (int)__reduce_max_sync(0xffffffffu, (unsigned)(__popc(peers) - 1)) : 0;
    float ww[3][3];
    quad_weights<float>(fx, ww);
    const float h = (float)P.h;
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
                unsigned rest = peers & ~(1u << leader);
                for (int k = 0; k < rounds; k++) {
                    const int src = rest ? __ffs(rest) - 1 : lane;
                    rest &= rest - 1;
#pragma unroll
                    for (int q = 0; q < 4; q++) {
                        const float o = __shfl_sync(0xffffffffu, val[q], src);
                        if (lane == leader && src != lane) val[q] += o;
                    }
                }
                if (!active || lane != leader) continue;
                if (!inside && !node_inside(P, base[0] + a, base[1] + b, base[2] + c)) continue;
                atomicAdd(acc + (ib + c), make_float4(val[0], val[1], val[2], val[3]));
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
__device__ __forceinline__ void p2g_scatter_pairs(const DevParams& P, float4* __restrict__ acc, bool active,
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
        const float h = (float)P.h;
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
                    if (emit) atomicAdd(acc + (ib + c), make_float4(val[0], val[1], val[2], val[3]));
                }
            }
        }
        return;
    }
    const float h = (float)P.h;
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
                atomicAdd(acc + (ib + c), make_float4(val[0], val[1], val[2], val[3]));
            }
        }
    }
}

// One particle's stencil as a lane of the split scatter walks it: loop node
// (a, b, c) is stencil node (a, b, c), or (2-a, 2-b, 2-c) when flipped. The
// flip permutes the per-dimension weights already computed for the particle
// (w_{2-k}(f) = w_k(2-f) for the quadratic B-spline), so each node gets the
// same weight numbers as in the unsplit loop. The affine part is walked
// incrementally: u = m v + S (x_node - x_p) at loop node (0,0,0), and each
// loop step in a, b, c adds sh = +-h S[:,d] (minus when flipped).
struct SplitStream {
    float m, u[3], s0h[3], s1h[3], s2h[3], wa[2], wb[3], wc[3];
};

__device__ __forceinline__ void split_stream(const DevParams& P, SplitStream& H, float m, const float mv[3],
                                             const float S[3][3], const float fx[3], bool flip) {
    float ww[3][3];
    quad_weights<float>(fx, ww);
    const float h = (float)P.h;
    const float sg = flip ? -h : h;
    const float k0 = flip ? 2.0f : 0.0f;
    H.m = m;
#pragma unroll
    for (int k = 0; k < 3; k++) {
        H.wb[k] = flip ? ww[2 - k][1] : ww[k][1];
        H.wc[k] = flip ? ww[2 - k][2] : ww[k][2];
        if (k < 2) H.wa[k] = flip ? ww[2 - k][0] : ww[k][0];
    }
    const float d0 = (k0 - fx[0]) * h, d1 = (k0 - fx[1]) * h, d2 = (k0 - fx[2]) * h;
#pragma unroll
    for (int r = 0; r < 3; r++) {
        H.u[r] = mv[r] + S[r][0] * d0 + S[r][1] * d1 + S[r][2] * d2;
        H.s0h[r] = S[r][0] * sg;
        H.s1h[r] = S[r][1] * sg;
        H.s2h[r] = S[r][2] * sg;
    }
}

// Split scatter (SCATTER 5). Pairs as in p2g_scatter_pairs (two adjacent
// lanes with the same base cell), but instead of shuffling 4 values per node
// the pair exchanges its payloads once and each lane adds BOTH particles'
// contributions over half of the 27 nodes: the first lane nodes 0..13 in
// (a, b, c) order, the second the mirror images of its loop nodes 0..12,
// i.e. nodes 26..14. A lone particle walks both halves itself, as two
// streams: nodes 0..13, then the mirrored 26..14. Each lane runs 14 loop
// nodes with two contributions each (27 of the 28 slots used) and one float4
// atomic per node (pairs) or two (lone particles). Warps with a stencil
// outside the grid take the checked loop of p2g_scatter_pairs.
__device__ __forceinline__ void p2g_scatter_split(const DevParams& P, float4* __restrict__ acc, bool active,
                                                  bool inside, const int base[3], const float fx[3], float mass,
                                                  const float mv[3], const float S[3][3], int lane, WxSlot wx) {
    if (!__all_sync(0xffffffffu, inside || !active)) {
        p2g_scatter_pairs(P, acc, active, inside, base, fx, mass, mv, S, lane, wx);
        return;
    }
    const int i0 = ((base[0] + P.halo) * P.Gy + base[1]) * P.Gz + base[2];
    const int key = active ? i0 : -1 - lane;
    const unsigned peers = __match_any_sync(0xffffffffu, key);
    const int rank = __popc(peers & ((1u << lane) - 1u));
    const int next_key = __shfl_down_sync(0xffffffffu, key, 1);
    const bool first = lane < 31 && next_key == key && (rank & 1) == 0;
    const bool second = __shfl_up_sync(0xffffffffu, (int)first, 1) != 0 && lane > 0;
    const bool merged = first || second;
    const int partner = first ? lane + 1 : (second ? lane - 1 : lane);
    // the partner's payload (a lone lane reads its own)
    float pm = __shfl_sync(0xffffffffu, mass, partner), pmv[3], pS[3][3], pfx[3];
#pragma unroll
    for (int r = 0; r < 3; r++) {
        pmv[r] = __shfl_sync(0xffffffffu, mv[r], partner);
        pfx[r] = __shfl_sync(0xffffffffu, fx[r], partner);
#pragma unroll
        for (int c = 0; c < 3; c++) pS[r][c] = __shfl_sync(0xffffffffu, S[r][c], partner);
    }
    // stream A: own particle, flipped on the second lane of a pair; stream B:
    // the partner's particle on a pair's lanes (same flip), the own particle
    // flipped on a lone lane (same base cell in every case)
    SplitStream A, B;
    split_stream(P, A, mass, mv, S, fx, second);
    split_stream(P, B, pm, pmv, pS, pfx, !first);
    const int slab = (int)P.slab, gz = P.Gz;
    const int i0f = i0 + 2 * slab + 2 * gz + 2;   // loop node (0,0,0) of a flipped walk
    const bool emit_a = active;
    const bool emit_b = active && !merged;
    // loop rows (a, b) = (0,0) (0,1) (0,2) (1,0) (1,1); u walks row starts
#pragma unroll
    for (int a = 0; a < 2; a++) {
#pragma unroll
        for (int b = 0; b < 3; b++) {
            if (9 * a + 3 * b > 13) continue;
            if (b > 0) {
#pragma unroll
                for (int r = 0; r < 3; r++) { A.u[r] += A.s1h[r]; B.u[r] += B.s1h[r]; }
            } else if (a > 0) {
#pragma unroll
                for (int r = 0; r < 3; r++) {
                    A.u[r] += A.s0h[r] - 2.0f * A.s1h[r];
                    B.u[r] += B.s0h[r] - 2.0f * B.s1h[r];
                }
            }
            const float wab_a = A.wa[a] * A.wb[b], wab_b = B.wa[a] * B.wb[b];
            float za[3], zb[3];
#pragma unroll
            for (int r = 0; r < 3; r++) { za[r] = A.u[r]; zb[r] = B.u[r]; }
            const int off_ab = a * slab + b * gz;
#pragma unroll
            for (int c = 0; c < 3; c++) {
                const int j = 9 * a + 3 * b + c;
                if (j > 13) continue;
                if (c > 0) {
#pragma unroll
                    for (int r = 0; r < 3; r++) { za[r] += A.s2h[r]; zb[r] += B.s2h[r]; }
                }
                const float wa_ = wab_a * A.wc[c], wb_ = wab_b * B.wc[c];
                float va[4] = {wa_ * A.m, wa_ * za[0], wa_ * za[1], wa_ * za[2]};
                const float vb[4] = {wb_ * B.m, wb_ * zb[0], wb_ * zb[1], wb_ * zb[2]};
                if (merged) {
#pragma unroll
                    for (int q = 0; q < 4; q++) va[q] += vb[q];
                }
                const int off = off_ab + c;
                // the centre node (j == 13) belongs to the unflipped walk only
                if (emit_a && !(j == 13 && second))
                    atomicAdd(acc + (second ? i0f - off : i0 + off), make_float4(va[0], va[1], va[2], va[3]));
                if (emit_b && j != 13)
                    atomicAdd(acc + (first ? i0 + off : i0f - off), make_float4(vb[0], vb[1], vb[2], vb[3]));
            }
        }
    }
}

// Shared-memory tile variant of the scatter. The block's particles (a
// contiguous range of the cell-sorted order) span a small box of nodes; the
// block accumulates the box with FP32 shared-memory atomics and adds each non-empty node to the grid once, as one
// float4 vector atomic. Returns false (nothing done) when the box exceeds the
// tile; the caller then scatters directly. Must be called by the whole block.
template <int BLOCK>
__device__ __forceinline__ bool p2g_scatter_tile(const DevParams& P, float4* __restrict__ acc, float* __restrict__ tile,
                                                 int tile_cap, bool active, bool inside, const int base[3],
                                                 const float fx[3], float mass, const float mv[3], const float S[3][3],
                                                 int lane) {
    __shared__ int s_box[6];
    if (threadIdx.x < 3) { s_box[threadIdx.x] = INT_MAX; s_box[3 + threadIdx.x] = INT_MIN; }
    __syncthreads();
    const bool in_box = active && inside;
#pragma unroll
    for (int d = 0; d < 3; d++) {
        int lo = in_box ? base[d] : INT_MAX, hi = in_box ? base[d] + 2 : INT_MIN;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
            hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
        }
        if (lane == 0) { atomicMin(&s_box[d], lo); atomicMax(&s_box[3 + d], hi); }
    }
    __syncthreads();
    const int bx = s_box[0], by = s_box[1], bz = s_box[2];
    const int ex = s_box[3] - bx + 1, ey = s_box[4] - by + 1, ez = s_box[5] - bz + 1;
    if (bx > s_box[3]) return true;   // no particle of the block is inside
    const long long vol = (long long)ex * ey * ez;
    if (vol > tile_cap) return false;
    const int nv = (int)vol;
    for (int k = threadIdx.x; k < 4 * nv; k += BLOCK) tile[k] = 0.f;
    __syncthreads();
    // particles of the block whose stencil leaves the grid go direct
    if (active && !inside) {
        p2g_scatter_mixed<false>(P, acc, active, inside, base, fx, mass, mv, S, lane);
    } else {
        const int t0 = ((base[0] - bx) * ey + (base[1] - by)) * ez + (base[2] - bz);
        float ww[3][3];
        quad_weights<float>(fx, ww);
        const float h = (float)P.h;
#pragma unroll 1
        for (int a = 0; a < 3; a++) {
            const float dx = (a - fx[0]) * h;
#pragma unroll
            for (int b = 0; b < 3; b++) {
                const float dy = (b - fx[1]) * h;
                const float wab = pick3(a, ww[0][0], ww[1][0], ww[2][0]) * ww[b][1];
                const int tb = t0 + (a * ey + b) * ez;
                float part[3];
#pragma unroll
                for (int m = 0; m < 3; m++) part[m] = mv[m] + S[m][0] * dx + S[m][1] * dy;
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    const float dz = (c - fx[2]) * h;
                    const float W = wab * ww[c][2];
                    if (!in_box) continue;
                    const int t = tb + c;
                    atomicAdd(tile + t, W * mass);
                    atomicAdd(tile + nv + t, W * (part[0] + S[0][2] * dz));
                    atomicAdd(tile + 2 * nv + t, W * (part[1] + S[1][2] * dz));
                    atomicAdd(tile + 3 * nv + t, W * (part[2] + S[2][2] * dz));
                }
            }
        }
    }
    __syncthreads();
    const int slab = (int)P.slab, gz = P.Gz;
    const int g0 = ((bx + P.halo) * P.Gy + by) * gz + bz;
    for (int t = threadIdx.x; t < nv; t += BLOCK) {
        const float m = tile[t];
        if (m == 0.f) continue;
        const int tz = t % ez, ty = (t / ez) % ey, tx = t / (ez * ey);
        atomicAdd(acc + (g0 + tx * slab + ty * gz + tz), make_float4(m, tile[nv + t], tile[2 * nv + t], tile[3 * nv + t]));
    }
    return true;
}

// Shared-memory tile in 32-bit block fixed point. As p2g_scatter_tile, but
// the tile holds integers: each contribution v is added as round(v * 2^e)
// with native 32-bit shared atomics (order-independent sums), e chosen per
// block from its largest possible contribution so that a node can absorb up
// to 128 of them without overflow (2^-23 of that bound per unit). The flush
// converts each node back to FP32 and adds it to the grid with one float4
// atomic. Must be called by the whole block of 128 threads.
__device__ __forceinline__ int fx32_exponent(float bound) {
    int ex;
    frexpf(fmaxf(bound, 1e-30f), &ex);   // bound < 2^ex
    return 23 - ex;                        // 128 * bound * 2^e < 2^30
}

template <int BLOCK>
__device__ __forceinline__ bool p2g_scatter_tile_fx(const DevParams& P, float4* __restrict__ acc, int* __restrict__ tile,
                                                    int tile_cap, bool active, bool inside, const int base[3],
                                                    const float fx[3], float mass, const float mv[3],
                                                    const float S[3][3], int lane) {
    __shared__ int s_box[8];
    if (threadIdx.x < 3) { s_box[threadIdx.x] = INT_MAX; s_box[3 + threadIdx.x] = INT_MIN; }
    if (threadIdx.x == 0) { s_box[6] = 0; s_box[7] = 0; }
    __syncthreads();
    const bool in_box = active && inside;
    // bound of |w (m v + S (x_i - x_p))| over the stencil: w <= 1, |x_i - x_p| <= 1.5 h per axis
    const float h15 = 1.5f * (float)P.h;
    float pb = 0.f;
    if (in_box) {
#pragma unroll
        for (int m = 0; m < 3; m++)
            pb = fmaxf(pb, fabsf(mv[m]) + h15 * (fabsf(S[m][0]) + fabsf(S[m][1]) + fabsf(S[m][2])));
    }
    float mb = in_box ? mass : 0.f;
#pragma unroll
    for (int d = 0; d < 3; d++) {
        int lo = in_box ? base[d] : INT_MAX, hi = in_box ? base[d] + 2 : INT_MIN;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
            hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
        }
        if (lane == 0) { atomicMin(&s_box[d], lo); atomicMax(&s_box[3 + d], hi); }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        pb = fmaxf(pb, __shfl_xor_sync(0xffffffffu, pb, o));
        mb = fmaxf(mb, __shfl_xor_sync(0xffffffffu, mb, o));
    }
    if (lane == 0) { atomicMax(&s_box[6], __float_as_int(pb)); atomicMax(&s_box[7], __float_as_int(mb)); }
    __syncthreads();
    const int bx = s_box[0], by = s_box[1], bz = s_box[2];
    if (bx > s_box[3]) return true;   // no particle of the block is inside
    const int ex = s_box[3] - bx + 1, ey = s_box[4] - by + 1, ez = s_box[5] - bz + 1;
    const long long vol = (long long)ex * ey * ez;
    if (vol > tile_cap) return false;
    const int nv = (int)vol;
    const int e_p = fx32_exponent(__int_as_float(s_box[6]));
    const int e_m = fx32_exponent(__int_as_float(s_box[7]));
    const float sc_p = ldexpf(1.0f, e_p), sc_m = ldexpf(1.0f, e_m);
    for (int k = threadIdx.x; k < 4 * nv; k += BLOCK) tile[k] = 0;
    __syncthreads();
    if (active && !inside) {
        p2g_scatter_mixed<false>(P, acc, active, inside, base, fx, mass, mv, S, lane);
    } else if (in_box) {
        const int t0 = ((base[0] - bx) * ey + (base[1] - by)) * ez + (base[2] - bz);
        float ww[3][3];
        quad_weights<float>(fx, ww);
        const float h = (float)P.h;
        const float msc = mass * sc_m;
        float Ssc[3][3], mvsc[3];
#pragma unroll
        for (int m = 0; m < 3; m++) {
            mvsc[m] = mv[m] * sc_p;
#pragma unroll
            for (int k = 0; k < 3; k++) Ssc[m][k] = S[m][k] * sc_p;
        }
#pragma unroll 1
        for (int a = 0; a < 3; a++) {
            const float dx = (a - fx[0]) * h;
#pragma unroll
            for (int b = 0; b < 3; b++) {
                const float dy = (b - fx[1]) * h;
                const float wab = pick3(a, ww[0][0], ww[1][0], ww[2][0]) * ww[b][1];
                const int tb = t0 + (a * ey + b) * ez;
                float part[3];
#pragma unroll
                for (int m = 0; m < 3; m++) part[m] = mvsc[m] + Ssc[m][0] * dx + Ssc[m][1] * dy;
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    const float dz = (c - fx[2]) * h;
                    const float W = wab * ww[c][2];
                    const int t = tb + c;
                    atomicAdd(tile + t, __float2int_rn(W * msc));
                    atomicAdd(tile + nv + t, __float2int_rn(W * (part[0] + Ssc[0][2] * dz)));
                    atomicAdd(tile + 2 * nv + t, __float2int_rn(W * (part[1] + Ssc[1][2] * dz)));
                    atomicAdd(tile + 3 * nv + t, __float2int_rn(W * (part[2] + Ssc[2][2] * dz)));
                }
            }
        }
    }
    __syncthreads();
    const float inv_m = ldexpf(1.0f, -e_m), inv_p = ldexpf(1.0f, -e_p);
    const int slab = (int)P.slab, gz = P.Gz;
    const int g0 = ((bx + P.halo) * P.Gy + by) * gz + bz;
    for (int t = threadIdx.x; t < nv; t += BLOCK) {
        const int m = tile[t];
        if (m == 0) continue;
        const int tz = t % ez, ty = (t / ez) % ey, tx = t / (ez * ey);
        atomicAdd(acc + (g0 + tx * slab + ty * gz + tz),
                  make_float4((float)m * inv_m, (float)tile[nv + t] * inv_p, (float)tile[2 * nv + t] * inv_p,
                              (float)tile[3 * nv + t] * inv_p));
    }
    return true;
}

// P2G payload of a particle: S = m C - dt V Dp^-1 tau (mpm_kernels.cuh:63)
__device__ __forceinline__ void p2g_payload_mixed(const DevParams& P, const float E[3][3], const float C[3][3],
                                                  const float v[3], bool liquid, float Jpm1, float& mass, float mv[3],
                                                  float S[3][3]) {
    mass = (float)(liquid ? P.liquid_mass : P.particle_mass);
    float tau[3][3];
    if (liquid) {
        // kappa (1 - J^-3) with J = 1 + d: (J^3 - 1) / J^3 = d (3 + 3d + d^2) / J^3, free of cancellation
        const float J = 1.0f + Jpm1;
        const float pw = (float)P.kappa * (Jpm1 * (3.0f + Jpm1 * (3.0f + Jpm1)) / (J * J * J));
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = 0; j < 3; j++) tau[i][j] = (i == j) ? pw : 0.f;
    } else {
        kirchhoff_mixed(P, E, tau);
    }
    const float dvd = (float)P.dt_vol_Dpinv;
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

// Standalone P2G from the stored state (first step, phase API).
__global__ void __launch_bounds__(256) k_p2g_mixed(DevParams P, MixedState s, int n, float4* __restrict__ acc,
                                                   int* err) {
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
    p2g_scatter_mixed(P, acc, active, inside, base, fx, mass, mv, S, lane);
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
        const float dt = (float)P.dt;
        const float adv = dt * (float)P.h_inv * kFixScale;
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
            mass = (float)P.particle_mass;
            float tau[3][3];
            tau_inv(P, inv, tau);
            const float dvd = (float)P.dt_vol_Dpinv;
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

// Fused G2P (this step) -> P2G (next step). do_p2g = 0 gives a plain G2P.
// SCATTER: 0 = warp-reduced direct float4 atomics, 1 = direct float4
// atomics, 2 = FP32 shared-memory tile, 3 = int32 fixed-point shared-memory
// tile (2 and 3 fall back to 0 when the box is too big), 4 = direct float4
// atomics with same-cell pairs merged, 5 = split scatter of merged pairs.
// GATHER: 0 = from the grid through L1, 1 = from the warp's velocity box
// staged in shared memory by the warp's loads (dynamic shared memory of
// 4 x kVBoxNodes float4), 2 = the box brought in by one TMA tensor copy per
// warp (4 x kTmaSliceNodes float4; vel_map).
constexpr int kVBoxNodes = 256;
template <int MINB, int SCATTER, int GATHER = 0>
__global__ void __launch_bounds__(128, MINB) k_g2p2g_mixed(DevParams P, MixedState s, int n,
                                                           const float4* __restrict__ vel, float4* __restrict__ acc,
                                                           int do_p2g, int record_pq, int store_vc, int* err,
                                                           int tile_cap, int* __restrict__ rm_list,
                                                           int* __restrict__ rm_count,
                                                           const __grid_constant__ CUtensorMap vel_map) {
    extern __shared__ __align__(128) float mixed_tile[];
    __shared__ unsigned long long vbox_bar[4];
    __shared__ float wx_slots[3 * 128];
    const WxSlot wx{wx_slots + threadIdx.x};
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31;
    bool active = i < n;
    int X[3] = {0, 0, 0}, st = (int)kDisabled;
    float E[3][3], Jpm1 = 0.f;
    // positions and status first: the gather box (and its copy) depends on them
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
    float4* const vbox_tma = reinterpret_cast<float4*>(mixed_tile) + (threadIdx.x >> 5) * kTmaSliceNodes;
    WarpBox wbox;
    if (GATHER == 2)
        wbox = warp_box_issue(P, &vel_map, vbox_tma, &vbox_bar[threadIdx.x >> 5], active && e0 == 0, base, lane);
    if (active) {
#pragma unroll
        for (int r = 0; r < 3; r++)
#pragma unroll
            for (int c = 0; c < 3; c++) E[r][c] = s.E[(3 * r + c) * s.pitch + i];
        Jpm1 = s.Jpm1[i];
    }
    const int st_in = st;
    const float jpm1_in = Jpm1;
    if (GATHER == 2) {
        g2p_gather_tma<kTmaSliceNodes>(P, wbox, vel, vbox_tma, &vbox_bar[threadIdx.x >> 5], active && e0 == 0,
                                       active, base, fx, v, C, lane, wx, err);
    } else if (GATHER == 1) {
        float4* vbox = reinterpret_cast<float4*>(mixed_tile) + (threadIdx.x >> 5) * kVBoxNodes;
        g2p_gather_staged<kVBoxNodes>(P, vel, vbox, active && e0 == 0, active, base, fx, v, C, lane, wx);
    } else if (active) {
        g2p_gather_mixed(P, vel, base, fx, v, C, e0 != 0, wx);
    }
    const bool need_rm = fused_update_state(P, s, i, active, X, st, st_in, jpm1_in, E, Jpm1, v, C, inv, record_pq,
                                            store_vc, rm_list, rm_count, lane);
    active = active && !need_rm;   // crushed points scatter in k_return_map_mixed
    if (!do_p2g) return;   // uniform across the launch
    float mass, mv[3], S[3][3];
    fused_payload(P, active, X, st, E, C, v, Jpm1, inv, base, fx, mass, mv, S, inside, err);
    if (SCATTER == 2 && p2g_scatter_tile<128>(P, acc, mixed_tile, tile_cap, active, inside, base, fx, mass, mv, S, lane))
        return;
    if (SCATTER == 3 && p2g_scatter_tile_fx<128>(P, acc, reinterpret_cast<int*>(mixed_tile), tile_cap, active, inside,
                                                 base, fx, mass, mv, S, lane))
        return;
    if (SCATTER == 5) p2g_scatter_split(P, acc, active, inside, base, fx, mass, mv, S, lane, wx);
    else if (SCATTER == 4) p2g_scatter_pairs(P, acc, active, inside, base, fx, mass, mv, S, lane, wx);
    else if (SCATTER == 1) p2g_scatter_mixed<false>(P, acc, active, inside, base, fx, mass, mv, S, lane);
    else p2g_scatter_mixed<true>(P, acc, active, inside, base, fx, mass, mv, S, lane);
}

// Return map (FP64, mpm_kernels.cuh:486-544) of the crushed points listed by
// k_g2p2g_mixed, then their P2G (direct float4 atomics) when do_p2g. The
// list holds *count indices; the kernel also clears next_count, the counter
// the next fused launch appends to. Grid-stride over the list.
__global__ void __launch_bounds__(128) k_return_map_mixed(DevParams P, MixedState s, const int* __restrict__ rm_list,
                                                          const int* __restrict__ count, int* __restrict__ next_count,
                                                          float4* __restrict__ acc, int do_p2g, int* err) {
    if (blockIdx.x == 0 && threadIdx.x == 0) *next_count = 0;
    const int m = *count;
    const int lane = threadIdx.x & 31;
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
        p2g_scatter_mixed<false>(P, acc, true, e == 0, base, fx, mass, mv, S, lane);
    }
}

// Node update for the mixed grid: FP64 arithmetic on the FP32 sums (one
// reciprocal of the mass), contact force in FP64 (sensor and per-substep
// total), velocities written as float4, the accumulator cleared for the next
// P2G. Node coordinates by reciprocal multiplication (no integer division).
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_update_mixed(DevParams P, float4* __restrict__ acc, float4* __restrict__ vel,
                                                        double ind_x, double ind_y, double* __restrict__ sensor,
                                                        double* __restrict__ force3) {
    const int idx = blockIdx.x * BLOCK + threadIdx.x;   // the handle keeps nodes < 2^31
    double f[3] = {0, 0, 0};
    if (idx < P.nodes) {
        const float4 a = acc[idx];
        const double mass = a.x;
        if (mass != 0) {
            acc[idx] = make_float4(0.f, 0.f, 0.f, 0.f);
            int idx_z, idx_y;
            const int col = div_by(idx, P.Gz, P.inv_gz, idx_z);
            const int idx_x = div_by(col, P.Gy, P.inv_gy, idx_y);
            const int gx = idx_x - P.halo, gy = idx_y, gz = idx_z;
            const double inv_m = 1.0 / mass;
            double v[3] = {(double)a.y * inv_m, (double)a.z * inv_m, (double)a.w * inv_m};
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
#pragma unroll
                        for (int k = 0; k < 3; k++) f[k] = (prev[k] - v[k]) * mass / P.dt;
                        float angle = atan2f((float)n0, (float)n1);
                        angle = (float)((double)angle + MPM_PI);
                        angle = (float)((double)angle * (P.subdiv / (2 * MPM_PI)));
                        const int ia = min(max((int)angle, 0), P.subdiv - 1);
                        const int iz = min(max(idx_z, 0), P.Gz - 1);
                        double* s = sensor + 3 * (iz + ia * P.Gz);
                        atomicAdd(s + 0, f[0]);
                        atomicAdd(s + 1, f[1]);
                        atomicAdd(s + 2, f[2]);
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
