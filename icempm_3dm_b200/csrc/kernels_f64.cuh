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

// Lanes whose particles share a base cell share all 27 stencil nodes. The
// group's lowest lane (leader) sums the peers' node values (lane order, so
// the sum is deterministic for a given warp content) and alone writes them.
struct WarpGroup {
    unsigned peers;   // lanes of this lane's group
    int leader;
    int rounds;       // warp-uniform: max group size - 1
};

__device__ __forceinline__ WarpGroup warp_group(long long key) {
    WarpGroup g;
    g.peers = __match_any_sync(0xffffffffu, key);
    g.leader = __ffs(g.peers) - 1;
    g.rounds = (int)__reduce_max_sync(0xffffffffu, (unsigned)(__popc(g.peers) - 1));
    return g;
}

__device__ __forceinline__ void group_reduce(const WarpGroup& g, int lane, double v[4]) {
    unsigned rest = g.peers & ~(1u << g.leader);
    for (int k = 0; k < g.rounds; k++) {
        const int src = rest ? __ffs(rest) - 1 : lane;
        rest &= rest - 1;
#pragma unroll
        for (int c = 0; c < 4; c++) {
            const double o = __shfl_sync(0xffffffffu, v[c], src);
            if (lane == g.leader && src != lane) v[c] += o;
        }
    }
}

// Group key of a particle for the warp reduction: its base-cell index, or a
// lane-unique negative value for lanes that must act alone (inactive, or a
// stencil reaching outside the grid).
__device__ __forceinline__ long long base_key(const DevParams& P, const P2GPoint& q, bool ok, int lane) {
    if (!ok) return -1 - lane;
    return node_index(P, q.base[0], q.base[1], q.base[2]);
}

// Variant 1: one thread per particle, 27 x 4 FP64 atomics into the SoA grid.
__global__ void k_p2g_direct_f64(DevParams P, const double* __restrict__ pts, size_t pitch, int n,
                                 double* __restrict__ grid, int* err) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    P2GPoint q;
    if (!p2g_prepare(P, pts, pitch, i, q, err)) return;
    p2g_scatter(P, q, [&](int a, int b, int c, double incM, const double incV[3]) {
        const int x = q.base[0] + a, y = q.base[1] + b, z = q.base[2] + c;
        if (!node_inside(P, x, y, z)) return;
        grid_atomic_add(grid, P.gstride, node_index(P, x, y, z), incM, incV);
    });
}

// Variant 2: as 1, with the warp reduction over lanes sharing a base cell.
__global__ void k_p2g_warpagg_f64(DevParams P, const double* __restrict__ pts, size_t pitch, int n,
                                  double* __restrict__ grid, int* err) {
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
    const WarpGroup g = warp_group(base_key(P, q, inside, lane));
    p2g_scatter(P, q, [&](int a, int b, int c, double incM, const double incV[3]) {
        const int x = q.base[0] + a, y = q.base[1] + b, z = q.base[2] + c;
        double v[4] = {incM, incV[0], incV[1], incV[2]};
        group_reduce(g, lane, v);
        if (lane != g.leader) return;
        if (active && !inside) {
            if (!node_inside(P, x, y, z)) return;
        } else if (!active) {
            return;
        }
        const double vv[3] = {v[1], v[2], v[3]};
        grid_atomic_add(grid, P.gstride, node_index(P, x, y, z), v[0], vv);
    });
}

// Variant 5: lanes that share a base cell merged in pairs by one shuffle
// round per node (cell-sorted order puts them in neighbouring lanes; the
// odd-ranked partner's four sums go to the even-ranked lane, which issues the
// FP64 atomics for both), 128-thread blocks at MINB blocks per SM.
template <int MINB>
__global__ void __launch_bounds__(128, MINB) k_p2g_pairs_f64(DevParams P, const double* __restrict__ pts, size_t pitch,
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

// Shared-memory tile P2G (variants 0 and 3): the block's particles (a
// contiguous range of the cell-sorted order) span a small box of nodes. The
// block accumulates its box in shared memory (SoA, tile_cap nodes per
// array), then adds each non-empty tile node to the grid once. Blocks whose
// box does not fit fall back to direct atomics.
__device__ __forceinline__ void block_box(int lo_in[3], int hi_in[3], int lo_out[3], int hi_out[3]) {
    __shared__ int s_lo[3], s_hi[3];
    if (threadIdx.x < 3) { s_lo[threadIdx.x] = INT_MAX; s_hi[threadIdx.x] = INT_MIN; }
    __syncthreads();
#pragma unroll
    for (int d = 0; d < 3; d++) {
        int lo = lo_in[d], hi = hi_in[d];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
            hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
        }
        if ((threadIdx.x & 31) == 0) { atomicMin(&s_lo[d], lo); atomicMax(&s_hi[d], hi); }
    }
    __syncthreads();
#pragma unroll
    for (int d = 0; d < 3; d++) { lo_out[d] = s_lo[d]; hi_out[d] = s_hi[d]; }
    __syncthreads();
}

template <int BLOCK, bool AGG>
__global__ void __launch_bounds__(BLOCK) k_p2g_tile_f64(DevParams P, const double* __restrict__ pts, size_t pitch,
                                                        int n, double* __restrict__ grid, int* err, int tile_cap) {
    extern __shared__ double tile[];
    const int i = blockIdx.x * BLOCK + threadIdx.x;
    const int lane = threadIdx.x & 31;
    P2GPoint q;
    bool active = (i < n) && p2g_prepare(P, pts, pitch, i, q, err);
    if (active && stencil_error(P, q.base[0], q.base[1], q.base[2])) {
        // out-of-grid stencils go the direct way (their in-grid nodes only)
        p2g_scatter(P, q, [&](int a, int b, int c, double incM, const double incV[3]) {
            const int x = q.base[0] + a, y = q.base[1] + b, z = q.base[2] + c;
            if (!node_inside(P, x, y, z)) return;
            grid_atomic_add(grid, P.gstride, node_index(P, x, y, z), incM, incV);
        });
        active = false;
    }
    int lo[3], hi[3];
#pragma unroll
    for (int d = 0; d < 3; d++) {
        lo[d] = active ? q.base[d] : INT_MAX;
        hi[d] = active ? q.base[d] + 2 : INT_MIN;
    }
    int blo[3], bhi[3];
    block_box(lo, hi, blo, bhi);
    if (blo[0] > bhi[0]) return;   // no active particle in the block
    const int ex = bhi[0] - blo[0] + 1, ey = bhi[1] - blo[1] + 1, ez = bhi[2] - blo[2] + 1;
    const long long vol = (long long)ex * ey * ez;
    if (!active) {
#pragma unroll
        for (int d = 0; d < 3; d++) { q.base[d] = blo[d]; q.fx[d] = 1.0; q.mv[d] = 0; }
#pragma unroll
        for (int r = 0; r < 3; r++)
#pragma unroll
            for (int c = 0; c < 3; c++) q.S[r][c] = 0;
        q.mass = 0;
    }
    if (vol > tile_cap) {
        if (!active) return;
        p2g_scatter(P, q, [&](int a, int b, int c, double incM, const double incV[3]) {
            grid_atomic_add(grid, P.gstride, node_index(P, q.base[0] + a, q.base[1] + b, q.base[2] + c), incM, incV);
        });
        return;
    }
    const int nv = (int)vol;
    for (int k = threadIdx.x; k < 4 * nv; k += BLOCK) {
        const int comp = k / nv;
        tile[comp * tile_cap + (k - comp * nv)] = 0.0;
    }
    __syncthreads();
    const int ox = q.base[0] - blo[0], oy = q.base[1] - blo[1], oz = q.base[2] - blo[2];
    if (AGG) {
        const WarpGroup g = warp_group(active ? (long long)((ox * ey + oy) * ez + oz) : -1 - lane);
        p2g_scatter(P, q, [&](int a, int b, int c, double incM, const double incV[3]) {
            double v[4] = {incM, incV[0], incV[1], incV[2]};
            group_reduce(g, lane, v);
            if (!active || lane != g.leader) return;
            const int t = ((ox + a) * ey + (oy + b)) * ez + (oz + c);
#pragma unroll
            for (int k = 0; k < 4; k++) atomicAdd(tile + k * tile_cap + t, v[k]);
        });
    } else if (active) {
        p2g_scatter(P, q, [&](int a, int b, int c, double incM, const double incV[3]) {
            const int t = ((ox + a) * ey + (oy + b)) * ez + (oz + c);
            atomicAdd(tile + t, incM);
            atomicAdd(tile + tile_cap + t, incV[0]);
            atomicAdd(tile + 2 * tile_cap + t, incV[1]);
            atomicAdd(tile + 3 * tile_cap + t, incV[2]);
        });
    }
    __syncthreads();
    // flush: consecutive threads take consecutive tile nodes (consecutive z)
    // of one array, so the global atomics of a warp fall on few sectors
    for (int k = threadIdx.x; k < 4 * nv; k += BLOCK) {
        const int comp = k / nv, t = k - comp * nv;
        const double v = tile[comp * tile_cap + t];
        if (v == 0.0) continue;
        const int tz = t % ez, ty = (t / ez) % ey, tx = t / (ez * ey);
        atomicAdd(grid + comp * P.gstride + node_index(P, blo[0] + tx, blo[1] + ty, blo[2] + tz), v);
    }
}

// Variant 4 (default): block fixed-point tile.
//
// A block takes a chunk of BLOCK*PPT consecutive particles of the sorted
// order. Their 27-node stencils fall in a small box of nodes, accumulated in
// shared memory as 64-bit integers: value v is stored as round(v * 2^e),
// with e chosen so that the box can absorb the chunk's contributions without
// overflow (a per-chunk bound on |contribution| measured in the previous
// launch, with margin). Integer sums are exact and order-independent, so the
// tile result does not depend on thread scheduling; the resolution 2^-e is
// ~2^-50 of the chunk's largest contribution, the rounding level of an FP64
// sum. Contributions beyond the bound (a particle that sped up, the first
// launch) go straight to the grid with FP64 atomics. The tile is converted
// back to FP64 and added to the grid once per node.
constexpr int kFxHeadroomBits = 10;          // up to 1024 contributions per node
constexpr double kFxMaxUnits = 4503599627370496.0;   // 2^52: |round(v 2^e)| limit

__device__ __forceinline__ int fx_exponent(double bound) {
    // smallest e with bound * 2^e <= 2^52 (bound includes a 4x margin)
    int ex;
    frexp(bound * 4.0, &ex);
    return 52 - ex;
}

template <int BLOCK, int PPT>
__global__ void __launch_bounds__(BLOCK, 2) k_p2g_fx_f64(DevParams P, const double* __restrict__ pts, size_t pitch,
                                                         int n, double* __restrict__ grid, int* err, int tile_cap,
                                                         float* __restrict__ chunk_bound) {
    extern __shared__ long long tl[];
    __shared__ float s_max;
    const int chunk0 = blockIdx.x * BLOCK * PPT;
    // pass A: node box of the chunk's stencils (positions only)
    int lo[3] = {INT_MAX, INT_MAX, INT_MAX}, hi[3] = {INT_MIN, INT_MIN, INT_MIN};
    for (int k = 0; k < PPT; k++) {
        const int i = chunk0 + k * BLOCK + threadIdx.x;
        if (i >= n) break;
        const long long util = __double_as_longlong(pts[i]);
        if (util & kDisabled) continue;
        int b[3];
#pragma unroll
        for (int d = 0; d < 3; d++) b[d] = (int)(pts[(MPM_POSX + d) * pitch + i] * P.h_inv - 0.5);
        if (stencil_error(P, b[0], b[1], b[2])) continue;
#pragma unroll
        for (int d = 0; d < 3; d++) { lo[d] = min(lo[d], b[d]); hi[d] = max(hi[d], b[d] + 2); }
    }
    int blo[3], bhi[3];
    block_box(lo, hi, blo, bhi);
    const bool have_box = blo[0] <= bhi[0];
    const int ex = have_box ? bhi[0] - blo[0] + 1 : 0, ey = have_box ? bhi[1] - blo[1] + 1 : 0,
              ez = have_box ? bhi[2] - blo[2] + 1 : 0;
    const long long vol = (long long)ex * ey * ez;
    const bool use_tile = have_box && vol <= tile_cap;
    const int nv = use_tile ? (int)vol : 0;
    if (threadIdx.x == 0) s_max = 0.f;
    for (int k = threadIdx.x; k < 4 * nv; k += BLOCK) {
        const int comp = k / nv;
        tl[comp * tile_cap + (k - comp * nv)] = 0;
    }
    __syncthreads();

    const double mmax = fmax(P.particle_mass, P.liquid_mass);
    const int e_m = fx_exponent(mmax);
    const float prev = chunk_bound[blockIdx.x];
    const int e_p = fx_exponent(prev > 0.f ? (double)prev : mmax * 16.0);
    const double s_m = ldexp(1.0, e_m), s_p = ldexp(1.0, e_p);
    float my_max = 0.f;

    // pass B: contributions
    for (int k = 0; k < PPT; k++) {
        const int i = chunk0 + k * BLOCK + threadIdx.x;
        if (i >= n) break;
        P2GPoint q;
        if (!p2g_prepare(P, pts, pitch, i, q, err)) continue;
        const bool in_tile = use_tile && !stencil_error(P, q.base[0], q.base[1], q.base[2]);
        if (!in_tile) {
            p2g_scatter(P, q, [&](int a, int b, int c, double incM, const double incV[3]) {
                const int x = q.base[0] + a, y = q.base[1] + b, z = q.base[2] + c;
                if (!node_inside(P, x, y, z)) return;
                grid_atomic_add(grid, P.gstride, node_index(P, x, y, z), incM, incV);
            });
            continue;
        }
        const int ox = q.base[0] - blo[0], oy = q.base[1] - blo[1], oz = q.base[2] - blo[2];
        p2g_scatter(P, q, [&](int a, int b, int c, double incM, const double incV[3]) {
            const int t = ((ox + a) * ey + (oy + b)) * ez + (oz + c);
            const double am = fmax(fabs(incV[0]), fmax(fabs(incV[1]), fabs(incV[2])));
            my_max = fmaxf(my_max, (float)am);
            if (am * s_p < kFxMaxUnits) {
                atomicAdd((unsigned long long*)(tl + tile_cap + t), (unsigned long long)__double2ll_rn(incV[0] * s_p));
                atomicAdd((unsigned long long*)(tl + 2 * tile_cap + t), (unsigned long long)__double2ll_rn(incV[1] * s_p));
                atomicAdd((unsigned long long*)(tl + 3 * tile_cap + t), (unsigned long long)__double2ll_rn(incV[2] * s_p));
            } else {
                const long long ni = node_index(P, q.base[0] + a, q.base[1] + b, q.base[2] + c);
                atomicAdd(grid + P.gstride + ni, incV[0]);
                atomicAdd(grid + 2 * P.gstride + ni, incV[1]);
                atomicAdd(grid + 3 * P.gstride + ni, incV[2]);
            }
            atomicAdd((unsigned long long*)(tl + t), (unsigned long long)__double2ll_rn(incM * s_m));
        });
    }
    // new bound of this chunk for the next launch
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) my_max = fmaxf(my_max, __shfl_xor_sync(0xffffffffu, my_max, o));
    if ((threadIdx.x & 31) == 0 && my_max > 0.f) atomicMax((int*)&s_max, __float_as_int(my_max));
    __syncthreads();
    if (threadIdx.x == 0) chunk_bound[blockIdx.x] = s_max;
    // flush: consecutive threads take consecutive tile nodes of one array
    const double inv_m = ldexp(1.0, -e_m), inv_p = ldexp(1.0, -e_p);
    for (int k = threadIdx.x; k < 4 * nv; k += BLOCK) {
        const int comp = k / nv, t = k - comp * nv;
        const long long u = tl[comp * tile_cap + t];
        if (u == 0) continue;
        const double v = (double)u * (comp == 0 ? inv_m : inv_p);
        const int tz = t % ez, ty = (t / ez) % ey, tx = t / (ez * ey);
        atomicAdd(grid + comp * P.gstride + node_index(P, blo[0] + tx, blo[1] + ty, blo[2] + tz), v);
    }
}

// ----------------------------------------------------------- grid update

// partition_kernel_update_nodes (mpm_kernels.cuh:138-232) for one partition:
// v = mv/m, gravity, speed clamp, cylindrical indenter contact with its force
// added to the angle x z sensor and to this substep's total, wall conditions.
// force3 receives the block-reduced force of this substep (3 doubles).
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_update_f64(DevParams P, double* __restrict__ grid, double ind_x, double ind_y,
                                                      double* __restrict__ sensor, double* __restrict__ force3) {
    const long long idx = (long long)blockIdx.x * BLOCK + threadIdx.x;
    double f[3] = {0, 0, 0};
    if (idx < P.nodes) {
        const double mass = grid[idx];
        if (mass != 0) {
            double v[3] = {grid[P.gstride + idx], grid[2 * P.gstride + idx], grid[3 * P.gstride + idx]};
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
            grid[P.gstride + idx] = v[0];
            grid[2 * P.gstride + idx] = v[1];
            grid[3 * P.gstride + idx] = v[2];
        }
    }
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

// The particle update after the gather (mpm_kernels.cuh:307-327).
template <class K>
__device__ __forceinline__ void g2p_advance(const DevParams& P, double pos[3], const double vel[3],
                                            const double C[3][3], double F[3][3], double& Jp_inv, long long& util,
                                            double p0, double& p_tr, double& q_tr) {
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
        return;
    }
    double Je;
    trial_pq(P, F, Je, p_tr, q_tr);
    if (!(util & kCrushed)) {
        if (outside_failure_surface(P, (short)util, p_tr, q_tr)) util |= kCrushed;
    }
    if (util & kCrushed) drucker_prager_return<K>(P, F, Jp_inv, Je, p_tr, q_tr, p0);
}

// partition_kernel_g2p without migration (mpm_kernels.cuh:237-351).
template <class K, int MINB>
__global__ void __launch_bounds__(128, MINB) k_g2p_f64(DevParams P, double* __restrict__ pts, size_t pitch, int n,
                                                 const double* __restrict__ grid, int record_pq,
                                                 const double* __restrict__ p0_arr, int* err) {
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
    const double p0 = p0_arr ? p0_arr[i] : P.p0;

    double vel[3], C[3][3];
    g2p_gather(P, grid, pos, vel, C, err);
    double p_tr, q_tr;
    g2p_advance<K>(P, pos, vel, C, F, Jp_inv, util, p0, p_tr, q_tr);

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

}  // namespace icempm
