// Kernels of the x-slab partitions (GPU_Implementation6 with nPartitions > 1):
// adding a neighbour's halo slabs into the grid, and moving the particles that
// left a partition's slab to the neighbour's particle list.
//
// Each partition keeps a grid for the whole domain (B200 HBM holds it many
// times over) and works on its window of it: the columns x0 - halo .. x0 +
// gxp + halo - 1. Node indices are therefore the same in every partition, and
// a halo exchange is a copy of the same node range between two grids.
#pragma once

#include "device_common.cuh"
#include "kernels_mixed.cuh"

namespace icempm {

// partition_kernel_receive_halos_left/_right (mpm_kernels.cuh:103-135): the
// 4 FP64 arrays of hn nodes from a neighbour's packed slabs (array c at c*hn)
// added into this grid at node offset off.
__global__ void k_halo_add_f64(double* __restrict__ grid, long long gstride, long long off, int hn,
                               const double* __restrict__ src) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= hn) return;
#pragma unroll
    for (int c = 0; c < 4; c++) grid[c * gstride + off + i] += src[(size_t)c * hn + i];
}

// The same for the mixed accumulator {m, m v} (float4 per node).
__global__ void k_halo_add_f4(float4* __restrict__ acc, long long off, int hn, const float4* __restrict__ src) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= hn) return;
    const float4 a = acc[off + i], b = src[i];
    acc[off + i] = make_float4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w);
}

// The same for the fixed-point accumulator (4 int64 per node): an exact sum.
__global__ void k_halo_add_q(unsigned long long* __restrict__ acc, long long off, int hn,
                             const unsigned long long* __restrict__ src) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 4 * hn) return;
    acc[4 * off + i] += src[i];
}

// One particle record of a point transfer. FP64 handles: 32 doubles (the
// 28 SoA rows, the apex shift p0, the upload id as bits, 2 unused); mixed
// handles: 32 words (the 28 rows of the mixed state, p0 as a double in two
// words, the upload id, 1 unused). 256 / 128 bytes, so records stay aligned.
constexpr int kRecWords = 32;

struct XferGeom {
    int x0, gxp;        // the partition's columns [x0, x0 + gxp)
    int keep_track;     // halo / 2 - 1 (mpm_kernels.cuh:361)
    int cap;            // records per direction (VectorCapacity_transfer)
    int left_ok, right_ok;   // a neighbour exists on that side
    double h_inv;
};

// The transfer part of partition_kernel_g2p (mpm_kernels.cuh:353-398) for one
// particle with base x-node bx: tracks the deviation beyond the slab
// (counters[2], atomic max) and returns -1 / +1 when the particle flies to the
// left / right neighbour (more than 3 cells past the slab), else 0.
__device__ __forceinline__ int transfer_side(const XferGeom& G, int bx, int* counters) {
    if (bx - G.x0 < -G.keep_track) atomicMax(counters + 2, -(bx - G.x0));
    else if (bx - (G.x0 + G.gxp - 3) > G.keep_track) atomicMax(counters + 2, bx - (G.x0 + G.gxp - 3));
    constexpr int fly = 3;
    if (bx - G.x0 < -fly && G.left_ok) return -1;
    if (bx - (G.x0 + G.gxp - 3) > fly && G.right_ok) return 1;
    return 0;
}

// Reserves a slot in the side's buffer; -1 when it is full (the reference
// then pins the counter at the capacity and keeps the particle,
// mpm_kernels.cuh:383-384,395-396).
__device__ __forceinline__ int transfer_slot(const XferGeom& G, int side, int* counters) {
    int* c = counters + (side < 0 ? 0 : 1);
    const int k = atomicAdd(c, 1);
    if (k < G.cap) return k;
    atomicMin(c, G.cap);
    return -1;
}

// FP64 SoA: the particles leaving the slab are copied to the left / right
// record buffers and disabled (the whole status word set to the disabled
// bit, as mpm_kernels.cuh:381,393).
__global__ void k_points_out_f64(XferGeom G, double* __restrict__ pts, size_t pitch, const double* __restrict__ p0,
                                 const unsigned* __restrict__ ids, int n, double* __restrict__ left,
                                 double* __restrict__ right, int* __restrict__ counters) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const long long util = __double_as_longlong(pts[i]);
    if ((util & kDisabled) == kDisabled) return;
    const int bx = (int)(pts[MPM_POSX * pitch + i] * G.h_inv - 0.5);
    const int side = transfer_side(G, bx, counters);
    if (side == 0) return;
    const int k = transfer_slot(G, side, counters);
    if (k < 0) return;
    double* rec = (side < 0 ? left : right) + (size_t)k * kRecWords;
#pragma unroll 4
    for (int r = 0; r < MPM_N_PTS_ARRAYS; r++) rec[r] = pts[r * pitch + i];
    rec[28] = p0 ? p0[i] : 0.0;
    rec[29] = __longlong_as_double((long long)ids[i]);
    pts[i] = __longlong_as_double(kDisabled);
}

// partition_kernel_receive_points (mpm_kernels.cuh:411-427) for FP64 SoA:
// records appended at particle index n0 (the caller checked the capacity).
__global__ void k_points_in_f64(double* __restrict__ pts, size_t pitch, double* __restrict__ p0,
                                unsigned* __restrict__ ids, int n0, int count, const double* __restrict__ recs) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count) return;
    const int i = n0 + k;
    const double* rec = recs + (size_t)k * kRecWords;
#pragma unroll 4
    for (int r = 0; r < MPM_N_PTS_ARRAYS; r++) pts[r * pitch + i] = rec[r];
    if (p0) p0[i] = rec[28];
    ids[i] = (unsigned)__double_as_longlong(rec[29]);
}

// The same for the mixed state (28 rows of 4-byte words; base x from the
// fixed-point position, as fix_base computes it for the kernels).
__global__ void k_points_out_mixed(XferGeom G, unsigned* __restrict__ mx, size_t pitch, const double* __restrict__ p0,
                                   const unsigned* __restrict__ ids, int n, unsigned* __restrict__ left,
                                   unsigned* __restrict__ right, int* __restrict__ counters) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int st = (int)mx[25 * pitch + i];
    if ((st & (int)kDisabled) == (int)kDisabled) return;
    int bx;
    float fx;
    fix_base((int)mx[i], bx, fx);
    const int side = transfer_side(G, bx, counters);
    if (side == 0) return;
    const int k = transfer_slot(G, side, counters);
    if (k < 0) return;
    unsigned* rec = (side < 0 ? left : right) + (size_t)k * kRecWords;
#pragma unroll 4
    for (int r = 0; r < MPM_N_PTS_ARRAYS; r++) rec[r] = mx[r * pitch + i];
    const unsigned long long pb = p0 ? (unsigned long long)__double_as_longlong(p0[i]) : 0ull;
    rec[28] = (unsigned)pb;
    rec[29] = (unsigned)(pb >> 32);
    rec[30] = ids[i];
    mx[25 * pitch + i] = (unsigned)kDisabled;
}

__global__ void k_points_in_mixed(unsigned* __restrict__ mx, size_t pitch, double* __restrict__ p0,
                                  float* __restrict__ p0f, unsigned* __restrict__ ids, int n0, int count,
                                  const unsigned* __restrict__ recs) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count) return;
    const int i = n0 + k;
    const unsigned* rec = recs + (size_t)k * kRecWords;
#pragma unroll 4
    for (int r = 0; r < MPM_N_PTS_ARRAYS; r++) mx[r * pitch + i] = rec[r];
    const double v = __longlong_as_double((long long)(((unsigned long long)rec[29] << 32) | rec[28]));
    if (p0) p0[i] = v;
    if (p0f) p0f[i] = (float)v;
    ids[i] = rec[30];
}

}  // namespace icempm
