// Stable cell-key sort of the particles on the device.
//
// HostSideSOA::RemoveDisabledAndSort (host_side_soa.cpp:56-67) removes
// disabled points and std::sorts the rest by ProxyPoint3D::getCellIndex
// (proxypoint3d.cpp:158-163): key = ix*GridY*GridZ + iy*GridZ + iz with
// i = (int)(x/h + 0.5). Here the same key is sorted stably (ties keep their
// previous order) by a counting sort, since keys are bounded integers:
//   1. bucket = key + halo*GridY*GridZ (so keys of points anywhere in the
//      halo-extended grid are >= 0); disabled points go to a last bucket
//      that is dropped; points outside the range raise MPM_ERR_SORT_RANGE;
//   2. histogram (atomics) and an exclusive scan give each bucket's start;
//   3. points are scattered to their bucket (atomic slots, unordered), then
//      each bucket's slot list is put back into increasing source order;
//   4. every particle array is gathered through the permutation.
#pragma once

#include "device_common.cuh"

namespace icempm {

struct SortGeom {
    int slab;          // GridY * GridZ
    int gz;
    int key_shift;     // halo * slab
    int nb;            // number of valid buckets; bucket nb = disabled
    double h_inv;
};

__global__ void k_sort_keys(SortGeom G, const double* __restrict__ pts, size_t pitch, int n,
                            int* __restrict__ bucket, int* __restrict__ count, int* err) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const long long util = __double_as_longlong(pts[i]);
    int b;
    if ((util & kDisabled) == kDisabled) {
        b = G.nb;
    } else {
        const double hx = pts[MPM_POSX * pitch + i] * G.h_inv + 0.5;
        const double hy = pts[(MPM_POSX + 1) * pitch + i] * G.h_inv + 0.5;
        const double hz = pts[(MPM_POSX + 2) * pitch + i] * G.h_inv + 0.5;
        const double lim = 1.0e9;
        if (!(fabs(hx) < lim && fabs(hy) < lim && fabs(hz) < lim)) {
            raise_error(err, MPM_ERR_SORT_RANGE);
            b = G.nb - 1;
        } else {
            const long long key = (long long)(int)hx * G.slab + (long long)(int)hy * G.gz + (int)hz;
            const long long bb = key + G.key_shift;
            if (bb < 0 || bb >= G.nb) {
                raise_error(err, MPM_ERR_SORT_RANGE);
                b = bb < 0 ? 0 : G.nb - 1;
            } else {
                b = (int)bb;
            }
        }
    }
    bucket[i] = b;
    atomicAdd(count + b, 1);
}

__global__ void k_sort_scatter(const int* __restrict__ bucket, int n, const int* __restrict__ start,
                               int* __restrict__ fill, unsigned* __restrict__ perm) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int b = bucket[i];
    const int slot = start[b] + atomicAdd(fill + b, 1);
    perm[slot] = (unsigned)i;
}

// Restores increasing source order inside every bucket (buckets hold a few
// points at the particle densities of MPM; insertion sort).
__global__ void k_sort_fix(int nb, const int* __restrict__ start, const int* __restrict__ count,
                           unsigned* __restrict__ perm) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nb) return;
    const int c = count[b];
    if (c < 2) return;
    unsigned* p = perm + start[b];
    for (int k = 1; k < c; k++) {
        const unsigned v = p[k];
        int j = k - 1;
        while (j >= 0 && p[j] > v) { p[j + 1] = p[j]; j--; }
        p[j + 1] = v;
    }
}

// dst[r*dpitch + k] = src[r*spitch + perm[k]] for rows r < nrows
template <typename T>
__global__ void k_gather_rows(const T* __restrict__ src, size_t spitch, T* __restrict__ dst, size_t dpitch,
                              int nrows, const unsigned* __restrict__ perm, int m) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= m) return;
    const unsigned s = perm[k];
    for (int r = blockIdx.y; r < nrows; r += gridDim.y) dst[(size_t)r * dpitch + k] = src[(size_t)r * spitch + s];
}

// ---------------------------------------------------------- exclusive scan
// Three-phase scan of int32 counts: per-block scan with block totals, a scan
// of the totals (recursively), and a uniform add.
constexpr int kScanBlock = 512;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanBlock * kScanItems;

__device__ __forceinline__ int block_exclusive_scan(int v, int* total) {
    __shared__ int warp_sums[kScanBlock / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[warp] = x;
    __syncthreads();
    if (warp == 0) {
        int w = lane < kScanBlock / 32 ? warp_sums[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < kScanBlock / 32) warp_sums[lane] = w;
    }
    __syncthreads();
    const int warp_off = warp ? warp_sums[warp - 1] : 0;
    *total = warp_sums[kScanBlock / 32 - 1];
    __syncthreads();
    return warp_off + x - v;
}

__global__ void __launch_bounds__(kScanBlock) k_scan_tiles(const int* __restrict__ in, int* __restrict__ out,
                                                            int n, int* __restrict__ tile_sums) {
    const long long base = (long long)blockIdx.x * kScanTile + (long long)threadIdx.x * kScanItems;
    int v[kScanItems];
    int s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; k++) {
        v[k] = (base + k < n) ? in[base + k] : 0;
        s += v[k];
    }
    int total;
    int off = block_exclusive_scan(s, &total);
#pragma unroll
    for (int k = 0; k < kScanItems; k++) {
        if (base + k < n) out[base + k] = off;
        off += v[k];
    }
    if (threadIdx.x == 0 && tile_sums) tile_sums[blockIdx.x] = total;
}

__global__ void k_scan_add(int* __restrict__ out, int n, const int* __restrict__ tile_offsets) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[i] += tile_offsets[i / kScanTile];
}

}  // namespace icempm
