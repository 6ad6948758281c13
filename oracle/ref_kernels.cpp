// CPU ORACLE — test infrastructure, not product code.
//
// Host build of the reference's own step kernels: this translation unit
// includes simulation/gpu_partition_3d.h, simulation/helper_math.cuh and
// simulation/mpm_kernels.cuh from the reference tree UNMODIFIED (include
// paths given by oracle/Makefile; nothing of them is copied here), with the
// stand-in headers of oracle/refshim/ in front of the reference's external
// dependencies (Eigen, rapidjson, HDF5, spdlog, CUDA headers), and supplies
// host definitions of the CUDA names the kernels use. Each exported ref_*
// function runs one kernel over its whole index range serially, one "thread"
// at a time in increasing index order (blockDim.x = 1), so the atomics of the
// kernels become plain additions in a fixed order.
//
// Host definitions (IEEE-754 semantics, not CUDA internals):
//   atomicAdd / atomicMax    plain read-modify-write when serial; a
//                            compare-and-swap loop when a ref_* call runs
//                            its index range over OpenMP threads (nthreads > 1)
//   rcbrt(x)                 1 / cbrt(x)
//   min / max                the usual comparisons
//   __fadd_rn / __fsub_rn    one correctly rounded float add / subtract
//   __frsqrt_rn              correctly rounded float 1/sqrt(x)
// The thread and block indices are thread-local, so a parallel call runs
// each index exactly once, as a launch does. This file is compiled with
// -ffp-contract=off: every product and sum is rounded separately. nvcc
// contracts a*b+c into fused multiply-adds in the reference's device build,
// so these outputs and the reference's GPU outputs can differ in the last
// bits; the tests compare within stated tolerances. The serial mode
// (nthreads <= 1) adds in increasing particle order and is deterministic;
// the parallel mode is what bench.py times as the reference's CPU arm.
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>

#define __global__
#define __device__
#define __host__
#define __constant__
#define __forceinline__ inline

struct RefThreadIndex {
    unsigned x, y, z;
};
static thread_local RefThreadIndex threadIdx = {0, 0, 0};
static thread_local RefThreadIndex blockIdx = {0, 0, 0};
static thread_local RefThreadIndex blockDim = {1, 1, 1};
static bool g_parallel = false;

static inline double atomicAdd(double* a, double v) {
    if (!g_parallel) {
        const double old = *a;
        *a = old + v;
        return old;
    }
    uint64_t* p = reinterpret_cast<uint64_t*>(a);
    uint64_t cur = __atomic_load_n(p, __ATOMIC_RELAXED);
    for (;;) {
        double old;
        std::memcpy(&old, &cur, sizeof(old));
        const double upd = old + v;
        uint64_t bits;
        std::memcpy(&bits, &upd, sizeof(bits));
        if (__atomic_compare_exchange_n(p, &cur, bits, true, __ATOMIC_RELAXED, __ATOMIC_RELAXED)) return old;
    }
}
static inline int atomicAdd(int* a, int v) {
    if (!g_parallel) {
        const int old = *a;
        *a = old + v;
        return old;
    }
    return __atomic_fetch_add(a, v, __ATOMIC_RELAXED);
}
static inline int atomicMax(int* a, int v) {
    if (!g_parallel) {
        const int old = *a;
        if (v > old) *a = v;
        return old;
    }
    int cur = __atomic_load_n(a, __ATOMIC_RELAXED);
    while (v > cur && !__atomic_compare_exchange_n(a, &cur, v, true, __ATOMIC_RELAXED, __ATOMIC_RELAXED)) {
    }
    return cur;
}
static inline double rcbrt(double x) { return 1.0 / std::cbrt(x); }
static inline int min(int a, int b) { return a < b ? a : b; }
static inline int max(int a, int b) { return a > b ? a : b; }
static inline double min(double a, double b) { return std::fmin(a, b); }
static inline double max(double a, double b) { return std::fmax(a, b); }
static inline float max(float a, float b) { return std::fmax(a, b); }
static inline float __fadd_rn(float a, float b) { return a + b; }
static inline float __fsub_rn(float a, float b) { return a - b; }
static inline float __frsqrt_rn(float x) { return (float)(1.0L / sqrtl((long double)x)); }

#include "gpu_partition_3d.h"
#include "helper_math.cuh"
#include "mpm_kernels.cuh"

namespace {
// Runs body(i) for i in [0, count): serially in increasing order, or over
// nthreads OpenMP threads (each with its own thread and block index).
template <class Body>
void launch(int count, int nthreads, Body body) {
    if (nthreads <= 1) {
        blockDim.x = 1;
        threadIdx.x = 0;
        for (int i = 0; i < count; i++) {
            blockIdx.x = (unsigned)i;
            body();
        }
        return;
    }
    g_parallel = true;
#pragma omp parallel num_threads(nthreads)
    {
        blockDim.x = 1;
        threadIdx.x = 0;
#pragma omp for schedule(static, 4096)
        for (int i = 0; i < count; i++) {
            blockIdx.x = (unsigned)i;
            body();
        }
    }
    g_parallel = false;
}
}  // namespace

extern "C" {

size_t ref_sizeof_params(void) { return sizeof(SimParams3D); }

// Byte offsets of fields spread over the struct, for a layout check against
// the product's SimParams3D: SetupType, GridXTotal, InitialTimeStep, mu,
// IndRSq, cellsize, ParticleMass, GridHaloSize, dt_vol_Dpinv, gbOffset,
// tpb_G2P, animation_threshold_pos.
void ref_params_layout(size_t out[12]) {
    out[0] = offsetof(SimParams3D, SetupType);
    out[1] = offsetof(SimParams3D, GridXTotal);
    out[2] = offsetof(SimParams3D, InitialTimeStep);
    out[3] = offsetof(SimParams3D, mu);
    out[4] = offsetof(SimParams3D, IndRSq);
    out[5] = offsetof(SimParams3D, cellsize);
    out[6] = offsetof(SimParams3D, ParticleMass);
    out[7] = offsetof(SimParams3D, GridHaloSize);
    out[8] = offsetof(SimParams3D, dt_vol_Dpinv);
    out[9] = offsetof(SimParams3D, gbOffset);
    out[10] = offsetof(SimParams3D, tpb_G2P);
    out[11] = offsetof(SimParams3D, animation_threshold_pos);
}

// GPU_Partition_3D::update_constants (gpu_partition_3d.cu:135-143): the
// parameter block into gprms, the error byte cleared.
int ref_set_params(const void* prms, size_t nbytes) {
    if (nbytes != sizeof(SimParams3D)) return -1;
    std::memcpy(&gprms, prms, sizeof(SimParams3D));
    gpu_error_indicator = 0;
    return 0;
}

int ref_error(void) { return (int)gpu_error_indicator; }
void ref_clear_error(void) { gpu_error_indicator = 0; }

// partition_kernel_p2g (mpm_kernels.cuh:20-100) over count_pts particles.
// Parallel mode: the kernel's atomics are CAS loops on the host, which
// serialise on the memory bus; instead particles are grouped by the x-window
// of their base node (windows of >= 3 cells, wider than a stencil) and the
// even windows run concurrently, then the odd ones. Two windows that run at
// the same time touch disjoint grid nodes, so the kernel's additions need no
// atomics; every particle is still one unmodified kernel invocation.
void ref_p2g(int gridX, int gridX_offset, int pitch_grid, int count_pts, int pitch_pts, const double* pts,
             double* grid, int nthreads) {
    auto body = [&] { partition_kernel_p2g(gridX, gridX_offset, pitch_grid, count_pts, pitch_pts, pts, grid); };
    if (nthreads <= 1 || count_pts == 0) {
        launch(count_pts, 1, body);
        return;
    }
    const double h_inv = gprms.cellsize_inv;
    const int halo = gprms.GridHaloSize;
    const int span = gridX + 2 * halo + 4;              // base x from -halo-2 up: window index >= 0
    const int width = std::max(3, span / (8 * nthreads));
    const int nwin = (span + width - 1) / width;
    std::vector<std::vector<int>> win(nwin);
    for (int i = 0; i < count_pts; i++) {
        const double x = pts[i + (size_t)pitch_pts * SimParams3D::posx];
        int bx = (int)(x * h_inv - 0.5) - gridX_offset + halo + 2;
        bx = std::min(std::max(bx, 0), span - 1);
        win[bx / width].push_back(i);
    }
    for (int parity = 0; parity < 2; parity++) {
#pragma omp parallel num_threads(nthreads)
        {
            blockDim.x = 1;
            threadIdx.x = 0;
#pragma omp for schedule(dynamic, 1)
            for (int w = parity; w < nwin; w += 2)
                for (int i : win[w]) {
                    blockIdx.x = (unsigned)i;
                    body();
                }
        }
    }
}

// partition_kernel_receive_halos_left, then _right (mpm_kernels.cuh:103-135),
// as GPU_Partition_3D::receive_halos launches them (gpu_partition_3d.cu:152-166)
void ref_receive_halos(int haloElementCount, int gridX_partition, int pitch_grid, double* grid, const double* halo0,
                       const double* halo1) {
    launch(haloElementCount, 1, [&] {
        partition_kernel_receive_halos_left(haloElementCount, gridX_partition, pitch_grid, grid, halo0, halo1);
    });
    launch(haloElementCount, 1, [&] {
        partition_kernel_receive_halos_right(haloElementCount, gridX_partition, pitch_grid, grid, halo0, halo1);
    });
}

// partition_kernel_update_nodes (mpm_kernels.cuh:138-232) over nNodes nodes;
// the indenter centre by value as in gpu_partition_3d.cu:250-253
void ref_update_nodes(double ind_x, double ind_y, int nNodes, int gridX_offset, int pitch_grid, double* grid,
                      double* sensor, int nthreads) {
    const Eigen::Vector2d centre(ind_x, ind_y);
    launch(nNodes, nthreads, [&] {
        partition_kernel_update_nodes(centre, nNodes, gridX_offset, pitch_grid, grid, sensor);
    });
}

// partition_kernel_g2p (mpm_kernels.cuh:237-399) over count_pts particles;
// utility receives the transfer counters (3 ints) when enablePointTransfer
void ref_g2p(int recordPQ, int enablePointTransfer, int gridX, int gridX_offset, int pitch_grid, int count_pts,
             int pitch_pts, double* pts, const double* grid, int* utility, int capacity_transfer, double* left,
             double* right, int nthreads) {
    launch(count_pts, nthreads, [&] {
        partition_kernel_g2p(recordPQ != 0, enablePointTransfer != 0, gridX, gridX_offset, pitch_grid, count_pts,
                             pitch_pts, pts, grid, utility, capacity_transfer, left, right);
    });
}

// partition_kernel_receive_points (mpm_kernels.cuh:411-427)
void ref_receive_points(int count_transfer, int count_pts, int pitch_pts, double* pts, double* transfer) {
    launch(count_transfer, 1,
           [&] { partition_kernel_receive_points(count_transfer, count_pts, pitch_pts, pts, transfer); });
}

}  // extern "C"
