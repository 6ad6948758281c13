// C-ABI of the single-partition MLS-MPM step (declared in include/icempm_b200.h).
//
// One handle = one partition on one device: particle SoA, grid, sensor array
// and scratch, all on one stream. The substep sequence and the bookkeeping of
// SimulationTime / SimulationStep follow Model3D::Step (model_3d.cpp:35-51)
// and GPU_Implementation6 (gpu_implementation6.cpp); the kernels are in the
// kernels_*.cuh / sort.cuh headers.

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <algorithm>
#include <cstring>
#include <mutex>
#include <new>
#include <vector>

#include <cuda.h>
#include <cuda_runtime.h>

#include "../../include/icempm_b200.h"
#include "../../include/icempm_b200_testing.h"
#include "device_common.cuh"
#include "kernels_f64.cuh"
#include "kernels_mixed.cuh"
#include "adjoint_f64.cuh"
#include "sort.cuh"
#include "frames.cuh"
#include "partition.cuh"

using namespace icempm;

namespace {
__global__ void k_narrow(const double* __restrict__ src, float* __restrict__ dst, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = (float)src[i];
}
// p0 = c / tan(phi) in place (and its FP32 copy for the mixed state)
__global__ void k_cohesion_to_apex(double* __restrict__ p0, float* __restrict__ p0f, int n, double tan_phi) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double v = p0[i] / tan_phi;
    p0[i] = v;
    if (p0f) p0f[i] = (float)v;
}
// ids = base, base + 1, ..., base + n - 1 (the upload order)
__global__ void k_iota(unsigned* __restrict__ ids, int n, unsigned base) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) ids[i] = base + (unsigned)i;
}
}  // namespace

struct mpm_handle {
    SimParams3D prms;
    DevParams dp;
    int precision = MPM_PRECISION_FP64;
    int device = 0;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    unsigned capacity = 0;
    unsigned n = 0;
    size_t pitch = 0;                 // doubles per SoA row on the device
    bool uploaded = false;

    double* pts = nullptr;            // 28 rows x pitch
    double* p0 = nullptr;             // per-particle apex shift (optional)
    unsigned* ids = nullptr;          // upload index of each particle
    double* grid = nullptr;           // AoS {m, mv} per node
    double* sensor = nullptr;         // 3 * subdiv * Gz
    double* force_steps = nullptr;    // 3 per substep of the running mpm_step
    int force_steps_cap = 0;
    double* force_phase = nullptr;    // 3, substep force of the phase API
    int* err = nullptr;

    // sort scratch (allocated on first sort)
    double* pts_alt = nullptr;
    double* p0_alt = nullptr;
    unsigned* ids_alt = nullptr;
    int* s_bucket = nullptr;
    int* s_count = nullptr;
    int* s_start = nullptr;
    unsigned* s_perm = nullptr;
    std::vector<int*> scan_levels;    // per-level tile sums and their scans
    std::vector<int> scan_sizes;
    int sort_interval = 0;
    int steps_since_sort = 0;

    // mixed precision (MPM_PRECISION_MIXED): 28 rows of 4-byte words
    // (X 0-2, v 3-5, E 6-14, C 15-23, Jp 24, status 25, P 26, Q 27); the FP64
    // SoA `pts` is then the staging copy for upload, download and sort
    void* mx = nullptr;
    float* p0f = nullptr;
    float4* gacc = nullptr;
    unsigned long long* gacc_q = nullptr;   // the fixed-point accumulator when selected (4 per node)
    float4* gvel = nullptr;
    bool p2g_ready = false;           // gacc holds the P2G of the current state
    int num_sms = 148;
    int* rm_list = nullptr;           // crushed points deferred to k_return_map_mixed (n entries)
    int* rm_counts = nullptr;         // two list counters, used alternately by successive launches
    int rm_parity = 0;

    // adjoint (FP64 modes): checkpoints of the recorded forward run
    std::vector<double*> ckpt;        // particle state at substeps 0, k, 2k, ...
    std::vector<SimParams3D> ckpt_prms;
    std::vector<double*> seg;         // states of one segment during the reverse sweep
    double* adj_A = nullptr;          // ADJ_ROWS x pitch particle adjoints
    double* adj_cgrad = nullptr;      // dL/dc per particle
    double* adj_Egrad = nullptr;      // dL/dE
    double* adj_g7 = nullptr;         // recomputed grid: m, P, final v (7 x gstride)
    double* adj_gb7 = nullptr;        // grid adjoints: vb, mb, Pb (7 x gstride)
    int adj_steps = 0, adj_every = 0;
    bool adj_ready = false;
    double* adj_force = nullptr;      // force history of a mixed adjoint forward (3 per substep)
    int adj_force_cap = 0;
    std::vector<double*> adj_gcache;  // P2G grid of each substep of the segment being reversed
    double* adj_rmv = nullptr;        // return-map VJP of the crushed points (10 x pitch)


    // animation-frame records (mpm_frame_records), allocated on first use
    float* fr_f = nullptr;            // visual state: pos 3, vel 3, Jp_inv rows x pitch
    unsigned char* fr_status = nullptr;
    int* fr_last = nullptr;           // frame of each visual point's last position refresh
    int* fr_i = nullptr;              // keep, rank, 3 flags, 3 offsets: 8 x (pitch + 1)
    unsigned char* fr_rec = nullptr;  // records: 44 bytes x pitch
    std::vector<int*> fr_scan_levels;
    bool fr_ready = false;            // a full frame has built the visual state
    cudaError_t last_cuda = cudaSuccess;

    // x-slab partition (mpm_set_partition); whole grid when part_gxp == 0
    int part_id = 0, part_x0 = 0, part_gxp = 0;
    unsigned id_base = 0;             // upload index of particle 0 (ids are global across partitions)
    int* xfer = nullptr;              // point transfer counters: to the left, to the right, max deviation
};

namespace {

thread_local char g_last_error[256] = "";

int cuda_fail(mpm_handle* h, cudaError_t e, const char* what) {
    if (h) h->last_cuda = e;
    std::snprintf(g_last_error, sizeof(g_last_error), "%s: %s", what, cudaGetErrorString(e));
    return MPM_ERR_CUDA;
}

#define CK(h, call)                                              \
    do {                                                         \
        cudaError_t e_ = (call);                                 \
        if (e_ != cudaSuccess) return cuda_fail((h), e_, #call); \
    } while (0)

#define CK_LAUNCH(h, what)                                      \
    do {                                                        \
        cudaError_t e_ = cudaGetLastError();                    \
        if (e_ != cudaSuccess) return cuda_fail((h), e_, what); \
    } while (0)

DevParams make_dev_params(const SimParams3D& p) {
    DevParams d;
    std::memset(&d, 0, sizeof(d));
    d.Gx = p.GridXTotal;
    d.Gy = p.GridY;
    d.Gz = p.GridZ;
    d.halo = p.GridHaloSize;
    d.setup_type = p.SetupType;
    d.subdiv = p.IndenterSubdivisions;
    d.slab = (long long)p.GridY * p.GridZ;
    d.inv_gz = 1.0 / (double)p.GridZ;
    d.inv_gy = 1.0 / (double)p.GridY;
    d.nodes = (long long)(p.GridXTotal + 2 * p.GridHaloSize) * d.slab;
    // one partition: the window is the whole grid (set_window narrows it)
    d.win_lo = -p.GridHaloSize;
    d.win_hi = p.GridXTotal + p.GridHaloSize - 3;
    d.own_lo = -p.GridHaloSize;
    d.own_hi = p.GridXTotal + p.GridHaloSize;
    d.node_lo = 0;
    d.node_hi = (int)d.nodes;
    d.gstride = (d.nodes + 31) / 32 * 32;
    d.h = p.cellsize;
    d.h_inv = p.cellsize_inv;
    d.dt = p.InitialTimeStep;
    d.particle_mass = p.ParticleMass;
    d.liquid_mass = p.LiquidParticleMass;
    d.dt_vol_Dpinv = p.dt_vol_Dpinv;
    d.dt_gravity = p.dt_Gravity;
    d.vmax = p.vmax;
    d.vmax_sq = p.vmax_squared;
    d.ind_rsq = p.IndRSq;
    d.ind_velocity = p.IndVelocity;
    d.mu = p.mu;
    d.kappa = p.kappa;
    d.pmax = p.IceCompressiveStrength;
    d.tensile = p.IceTensileStrength;
    d.shear = p.IceShearStrength;
    d.tensile2 = p.IceTensileStrength2;
    d.beta = p.NACC_beta;
    d.grain_var = p.GrainVariability;
    d.tan_phi = p.DP_tan_phi;
    d.p0 = p.DP_threshold_p;
    d.drag = p.DragGlobal;
    {   // GetParametersForGrain with var2 = var3 = 1 (mpm_kernels.cuh:434-450)
        const double pmax = p.IceCompressiveStrength, pmin = -p.IceTensileStrength, qmax = p.IceShearStrength;
        const double pmin2 = -p.IceTensileStrength2, beta = p.NACC_beta;
        const double q0 = 2 * std::sqrt(-pmax * pmin) * qmax / (pmax - pmin);
        d.fs_pmin2 = (float)pmin2;
        d.fs_k = (float)(-q0 / pmin2);
        d.fs_msq = (float)((4 * qmax * qmax * (1 + 2 * beta)) / ((pmax - pmin) * (pmax - pmin)));
        d.fs_1p2b = (float)(1. + 2. * beta);
        d.fs_bpmax = (float)(beta * pmax);
        d.fs_pmax = (float)pmax;
    }
    d.f_h = (float)p.cellsize;
    d.f_h_inv = (float)p.cellsize_inv;
    d.f_s4 = 4.0f * d.f_h_inv;
    d.f_dt = (float)p.InitialTimeStep;
    d.f_adv = d.f_dt * d.f_h_inv * kFixScale;
    d.f_mu = (float)p.mu;
    d.f_kappa = (float)p.kappa;
    d.f_hkappa = (float)(0.5 * p.kappa);
    d.f_qmu = (float)(kCoeff1 * p.mu);
    d.f_pmass = (float)p.ParticleMass;
    d.f_lmass = (float)p.LiquidParticleMass;
    d.f_dvd = (float)p.dt_vol_Dpinv;
    {   // fixed-point accumulator scales: 2^44 units per reference mass and
        // per reference momentum (the larger particle mass at vmax)
        double m_ref = std::max(p.ParticleMass, p.LiquidParticleMass);
        if (!(m_ref > 0)) m_ref = 1.0;
        const double v_ref = p.vmax > 0 ? p.vmax : 1.0;
        const double two44 = 17592186044416.0;
        d.f_qm = (float)(two44 / m_ref);
        d.f_qp = (float)(two44 / (m_ref * v_ref));
        d.q_inv_m = 1.0 / (double)d.f_qm;
        d.q_inv_p = 1.0 / (double)d.f_qp;
    }
    return d;
}

bool params_valid(const SimParams3D* p) {
    return p && p->GridXTotal > 0 && p->GridY > 0 && p->GridZ > 0 && p->GridHaloSize >= 0 && p->cellsize > 0 &&
           p->InitialTimeStep > 0 && p->IndenterSubdivisions > 0 && p->UpdateEveryNthStep > 0;
}

inline unsigned blocks_for(long long n, int tpb) { return (unsigned)((n + tpb - 1) / tpb); }

void free_all(mpm_handle* h) {
    cudaFree(h->pts); cudaFree(h->p0); cudaFree(h->ids); cudaFree(h->grid); cudaFree(h->sensor);
    cudaFree(h->force_steps); cudaFree(h->force_phase); cudaFree(h->err);
    cudaFree(h->pts_alt); cudaFree(h->p0_alt); cudaFree(h->ids_alt);
    cudaFree(h->s_bucket); cudaFree(h->s_count); cudaFree(h->s_start); cudaFree(h->s_perm);
    cudaFree(h->mx); cudaFree(h->p0f); cudaFree(h->gacc); cudaFree(h->gvel); cudaFree(h->gacc_q);
    cudaFree(h->rm_list); cudaFree(h->rm_counts); cudaFree(h->xfer);
    for (double* c : h->ckpt) cudaFree(c);
    for (double* c : h->seg) cudaFree(c);
    h->ckpt.clear();
    h->seg.clear();
    cudaFree(h->adj_A); cudaFree(h->adj_cgrad); cudaFree(h->adj_Egrad); cudaFree(h->adj_g7); cudaFree(h->adj_gb7);
    cudaFree(h->adj_force);
    for (double* c : h->adj_gcache) cudaFree(c);
    h->adj_gcache.clear();
    cudaFree(h->adj_rmv);
    for (int* p : h->scan_levels) cudaFree(p);
    h->scan_levels.clear();
    cudaFree(h->fr_f); cudaFree(h->fr_status); cudaFree(h->fr_last); cudaFree(h->fr_i); cudaFree(h->fr_rec);
    for (int* p : h->fr_scan_levels) cudaFree(p);
    h->fr_scan_levels.clear();
    if (h->own_stream) cudaStreamDestroy(h->own_stream);
}

size_t sensor_count(const SimParams3D& p) { return (size_t)3 * p.IndenterSubdivisions * p.GridZ; }

bool is_mixed(const mpm_handle* h) { return h->precision == MPM_PRECISION_MIXED; }

MixedState mixed_state(mpm_handle* h) {
    MixedState m;
    int* wi = static_cast<int*>(h->mx);
    float* wf = static_cast<float*>(h->mx);
    const size_t p = h->pitch;
    m.X = wi;
    m.v = wf + 3 * p;
    m.E = wf + 6 * p;
    m.C = wf + 15 * p;
    m.Jpm1 = wf + 24 * p;
    m.status = wi + 25 * p;
    m.PQ = wf + 26 * p;
    m.p0 = h->p0f;
    m.pitch = p;
    return m;
}

// staging (FP64 SoA) -> mixed state; p0 (FP64) -> p0f
int mixed_from_staging(mpm_handle* h) {
    if (!h->n) return MPM_OK;
    k_mixed_from_f64<<<blocks_for(h->n, 256), 256, 0, h->stream>>>(h->pts, h->pitch, (int)h->n, mixed_state(h),
                                                                  h->prms.cellsize_inv);
    CK_LAUNCH(h, "mixed from f64");
    if (h->p0) {
        if (!h->p0f) CK(h, cudaMalloc(&h->p0f, sizeof(float) * h->pitch));
        k_narrow<<<blocks_for(h->n, 256), 256, 0, h->stream>>>(h->p0, h->p0f, (int)h->n);
        CK_LAUNCH(h, "p0 narrow");
    }
    return MPM_OK;
}

int mixed_to_staging(mpm_handle* h) {
    if (!h->n) return MPM_OK;
    k_mixed_to_f64<<<blocks_for(h->n, 256), 256, 0, h->stream>>>(mixed_state(h), (int)h->n, h->pts, h->pitch,
                                                                h->prms.cellsize);
    CK_LAUNCH(h, "mixed to f64");
    return MPM_OK;
}

// ---------------------------------------------------------------- phases

int launch_p2g(mpm_handle* h) {
    const int n = (int)h->n;
    if (n == 0) return MPM_OK;
    if (is_mixed(h)) {
        if (h->gacc_q)
            k_p2g_mixed<<<blocks_for(n, 128), 128, 0, h->stream>>>(h->dp, mixed_state(h), n, AccQ{h->gacc_q}, h->err);
        else
            k_p2g_mixed<<<blocks_for(n, 128), 128, 0, h->stream>>>(h->dp, mixed_state(h), n, AccF4{h->gacc}, h->err);
        CK_LAUNCH(h, "p2g mixed");
        return MPM_OK;
    }
    k_p2g_pairs_f64<<<blocks_for(n, 128), 128, 0, h->stream>>>(h->dp, h->pts, h->pitch, n, h->grid, h->err);
    CK_LAUNCH(h, "p2g kernel");
    return MPM_OK;
}

int launch_update(mpm_handle* h, double ind_x, double ind_y, double* force3) {
    // the nodes of the partition's window (one partition: the whole grid), two per thread
    if (is_mixed(h)) {
        const unsigned nbm = blocks_for((long long)h->dp.node_hi - h->dp.node_lo, 256 * kUpdateNodesPerThread);
        if (h->gacc_q)
            k_update_mixed<256><<<nbm, 256, 0, h->stream>>>(h->dp, AccQ{h->gacc_q}, h->gvel, ind_x, ind_y, h->sensor,
                                                           force3);
        else
            k_update_mixed<256><<<nbm, 256, 0, h->stream>>>(h->dp, AccF4{h->gacc}, h->gvel, ind_x, ind_y, h->sensor,
                                                           force3);
        CK_LAUNCH(h, "update mixed");
        return MPM_OK;
    }
    k_update_f64<256><<<blocks_for((long long)h->dp.node_hi - h->dp.node_lo, 256 * kUpdateF64NodesPerThread), 256, 0,
                         h->stream>>>(
        h->dp, h->grid, ind_x, ind_y, h->sensor, force3);
    CK_LAUNCH(h, "update kernel");
    return MPM_OK;
}

// Return map and P2G of the crushed points the last fused launch listed
// (one persistent grid of 4 blocks per SM walks the list).
int launch_return_map_mixed(mpm_handle* h, int do_p2g) {
    const int cur = h->rm_parity;
    h->rm_parity ^= 1;
    if (h->gacc_q)
        k_return_map_mixed<<<h->num_sms * 4, 128, 0, h->stream>>>(h->dp, mixed_state(h), h->rm_list,
                                                                  h->rm_counts + cur, h->rm_counts + (cur ^ 1),
                                                                  AccQ{h->gacc_q}, do_p2g, h->err);
    else
        k_return_map_mixed<<<h->num_sms * 4, 128, 0, h->stream>>>(h->dp, mixed_state(h), h->rm_list,
                                                                  h->rm_counts + cur, h->rm_counts + (cur ^ 1),
                                                                  AccF4{h->gacc}, do_p2g, h->err);
    CK_LAUNCH(h, "return map mixed");
    return MPM_OK;
}

// Fused G2P -> P2G of all particles but the crushed ones, which it lists for
// launch_return_map_mixed (the caller launches that next, on the same
// stream). store_vc: write v and C to the state (needed before a download, a
// sort or a standalone P2G; the fused chain itself does not read them back).
int launch_g2p2g_mixed(mpm_handle* h, int do_p2g, int record_pq, int store_vc) {
    const int n = (int)h->n;
    if (n == 0) return MPM_OK;
    int* const rm_count = h->rm_counts + h->rm_parity;
    // the warps' velocity boxes: kVBoxNodes float4 of dynamic shared memory per warp
    const size_t vsm = sizeof(float4) * (kFusedBlock / 32) * kVBoxNodes;
    if (h->gacc_q)
        k_g2p2g_mixed<<<blocks_for(n, kFusedBlock), kFusedBlock, vsm, h->stream>>>(
            h->dp, mixed_state(h), n, h->gvel, AccQ{h->gacc_q}, do_p2g, record_pq, store_vc, h->err, h->rm_list,
            rm_count);
    else
        k_g2p2g_mixed<<<blocks_for(n, kFusedBlock), kFusedBlock, vsm, h->stream>>>(
            h->dp, mixed_state(h), n, h->gvel, AccF4{h->gacc}, do_p2g, record_pq, store_vc, h->err, h->rm_list,
            rm_count);
    CK_LAUNCH(h, "g2p2g mixed");
    return MPM_OK;
}

int launch_g2p(mpm_handle* h, int record_pq) {
    const int n = (int)h->n;
    if (n == 0) return MPM_OK;
    if (is_mixed(h)) {
        int r = launch_g2p2g_mixed(h, 0, record_pq, 1);
        return r ? r : launch_return_map_mixed(h, 0);
    }
    const unsigned nb = blocks_for(n, 128);
    const int cur = h->rm_parity;
    h->rm_parity ^= 1;
    int* const cnt = h->rm_counts + cur;
    int* const next = h->rm_counts + (cur ^ 1);
    const int rb = h->num_sms * 4;
    if (h->precision == MPM_PRECISION_FP64) {
        k_g2p_f64<SvdF32><<<nb, 128, 0, h->stream>>>(h->dp, h->pts, h->pitch, n, h->grid, record_pq, h->err,
                                                    h->rm_list, cnt);
        k_return_map_f64<SvdF32><<<rb, 128, 0, h->stream>>>(h->dp, h->pts, h->pitch, h->p0, h->rm_list, cnt, next);
    } else {
        k_g2p_f64<SvdF64><<<nb, 128, 0, h->stream>>>(h->dp, h->pts, h->pitch, n, h->grid, record_pq, h->err,
                                                    h->rm_list, cnt);
        k_return_map_f64<SvdF64><<<rb, 128, 0, h->stream>>>(h->dp, h->pts, h->pitch, h->p0, h->rm_list, cnt, next);
    }
    CK_LAUNCH(h, "g2p kernel");
    return MPM_OK;
}

int reset_grid(mpm_handle* h) {
    if (is_mixed(h)) {
        if (h->gacc_q)
            CK(h, cudaMemsetAsync(h->gacc_q, 0, sizeof(unsigned long long) * 4 * (size_t)h->dp.nodes, h->stream));
        else
            CK(h, cudaMemsetAsync(h->gacc, 0, sizeof(float4) * (size_t)h->dp.nodes, h->stream));
        h->p2g_ready = false;
        return MPM_OK;
    }
    if (h->dp.node_lo == 0 && h->dp.node_hi == h->dp.nodes) {
        CK(h, cudaMemsetAsync(h->grid, 0, sizeof(double) * 4 * (size_t)h->dp.gstride, h->stream));
        return MPM_OK;
    }
    // a partition clears its window's slabs of the 4 arrays
    const size_t cnt = (size_t)(h->dp.node_hi - h->dp.node_lo);
    for (int c = 0; c < 4; c++)
        CK(h, cudaMemsetAsync(h->grid + c * h->dp.gstride + h->dp.node_lo, 0, sizeof(double) * cnt, h->stream));
    return MPM_OK;
}

int read_error(mpm_handle* h, int* code) {
    CK(h, cudaMemcpyAsync(code, h->err, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    CK(h, cudaStreamSynchronize(h->stream));
    return MPM_OK;
}

// ------------------------------------------------------------------ sort

int ensure_sort_scratch(mpm_handle* h) {
    if (h->s_bucket) return MPM_OK;
    const SimParams3D& p = h->prms;
    const long long nb = (long long)(p.GridXTotal + 2 * p.GridHaloSize + 1) * p.GridY * p.GridZ;
    if (nb + 1 > 0x7fffffffLL) return MPM_ERR_ARG;
    CK(h, cudaMalloc(&h->pts_alt, sizeof(double) * MPM_N_PTS_ARRAYS * h->pitch));
    CK(h, cudaMalloc(&h->ids_alt, sizeof(unsigned) * h->pitch));
    CK(h, cudaMalloc(&h->s_bucket, sizeof(int) * h->pitch));
    CK(h, cudaMalloc(&h->s_perm, sizeof(unsigned) * h->pitch));
    CK(h, cudaMalloc(&h->s_count, sizeof(int) * (nb + 1)));
    CK(h, cudaMalloc(&h->s_start, sizeof(int) * (nb + 1)));
    long long m = nb + 1;
    while (m > kScanTile) {
        m = (m + kScanTile - 1) / kScanTile;
        int* sums = nullptr;
        int* scanned = nullptr;
        CK(h, cudaMalloc(&sums, sizeof(int) * m));
        CK(h, cudaMalloc(&scanned, sizeof(int) * m));
        h->scan_levels.push_back(sums);
        h->scan_levels.push_back(scanned);
        h->scan_sizes.push_back((int)m);
    }
    return MPM_OK;
}

// Exclusive scan of n ints; `levels` holds the tile sums and their scans of
// each level, sized for at least n (default: the sort's, sized for the cells).
int exclusive_scan(mpm_handle* h, const int* in, int* out, int n, size_t level,
                   const std::vector<int*>* levels = nullptr) {
    const std::vector<int*>& lv = levels ? *levels : h->scan_levels;
    const int tiles = (n + kScanTile - 1) / kScanTile;
    int* sums = tiles > 1 ? lv[2 * level] : nullptr;
    k_scan_tiles<<<tiles, kScanBlock, 0, h->stream>>>(in, out, n, sums);
    CK_LAUNCH(h, "scan tiles");
    if (tiles > 1) {
        int* scanned = lv[2 * level + 1];
        int r = exclusive_scan(h, sums, scanned, tiles, level + 1, levels);
        if (r) return r;
        k_scan_add<<<blocks_for(n, 256), 256, 0, h->stream>>>(out, n, scanned);
        CK_LAUNCH(h, "scan add");
    }
    return MPM_OK;
}

int do_sort_f64(mpm_handle* h);

int do_sort(mpm_handle* h) {
    if (!is_mixed(h)) return do_sort_f64(h);
    int r = mixed_to_staging(h);
    if (r) return r;
    r = do_sort_f64(h);
    if (r) return r;
    return mixed_from_staging(h);
}

int do_sort_f64(mpm_handle* h) {
    if (h->n == 0) return MPM_OK;
    int r = ensure_sort_scratch(h);
    if (r) return r;
    const SimParams3D& p = h->prms;
    SortGeom G;
    G.slab = p.GridY * p.GridZ;
    G.gz = p.GridZ;
    G.key_shift = p.GridHaloSize * G.slab;
    G.nb = (p.GridXTotal + 2 * p.GridHaloSize + 1) * G.slab;
    G.h_inv = p.cellsize_inv;
    const int n = (int)h->n;
    const int nb1 = G.nb + 1;
    CK(h, cudaMemsetAsync(h->s_count, 0, sizeof(int) * nb1, h->stream));
    k_sort_keys<<<blocks_for(n, 256), 256, 0, h->stream>>>(G, h->pts, h->pitch, n, h->s_bucket, h->s_count, h->err);
    CK_LAUNCH(h, "sort keys");
    r = exclusive_scan(h, h->s_count, h->s_start, nb1, 0);
    if (r) return r;
    CK(h, cudaMemsetAsync(h->s_count, 0, sizeof(int) * nb1, h->stream));
    k_sort_scatter<<<blocks_for(n, 256), 256, 0, h->stream>>>(h->s_bucket, n, h->s_start, h->s_count, h->s_perm);
    CK_LAUNCH(h, "sort scatter");
    k_sort_fix<<<blocks_for(G.nb, 256), 256, 0, h->stream>>>(G.nb, h->s_start, h->s_count, h->s_perm);
    CK_LAUNCH(h, "sort fix");
    int kept = 0;
    CK(h, cudaMemcpyAsync(&kept, h->s_start + G.nb, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    CK(h, cudaStreamSynchronize(h->stream));
    if (kept > 0) {
        dim3 grid(blocks_for(kept, 256), MPM_N_PTS_ARRAYS);
        k_gather_rows<double><<<grid, 256, 0, h->stream>>>(h->pts, h->pitch, h->pts_alt, h->pitch, MPM_N_PTS_ARRAYS,
                                                           h->s_perm, kept);
        CK_LAUNCH(h, "gather rows");
        k_gather_rows<unsigned><<<dim3(blocks_for(kept, 256), 1), 256, 0, h->stream>>>(h->ids, h->pitch, h->ids_alt,
                                                                                       h->pitch, 1, h->s_perm, kept);
        CK_LAUNCH(h, "gather ids");
        if (h->p0) {
            if (!h->p0_alt) CK(h, cudaMalloc(&h->p0_alt, sizeof(double) * h->pitch));
            k_gather_rows<double><<<dim3(blocks_for(kept, 256), 1), 256, 0, h->stream>>>(h->p0, h->pitch, h->p0_alt,
                                                                                         h->pitch, 1, h->s_perm, kept);
            CK_LAUNCH(h, "gather p0");
            std::swap(h->p0, h->p0_alt);
        }
        std::swap(h->pts, h->pts_alt);
        std::swap(h->ids, h->ids_alt);
    }
    h->n = (unsigned)kept;
    h->steps_since_sort = 0;
    return MPM_OK;
}

}  // namespace

// ==================================================================== ABI

extern "C" {

mpm_handle* mpm_create(const SimParams3D* prms, int precision, unsigned capacity, int device, int* status) {
    int st = MPM_OK;
    mpm_handle* h = nullptr;
    do {
        if (!params_valid(prms) || capacity == 0 ||
            (precision != MPM_PRECISION_FP64 && precision != MPM_PRECISION_FP64_SVD64 &&
             precision != MPM_PRECISION_MIXED)) {
            st = MPM_ERR_ARG;
            break;
        }
        if ((long long)(prms->GridXTotal + 2 * prms->GridHaloSize) * prms->GridY * prms->GridZ >= 0x7fffffffLL) {
            st = MPM_ERR_ARG;   // node indices are 32-bit in the kernels
            break;
        }
        if (precision == MPM_PRECISION_MIXED &&
            std::max(prms->GridXTotal + 2 * prms->GridHaloSize, std::max(prms->GridY, prms->GridZ)) >=
                (1 << (31 - kFixBits)) - 1) {
            st = MPM_ERR_ARG;   // positions are x / h in 32-bit fixed point with kFixBits fraction bits
            break;
        }
        int count = 0;
        if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0 || device < 0 || device >= count) {
            cudaGetLastError();
            st = MPM_ERR_NO_DEVICE;
            break;
        }
        cudaDeviceProp prop;
        if (cudaGetDeviceProperties(&prop, device) != cudaSuccess || prop.major < 10) {
            st = MPM_ERR_NO_DEVICE;
            break;
        }
        h = new (std::nothrow) mpm_handle();
        if (!h) { st = MPM_ERR_ARG; break; }
        h->prms = *prms;
        h->dp = make_dev_params(*prms);
        h->precision = precision;
        h->device = device;
        h->capacity = capacity;
        h->num_sms = prop.multiProcessorCount;
        h->pitch = ((size_t)capacity + 31) / 32 * 32;
        if (cudaSetDevice(device) != cudaSuccess) { st = MPM_ERR_CUDA; break; }
        if (cudaStreamCreateWithFlags(&h->own_stream, cudaStreamNonBlocking) != cudaSuccess) { st = MPM_ERR_CUDA; break; }
        h->stream = h->own_stream;
        const size_t ns = sensor_count(*prms);
        if (cudaMalloc(&h->pts, sizeof(double) * MPM_N_PTS_ARRAYS * h->pitch) != cudaSuccess ||
            cudaMalloc(&h->ids, sizeof(unsigned) * h->pitch) != cudaSuccess ||
            cudaMalloc(&h->grid, sizeof(double) * 4 * (size_t)h->dp.gstride) != cudaSuccess ||
            cudaMalloc(&h->sensor, sizeof(double) * ns) != cudaSuccess ||
            cudaMalloc(&h->force_phase, sizeof(double) * 3) != cudaSuccess ||
            cudaMalloc(&h->err, sizeof(int)) != cudaSuccess) {
            st = MPM_ERR_CUDA;
            break;
        }
        if (cudaMalloc(&h->rm_list, sizeof(int) * h->pitch) != cudaSuccess ||
            cudaMalloc(&h->rm_counts, sizeof(int) * 2) != cudaSuccess) {
            st = MPM_ERR_CUDA;
            break;
        }
        cudaMemsetAsync(h->rm_counts, 0, sizeof(int) * 2, h->stream);
        if (precision == MPM_PRECISION_MIXED) {
            if (cudaMalloc(&h->mx, sizeof(float) * MPM_N_PTS_ARRAYS * h->pitch) != cudaSuccess ||
                cudaMalloc(&h->gacc, sizeof(float4) * (size_t)h->dp.nodes) != cudaSuccess ||
                cudaMalloc(&h->gvel, sizeof(float4) * (size_t)h->dp.nodes) != cudaSuccess) {
                st = MPM_ERR_CUDA;
                break;
            }
            cudaMemsetAsync(h->mx, 0, sizeof(float) * MPM_N_PTS_ARRAYS * h->pitch, h->stream);
            cudaMemsetAsync(h->gacc, 0, sizeof(float4) * (size_t)h->dp.nodes, h->stream);
            cudaMemsetAsync(h->gvel, 0, sizeof(float4) * (size_t)h->dp.nodes, h->stream);
        }
        cudaMemsetAsync(h->pts, 0, sizeof(double) * MPM_N_PTS_ARRAYS * h->pitch, h->stream);
        cudaMemsetAsync(h->grid, 0, sizeof(double) * 4 * (size_t)h->dp.gstride, h->stream);
        cudaMemsetAsync(h->sensor, 0, sizeof(double) * ns, h->stream);
        cudaMemsetAsync(h->force_phase, 0, sizeof(double) * 3, h->stream);
        cudaMemsetAsync(h->err, 0, sizeof(int), h->stream);
        if (cudaStreamSynchronize(h->stream) != cudaSuccess) { st = MPM_ERR_CUDA; break; }
    } while (0);
    if (status) *status = st;
    if (st != MPM_OK) {
        if (h) { free_all(h); delete h; }
        return nullptr;
    }
    return h;
}

void mpm_destroy(mpm_handle* h) {
    if (!h) return;
    cudaSetDevice(h->device);
    cudaStreamSynchronize(h->stream);
    free_all(h);
    delete h;
}

int mpm_set_stream(mpm_handle* h, void* s) {
    if (!h) return MPM_ERR_ARG;
    CK(h, cudaStreamSynchronize(h->stream));
    h->stream = s ? (cudaStream_t)s : h->own_stream;
    return MPM_OK;
}

int mpm_update_constants(mpm_handle* h, const SimParams3D* prms) {
    if (!h || !params_valid(prms)) return MPM_ERR_ARG;
    if (prms->GridXTotal != h->prms.GridXTotal || prms->GridY != h->prms.GridY || prms->GridZ != h->prms.GridZ ||
        prms->GridHaloSize != h->prms.GridHaloSize || prms->IndenterSubdivisions != h->prms.IndenterSubdivisions)
        return MPM_ERR_ARG;
    h->prms = *prms;
    h->dp = make_dev_params(*prms);
    h->p2g_ready = false;
    CK(h, cudaMemsetAsync(h->err, 0, sizeof(int), h->stream));
    return MPM_OK;
}

int mpm_upload_soa(mpm_handle* h, const double* soa, unsigned pitch, unsigned n) {
    if (!h || (!soa && n) || pitch < n) return MPM_ERR_ARG;
    if (n > h->capacity) return MPM_ERR_CAPACITY;
    if (n) {
        CK(h, cudaMemcpy2DAsync(h->pts, sizeof(double) * h->pitch, soa, sizeof(double) * pitch, sizeof(double) * n,
                                MPM_N_PTS_ARRAYS, cudaMemcpyHostToDevice, h->stream));
        k_iota<<<blocks_for(n, 256), 256, 0, h->stream>>>(h->ids, (int)n, h->id_base);
        CK_LAUNCH(h, "ids");
        CK(h, cudaStreamSynchronize(h->stream));   // soa may be released when the call returns
    }
    h->n = n;
    h->uploaded = true;
    h->p2g_ready = false;
    h->fr_ready = false;   // new points: the next frame record must be a full frame
    if (is_mixed(h)) {
        int r = mixed_from_staging(h);
        if (r) return r;
    }
    CK(h, cudaMemsetAsync(h->err, 0, sizeof(int), h->stream));
    return MPM_OK;
}

int mpm_upload_cohesion(mpm_handle* h, const double* c, unsigned n) {
    if (!h) return MPM_ERR_ARG;
    if (!c) {
        cudaStreamSynchronize(h->stream);
        cudaFree(h->p0);
        cudaFree(h->p0_alt);
        cudaFree(h->p0f);
        h->p0 = h->p0_alt = nullptr;
        h->p0f = nullptr;
        h->p2g_ready = false;
        return MPM_OK;
    }
    if (n != h->n || h->prms.DP_tan_phi == 0) return MPM_ERR_ARG;
    if (!h->p0) CK(h, cudaMalloc(&h->p0, sizeof(double) * h->pitch));
    if (is_mixed(h) && !h->p0f) CK(h, cudaMalloc(&h->p0f, sizeof(float) * h->pitch));
    h->p2g_ready = false;
    if (n == 0) return MPM_OK;
    // cohesion to the device as given, then p0 = c / tan(phi) there (the same
    // correctly rounded FP64 division as on the host)
    CK(h, cudaMemcpyAsync(h->p0, c, sizeof(double) * n, cudaMemcpyHostToDevice, h->stream));
    k_cohesion_to_apex<<<blocks_for(n, 256), 256, 0, h->stream>>>(h->p0, is_mixed(h) ? h->p0f : nullptr, (int)n,
                                                                  h->prms.DP_tan_phi);
    CK_LAUNCH(h, "cohesion to apex shift");
    CK(h, cudaStreamSynchronize(h->stream));   // c may be released when the call returns
    return MPM_OK;
}

int mpm_download_soa(mpm_handle* h, double* soa, unsigned pitch, unsigned* n) {
    if (!h || !soa || pitch < h->n) return MPM_ERR_ARG;
    if (is_mixed(h)) {
        int r = mixed_to_staging(h);
        if (r) return r;
    }
    if (h->n) {
        CK(h, cudaMemcpy2DAsync(soa, sizeof(double) * pitch, h->pts, sizeof(double) * h->pitch, sizeof(double) * h->n,
                                MPM_N_PTS_ARRAYS, cudaMemcpyDeviceToHost, h->stream));
    }
    int code = 0;
    int r = read_error(h, &code);
    if (r) return r;
    if (n) *n = h->n;
    return code;
}

int mpm_download_ids(mpm_handle* h, unsigned* ids, unsigned* n) {
    if (!h || !ids) return MPM_ERR_ARG;
    if (h->n) CK(h, cudaMemcpyAsync(ids, h->ids, sizeof(unsigned) * h->n, cudaMemcpyDeviceToHost, h->stream));
    CK(h, cudaStreamSynchronize(h->stream));
    if (n) *n = h->n;
    return MPM_OK;
}

int mpm_upload_ids(mpm_handle* h, const unsigned* ids, unsigned n) {
    if (!h || (!ids && n)) return MPM_ERR_ARG;
    if (!h->uploaded) return MPM_ERR_STATE;
    if (n != h->n) return MPM_ERR_ARG;
    if (n) {
        CK(h, cudaMemcpyAsync(h->ids, ids, sizeof(unsigned) * n, cudaMemcpyHostToDevice, h->stream));
        CK(h, cudaStreamSynchronize(h->stream));
    }
    return MPM_OK;
}

int mpm_download_cohesion(mpm_handle* h, double* cohesion, unsigned* n) {
    if (!h || !cohesion || !n) return MPM_ERR_ARG;
    if (!h->p0) return MPM_ERR_STATE;
    std::vector<double> p0(h->n);
    if (h->n) {
        CK(h, cudaMemcpyAsync(p0.data(), h->p0, sizeof(double) * h->n, cudaMemcpyDeviceToHost, h->stream));
        CK(h, cudaStreamSynchronize(h->stream));
    }
    for (unsigned i = 0; i < h->n; i++) cohesion[i] = p0[i] * h->prms.DP_tan_phi;
    *n = h->n;
    return MPM_OK;
}

int mpm_sort(mpm_handle* h) {
    if (!h) return MPM_ERR_ARG;
    if (!h->uploaded) return MPM_ERR_STATE;
    int r = do_sort(h);
    if (r) return r;
    int code = 0;
    r = read_error(h, &code);
    return r ? r : code;
}

int mpm_set_grid_accumulation(mpm_handle* h, int mode) {
    if (!h || (mode != MPM_ACCUM_FLOAT && mode != MPM_ACCUM_FIXED)) return MPM_ERR_ARG;
    if (!is_mixed(h)) return mode == MPM_ACCUM_FLOAT ? MPM_OK : MPM_ERR_ARG;
    CK(h, cudaStreamSynchronize(h->stream));
    if (mode == MPM_ACCUM_FIXED && !h->gacc_q) {
        CK(h, cudaMalloc(&h->gacc_q, sizeof(unsigned long long) * 4 * (size_t)h->dp.nodes));
        CK(h, cudaMemsetAsync(h->gacc_q, 0, sizeof(unsigned long long) * 4 * (size_t)h->dp.nodes, h->stream));
    } else if (mode == MPM_ACCUM_FLOAT && h->gacc_q) {
        CK(h, cudaFree(h->gacc_q));
        h->gacc_q = nullptr;
    }
    h->p2g_ready = false;   // the next step computes its P2G into the selected accumulator
    return MPM_OK;
}

int mpm_set_sort_interval(mpm_handle* h, int k) {
    if (!h || k < 0) return MPM_ERR_ARG;
    h->sort_interval = k;
    return MPM_OK;
}

}  // extern "C"

namespace {

int ensure_frame_scratch(mpm_handle* h) {
    if (h->fr_f) return MPM_OK;
    const size_t p = h->pitch;
    CK(h, cudaMalloc(&h->fr_f, sizeof(float) * 7 * p));
    CK(h, cudaMalloc(&h->fr_status, p));
    CK(h, cudaMalloc(&h->fr_last, sizeof(int) * p));
    CK(h, cudaMalloc(&h->fr_i, sizeof(int) * 8 * (p + 1)));
    CK(h, cudaMalloc(&h->fr_rec, (sizeof(UpdPosRec) + sizeof(UpdJpRec) + sizeof(UpdStatusRec)) * p));
    long long m = (long long)p + 1;
    while (m > kScanTile) {
        m = (m + kScanTile - 1) / kScanTile;
        int* sums = nullptr;
        int* scanned = nullptr;
        CK(h, cudaMalloc(&sums, sizeof(int) * m));
        CK(h, cudaMalloc(&scanned, sizeof(int) * m));
        h->fr_scan_levels.push_back(sums);
        h->fr_scan_levels.push_back(scanned);
    }
    return MPM_OK;
}

template <class Pts>
int frame_records(mpm_handle* h, Pts pts, int frame, int full, mpm_visual_point* points, unsigned* n_points,
                  mpm_update_pos* upd_pos, unsigned* n_pos, mpm_update_jp* upd_jp, unsigned* n_jp,
                  mpm_update_status* upd_status, unsigned* n_status) {
    const int n = (int)h->n;
    const size_t p = h->pitch, m = p + 1;
    int* keep = h->fr_i;
    int* rank = keep + m;
    int* flags = rank + m;
    int* offs = flags + 3 * m;
    FrameVis v{h->fr_f, h->fr_f + 3 * p, h->fr_f + 6 * p, h->fr_status, h->fr_last, p};
    const unsigned nb = blocks_for(n, 256);
    CK(h, cudaMemsetAsync(keep + n, 0, sizeof(int), h->stream));
    if (n) {
        k_frame_keep<<<nb, 256, 0, h->stream>>>(pts, n, keep);
        CK_LAUNCH(h, "frame keep");
    }
    int r = exclusive_scan(h, keep, rank, n + 1, 0, &h->fr_scan_levels);
    if (r) return r;
    if (full) {
        auto* rec = reinterpret_cast<VisualPointRec*>(h->fr_rec);
        if (n) {
            k_frame_full<<<nb, 256, 0, h->stream>>>(pts, n, rank, v, frame, rec);
            CK_LAUNCH(h, "frame full");
        }
        int cnt = 0;
        CK(h, cudaMemcpyAsync(&cnt, rank + n, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
        CK(h, cudaStreamSynchronize(h->stream));
        if (cnt) CK(h, cudaMemcpyAsync(points, rec, sizeof(VisualPointRec) * cnt, cudaMemcpyDeviceToHost, h->stream));
        CK(h, cudaStreamSynchronize(h->stream));
        *n_points = (unsigned)cnt;
        h->fr_ready = true;
        return MPM_OK;
    }
    for (int k = 0; k < 3; k++) CK(h, cudaMemsetAsync(flags + k * m + n, 0, sizeof(int), h->stream));
    if (n) {
        k_frame_flags<<<nb, 256, 0, h->stream>>>(pts, n, rank, v, frame, h->prms.InitialTimeStep,
                                                 h->prms.UpdateEveryNthStep, h->prms.animation_threshold_pos,
                                                 flags, m);
        CK_LAUNCH(h, "frame flags");
    }
    for (int k = 0; k < 3; k++) {
        r = exclusive_scan(h, flags + k * m, offs + k * m, n + 1, 0, &h->fr_scan_levels);
        if (r) return r;
    }
    auto* upv = reinterpret_cast<UpdPosRec*>(h->fr_rec);
    auto* ujp = reinterpret_cast<UpdJpRec*>(h->fr_rec + sizeof(UpdPosRec) * p);
    auto* ust = reinterpret_cast<UpdStatusRec*>(h->fr_rec + (sizeof(UpdPosRec) + sizeof(UpdJpRec)) * p);
    if (n) {
        k_frame_emit<<<nb, 256, 0, h->stream>>>(pts, n, rank, flags, offs, m, upv, ujp, ust);
        CK_LAUNCH(h, "frame emit");
    }
    int cnt[3] = {0, 0, 0};
    for (int k = 0; k < 3; k++)
        CK(h, cudaMemcpyAsync(cnt + k, offs + k * m + n, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    CK(h, cudaStreamSynchronize(h->stream));
    if (cnt[0]) CK(h, cudaMemcpyAsync(upd_pos, upv, sizeof(UpdPosRec) * cnt[0], cudaMemcpyDeviceToHost, h->stream));
    if (cnt[1]) CK(h, cudaMemcpyAsync(upd_jp, ujp, sizeof(UpdJpRec) * cnt[1], cudaMemcpyDeviceToHost, h->stream));
    if (cnt[2])
        CK(h, cudaMemcpyAsync(upd_status, ust, sizeof(UpdStatusRec) * cnt[2], cudaMemcpyDeviceToHost, h->stream));
    CK(h, cudaStreamSynchronize(h->stream));
    *n_pos = (unsigned)cnt[0];
    *n_jp = (unsigned)cnt[1];
    *n_status = (unsigned)cnt[2];
    return MPM_OK;
}

}  // namespace

extern "C" {

int mpm_frame_records(mpm_handle* h, int frame, int full, mpm_visual_point* points, unsigned* n_points,
                      mpm_update_pos* upd_pos, unsigned* n_pos, mpm_update_jp* upd_jp, unsigned* n_jp,
                      mpm_update_status* upd_status, unsigned* n_status) {
    if (!h) return MPM_ERR_ARG;
    if (full ? (!points || !n_points) : (!upd_pos || !n_pos || !upd_jp || !n_jp || !upd_status || !n_status))
        return MPM_ERR_ARG;
    if (!h->uploaded || (!full && !h->fr_ready)) return MPM_ERR_STATE;
    int r = ensure_frame_scratch(h);
    if (r) return r;
    if (is_mixed(h))
        return frame_records(h, FramePointsMixed{mixed_state(h), h->prms.cellsize}, frame, full, points, n_points,
                             upd_pos, n_pos, upd_jp, n_jp, upd_status, n_status);
    return frame_records(h, FramePointsF64{h->pts, h->pitch}, frame, full, points, n_points, upd_pos, n_pos, upd_jp,
                         n_jp, upd_status, n_status);
}

int mpm_reset_grid(mpm_handle* h) {
    if (!h) return MPM_ERR_ARG;
    return reset_grid(h);
}

int mpm_p2g(mpm_handle* h) {
    if (!h) return MPM_ERR_ARG;
    if (!h->uploaded) return MPM_ERR_STATE;
    h->p2g_ready = false;
    return launch_p2g(h);
}

int mpm_update_nodes(mpm_handle* h, double indenter_x, double indenter_y) {
    if (!h) return MPM_ERR_ARG;
    h->p2g_ready = false;
    return launch_update(h, indenter_x, indenter_y, h->force_phase);
}

int mpm_g2p(mpm_handle* h, int record_pq) {
    if (!h) return MPM_ERR_ARG;
    if (!h->uploaded) return MPM_ERR_STATE;
    h->p2g_ready = false;
    return launch_g2p(h, record_pq);
}

int mpm_reset_indenter_force_accumulator(mpm_handle* h) {
    if (!h) return MPM_ERR_ARG;
    CK(h, cudaMemsetAsync(h->sensor, 0, sizeof(double) * sensor_count(h->prms), h->stream));
    return MPM_OK;
}

int mpm_step(mpm_handle* h, int nsteps, double* force_hist) {
    if (!h || nsteps < 0) return MPM_ERR_ARG;
    if (!h->uploaded) return MPM_ERR_STATE;
    if (nsteps == 0) return MPM_OK;
    if (nsteps > h->force_steps_cap) {
        CK(h, cudaStreamSynchronize(h->stream));
        cudaFree(h->force_steps);
        h->force_steps = nullptr;
        CK(h, cudaMalloc(&h->force_steps, sizeof(double) * 3 * (size_t)nsteps));
        h->force_steps_cap = nsteps;
    }
    CK(h, cudaMemsetAsync(h->force_steps, 0, sizeof(double) * 3 * (size_t)nsteps, h->stream));
    SimParams3D& p = h->prms;
    if (is_mixed(h) && !h->p2g_ready) {
        int r;
        if ((r = reset_grid(h))) return r;
        if ((r = launch_p2g(h))) return r;
        h->p2g_ready = true;
    }
    for (int s = 0; s < nsteps; s++) {
        p.SimulationTime += p.InitialTimeStep;
        p.indenter_x = p.indenter_x_initial + p.SimulationTime * p.IndVelocity;
        int r;
        if (is_mixed(h)) {
            // node update of this substep, then G2P of this substep fused with
            // the P2G of the next one (the accumulator stays ready)
            if ((r = launch_update(h, p.indenter_x, p.indenter_y, h->force_steps + 3 * s))) return r;
            const int record = (p.SimulationStep % p.UpdateEveryNthStep) == 0;
            const bool sort_next = h->sort_interval > 0 && h->steps_since_sort + 1 >= h->sort_interval;
            if ((r = launch_g2p2g_mixed(h, 1, record, s == nsteps - 1 || sort_next))) return r;
            if ((r = launch_return_map_mixed(h, 1))) return r;
            p.SimulationStep += 1;
            if (h->sort_interval > 0 && ++h->steps_since_sort >= h->sort_interval) {
                if ((r = do_sort(h))) return r;
            }
            continue;
        }
        if ((r = reset_grid(h))) return r;
        if ((r = launch_p2g(h))) return r;
        if ((r = launch_update(h, p.indenter_x, p.indenter_y, h->force_steps + 3 * s))) return r;
        const int record = (p.SimulationStep % p.UpdateEveryNthStep) == 0;
        if ((r = launch_g2p(h, record))) return r;
        p.SimulationStep += 1;
        if (h->sort_interval > 0 && ++h->steps_since_sort >= h->sort_interval) {
            if ((r = do_sort(h))) return r;
        }
    }
    if (force_hist) {
        CK(h, cudaMemcpyAsync(force_hist, h->force_steps, sizeof(double) * 3 * (size_t)nsteps, cudaMemcpyDeviceToHost,
                              h->stream));
    }
    int code = 0;
    int r = read_error(h, &code);
    return r ? r : code;
}

int mpm_sensors(mpm_handle* h, double* sensor, double total[3]) {
    if (!h) return MPM_ERR_ARG;
    const size_t ns = sensor_count(h->prms);
    std::vector<double> s(ns);
    CK(h, cudaMemcpyAsync(s.data(), h->sensor, sizeof(double) * ns, cudaMemcpyDeviceToHost, h->stream));
    CK(h, cudaStreamSynchronize(h->stream));
    const SimParams3D& p = h->prms;
    double t[3] = {0, 0, 0};
    for (size_t j = 0; j < ns / 3; j++)
        for (int k = 0; k < 3; k++) t[k] += s[3 * j + k];
    for (int k = 0; k < 3; k++) t[k] /= (double)p.UpdateEveryNthStep;
    const double norm = (double)(p.UpdateEveryNthStep * p.cellsize * p.cellsize);
    if (sensor)
        for (size_t j = 0; j < ns; j++) sensor[j] = s[j] / norm;
    if (total)
        for (int k = 0; k < 3; k++) total[k] = t[k];
    return MPM_OK;
}

int mpm_get_error(mpm_handle* h) {
    if (!h) return MPM_ERR_ARG;
    int code = 0;
    int r = read_error(h, &code);
    return r ? r : code;
}

int mpm_synchronize(mpm_handle* h) {
    if (!h) return MPM_ERR_ARG;
    CK(h, cudaStreamSynchronize(h->stream));
    return MPM_OK;
}

int mpm_get_params(mpm_handle* h, SimParams3D* out) {
    if (!h || !out) return MPM_ERR_ARG;
    *out = h->prms;
    return MPM_OK;
}

int mpm_count(mpm_handle* h, unsigned* n) {
    if (!h || !n) return MPM_ERR_ARG;
    *n = h->n;
    return MPM_OK;
}

const char* mpm_last_error_string(void) { return g_last_error; }

int mpm_host_alloc(size_t bytes, void** ptr) {
    if (!ptr) return MPM_ERR_ARG;
    *ptr = nullptr;
    if (bytes == 0) return MPM_OK;
    const cudaError_t e = cudaMallocHost(ptr, bytes);
    if (e != cudaSuccess) {
        *ptr = nullptr;
        return cuda_fail(nullptr, e, "cudaMallocHost");
    }
    return MPM_OK;
}

int mpm_host_free(void* ptr) {
    if (!ptr) return MPM_OK;
    const cudaError_t e = cudaFreeHost(ptr);
    return e == cudaSuccess ? MPM_OK : cuda_fail(nullptr, e, "cudaFreeHost");
}

}  // extern "C"

// ------------------------------------------------- x-slab partitions
//
// GPU_Implementation6 with nPartitions > 1 (gpu_implementation6.cpp:31-208,
// 340-382, model_3d.cpp:35-108): each partition is a handle that owns a slab
// of grid columns [x0, x0 + gxp) and the particles split to it; after P2G the
// partitions add each other's 2 * halo boundary slabs, and every
// UpdateEveryNthStep / PointTransferFrequency substeps the particles that
// left a slab move to the neighbour.

namespace {

size_t halo_nodes(const mpm_handle* h) { return (size_t)2 * h->prms.GridHaloSize * (size_t)h->dp.slab; }

// node offset of the first halo slab on a side of the window: columns
// x0 - halo (left) or x0 + gxp - halo (right), i.e. array slabs x0, x0 + gxp
long long halo_offset(const mpm_handle* h, int side) {
    const int x0 = h->part_x0, gxp = h->part_gxp ? h->part_gxp : h->prms.GridXTotal;
    return (long long)(side ? x0 + gxp : x0) * h->dp.slab;
}

size_t record_bytes(const mpm_handle* h) { return (is_mixed(h) ? sizeof(unsigned) : sizeof(double)) * kRecWords; }

}  // namespace

extern "C" {

int mpm_set_partition(mpm_handle* h, int id, int x0, int gxp, unsigned id_base) {
    if (!h || id < 0 || id > 255 || x0 < 0 || gxp < 1 || x0 + gxp > h->prms.GridXTotal) return MPM_ERR_ARG;
    const SimParams3D& p = h->prms;
    const bool whole = x0 == 0 && gxp == p.GridXTotal;
    if (!whole && p.GridHaloSize < 3) return MPM_ERR_ARG;   // a stencil spans 3 columns
    const int halo = p.GridHaloSize;
    h->part_id = id;
    h->part_x0 = x0;
    h->part_gxp = gxp;
    h->id_base = id_base;
    h->dp.win_lo = x0 - halo;
    h->dp.win_hi = x0 + gxp + halo - 3;
    h->dp.own_lo = x0 == 0 ? -halo : x0;
    h->dp.own_hi = x0 + gxp == p.GridXTotal ? p.GridXTotal + halo : x0 + gxp;
    h->dp.node_lo = (int)((long long)x0 * h->dp.slab);
    h->dp.node_hi = (int)((long long)(x0 + gxp + 2 * halo) * h->dp.slab);
    if (!h->xfer) CK(h, cudaMalloc(&h->xfer, sizeof(int) * 3));
    return MPM_OK;
}

size_t mpm_halo_bytes(const mpm_handle* h) {
    if (!h) return 0;
    return halo_nodes(h) * (is_mixed(h) && !h->gacc_q ? sizeof(float4) : 4 * sizeof(double));
}

int mpm_halo_pack(mpm_handle* h, int side, void* dst) {
    if (!h || !dst || (side != 0 && side != 1)) return MPM_ERR_ARG;
    const size_t hn = halo_nodes(h);
    if (!hn) return MPM_OK;
    const long long off = halo_offset(h, side);
    if (is_mixed(h)) {
        if (h->gacc_q)
            CK(h, cudaMemcpyAsync(dst, h->gacc_q + 4 * off, sizeof(unsigned long long) * 4 * hn,
                                  cudaMemcpyDeviceToDevice, h->stream));
        else
            CK(h, cudaMemcpyAsync(dst, h->gacc + off, sizeof(float4) * hn, cudaMemcpyDeviceToDevice, h->stream));
        return MPM_OK;
    }
    double* d = static_cast<double*>(dst);
    for (int c = 0; c < 4; c++)
        CK(h, cudaMemcpyAsync(d + c * hn, h->grid + c * h->dp.gstride + off, sizeof(double) * hn,
                              cudaMemcpyDeviceToDevice, h->stream));
    return MPM_OK;
}

int mpm_halo_add(mpm_handle* h, int side, const void* src) {
    if (!h || !src || (side != 0 && side != 1)) return MPM_ERR_ARG;
    const size_t hn = halo_nodes(h);
    if (!hn) return MPM_OK;
    const long long off = halo_offset(h, side);
    if (is_mixed(h) && h->gacc_q)
        k_halo_add_q<<<blocks_for(4 * hn, 256), 256, 0, h->stream>>>(h->gacc_q, off, (int)hn,
                                                                     static_cast<const unsigned long long*>(src));
    else if (is_mixed(h))
        k_halo_add_f4<<<blocks_for(hn, 256), 256, 0, h->stream>>>(h->gacc, off, (int)hn,
                                                                  static_cast<const float4*>(src));
    else
        k_halo_add_f64<<<blocks_for(hn, 256), 256, 0, h->stream>>>(h->grid, h->dp.gstride, off, (int)hn,
                                                                   static_cast<const double*>(src));
    CK_LAUNCH(h, "halo add");
    return MPM_OK;
}

size_t mpm_point_record_bytes(const mpm_handle* h) { return h ? record_bytes(h) : 0; }

int mpm_points_out(mpm_handle* h, void* left, void* right, unsigned capacity, unsigned* n_left, unsigned* n_right,
                   int* max_deviation) {
    if (!h || !n_left || !n_right || (capacity && (!left || !right))) return MPM_ERR_ARG;
    if (!h->uploaded) return MPM_ERR_STATE;
    if (!h->xfer) CK(h, cudaMalloc(&h->xfer, sizeof(int) * 3));
    CK(h, cudaMemsetAsync(h->xfer, 0, sizeof(int) * 3, h->stream));
    const SimParams3D& p = h->prms;
    XferGeom G;
    G.x0 = h->part_x0;
    G.gxp = h->part_gxp ? h->part_gxp : p.GridXTotal;
    G.keep_track = p.GridHaloSize / 2 - 1;
    G.cap = (int)std::min<unsigned>(capacity, 0x7fffffff);
    G.left_ok = G.x0 > 0 && capacity > 0;
    G.right_ok = G.x0 + G.gxp < p.GridXTotal && capacity > 0;
    G.h_inv = p.cellsize_inv;
    const int n = (int)h->n;
    if (n) {
        if (is_mixed(h))
            k_points_out_mixed<<<blocks_for(n, 256), 256, 0, h->stream>>>(
                G, static_cast<unsigned*>(h->mx), h->pitch, h->p0, h->ids, n, static_cast<unsigned*>(left),
                static_cast<unsigned*>(right), h->xfer);
        else
            k_points_out_f64<<<blocks_for(n, 256), 256, 0, h->stream>>>(G, h->pts, h->pitch, h->p0, h->ids, n,
                                                                        static_cast<double*>(left),
                                                                        static_cast<double*>(right), h->xfer);
        CK_LAUNCH(h, "points out");
    }
    int c[3] = {0, 0, 0};
    CK(h, cudaMemcpyAsync(c, h->xfer, sizeof(c), cudaMemcpyDeviceToHost, h->stream));
    CK(h, cudaStreamSynchronize(h->stream));
    *n_left = (unsigned)std::min(c[0], G.cap);
    *n_right = (unsigned)std::min(c[1], G.cap);
    if (max_deviation) *max_deviation = c[2];
    return MPM_OK;
}

int mpm_points_in(mpm_handle* h, const void* records, unsigned count) {
    if (!h || (count && !records)) return MPM_ERR_ARG;
    if (!h->uploaded) return MPM_ERR_STATE;
    if (!count) return MPM_OK;
    if ((size_t)h->n + count > h->capacity) return MPM_ERR_RECEIVE;   // mpm_kernels.cuh:420
    if (is_mixed(h))
        k_points_in_mixed<<<blocks_for(count, 256), 256, 0, h->stream>>>(
            static_cast<unsigned*>(h->mx), h->pitch, h->p0, h->p0f, h->ids, (int)h->n, (int)count,
            static_cast<const unsigned*>(records));
    else
        k_points_in_f64<<<blocks_for(count, 256), 256, 0, h->stream>>>(h->pts, h->pitch, h->p0, h->ids, (int)h->n,
                                                                       (int)count,
                                                                       static_cast<const double*>(records));
    CK_LAUNCH(h, "points in");
    h->n += count;
    h->fr_ready = false;
    return MPM_OK;
}

}  // extern "C"

// The two halves of a partitioned substep, around the halo exchange.
// First: the P2G sums of the current state in the grid (FP64: the window
// cleared and P2G; mixed: already there from the previous substep's fused
// kernel, else a standalone P2G).
int substep_p2g(mpm_handle* h) {
    int r;
    if (is_mixed(h)) {
        if (!h->p2g_ready) {
            if ((r = reset_grid(h)) || (r = launch_p2g(h))) return r;
            h->p2g_ready = true;
        }
        return MPM_OK;
    }
    if ((r = reset_grid(h)) || (r = launch_p2g(h))) return r;
    return MPM_OK;
}

// Second: node update at the indenter position of the substep, G2P (mixed:
// fused with the next substep's P2G, then the return map of the points that
// crushed); force3 (device) accumulates the substep's force.
int substep_update_g2p(mpm_handle* h, double ind_x, double ind_y, int record, int store_vc, double* force3) {
    int r;
    if ((r = launch_update(h, ind_x, ind_y, force3))) return r;
    if (is_mixed(h)) {
        if ((r = launch_g2p2g_mixed(h, 1, record, store_vc))) return r;
        return launch_return_map_mixed(h, 1);
    }
    return launch_g2p(h, record);
}

extern "C" {

int mpm_substep_p2g(mpm_handle* h) {
    if (!h) return MPM_ERR_ARG;
    if (!h->uploaded) return MPM_ERR_STATE;
    return substep_p2g(h);
}

int mpm_substep_update_g2p(mpm_handle* h, int store_vc, double force3[3]) {
    if (!h) return MPM_ERR_ARG;
    if (!h->uploaded) return MPM_ERR_STATE;
    SimParams3D& p = h->prms;
    p.SimulationTime += p.InitialTimeStep;
    p.indenter_x = p.indenter_x_initial + p.SimulationTime * p.IndVelocity;
    const int record = (p.SimulationStep % p.UpdateEveryNthStep) == 0;
    CK(h, cudaMemsetAsync(h->force_phase, 0, sizeof(double) * 3, h->stream));
    int r = substep_update_g2p(h, p.indenter_x, p.indenter_y, record, store_vc, h->force_phase);
    if (r) return r;
    p.SimulationStep += 1;
    if (force3) {
        CK(h, cudaMemcpyAsync(force3, h->force_phase, sizeof(double) * 3, cudaMemcpyDeviceToHost, h->stream));
        CK(h, cudaStreamSynchronize(h->stream));
    }
    return MPM_OK;
}

}  // extern "C"

// -------------------------------------- partitions driven in one process

struct mpm_multi {
    SimParams3D prms;
    int precision = MPM_PRECISION_FP64;
    int np = 0;
    unsigned capacity = 0;            // particles per partition
    unsigned xfer_cap = 0;            // records per direction (VectorCapacity_transfer)
    bool cohesion = false;
    std::vector<mpm_handle*> part;
    std::vector<unsigned> disabled;   // nPts_disabled of each partition
    // per partition, on its device: halo send buffers (left, right), halo
    // receive buffers, point-record out buffers (left, right) and an in buffer
    std::vector<void*> hsend[2], hrecv[2], pout[2], pin;
    std::vector<cudaEvent_t> ev_packed, ev_received, ev_out;
    int max_deviation = 0;
    int max_sent = 0;
    int rebalances = 0;
    std::vector<double> force;        // per-substep force of the running step call, summed over partitions
};

namespace {

void multi_free(mpm_multi* m) {
    for (int i = 0; i < (int)m->part.size(); i++) {
        mpm_handle* h = m->part[i];
        if (!h) continue;
        cudaSetDevice(h->device);
        for (int s = 0; s < 2; s++) {
            if (i < (int)m->hsend[s].size()) cudaFree(m->hsend[s][i]);
            if (i < (int)m->hrecv[s].size()) cudaFree(m->hrecv[s][i]);
            if (i < (int)m->pout[s].size()) cudaFree(m->pout[s][i]);
        }
        if (i < (int)m->pin.size()) cudaFree(m->pin[i]);
        if (i < (int)m->ev_packed.size()) cudaEventDestroy(m->ev_packed[i]);
        if (i < (int)m->ev_received.size()) cudaEventDestroy(m->ev_received[i]);
        if (i < (int)m->ev_out.size()) cudaEventDestroy(m->ev_out[i]);
        mpm_destroy(h);
    }
    m->part.clear();
}

// ProxyPoint3D::getCellIndex / getXIndex (proxypoint3d.cpp:158-170)
inline long long cell_key(const SimParams3D& p, double x, double y, double z) {
    return (long long)(int)(x * p.cellsize_inv + 0.5) * p.GridY * p.GridZ + (long long)(int)(y * p.cellsize_inv + 0.5) * p.GridZ +
           (int)(z * p.cellsize_inv + 0.5);
}
inline int x_index(const SimParams3D& p, double x) { return (int)(x * p.cellsize_inv + 0.5); }

inline bool disabled_word(double u) {
    long long v;
    std::memcpy(&v, &u, sizeof(v));
    return (v & MPM_STATUS_DISABLED) == MPM_STATUS_DISABLED;
}

// HostSideSOA::RemoveDisabledAndSort (host_side_soa.cpp:56-67) as a stable
// sort: the order of the kept particles, by cell key.
std::vector<unsigned> sorted_order(const SimParams3D& p, const double* soa, size_t pitch, unsigned n) {
    std::vector<unsigned> idx;
    idx.reserve(n);
    for (unsigned i = 0; i < n; i++)
        if (!disabled_word(soa[i])) idx.push_back(i);
    std::vector<long long> key(n);
    for (unsigned i : idx)
        key[i] = cell_key(p, soa[MPM_POSX * pitch + i], soa[(MPM_POSX + 1) * pitch + i], soa[(MPM_POSX + 2) * pitch + i]);
    std::stable_sort(idx.begin(), idx.end(), [&](unsigned a, unsigned b) { return key[a] < key[b]; });
    return idx;
}

// split_hssoa_into_partitions (gpu_implementation6.cpp:340-382) of a sorted
// SoA (n particles, row stride pitch) and its upload: partition i takes
// (n - done) / (np - i) particles; its slab ends at the x index of the first
// particle of the next one; the partition id goes into bits 24-31 of each
// particle's status word (ProxyPoint3D::setPartition, proxypoint3d.cpp:89-110).
// ids: the global id of each particle (may be null: 0, 1, ...).
int multi_split_upload(mpm_multi* m, std::vector<double>& soa, size_t pitch, unsigned n, const double* cohesion,
                       const std::vector<unsigned>* ids) {
    const SimParams3D& p = m->prms;
    std::vector<int> x0(m->np), cnt(m->np);
    unsigned done = 0;
    int off = 0;
    for (int i = 0; i < m->np; i++) {
        cnt[i] = (int)((n - done) / (unsigned)(m->np - i));
        x0[i] = off;
        if (i < m->np - 1) {
            const unsigned first_next = done + (unsigned)cnt[i];
            off = first_next < n ? x_index(p, soa[MPM_POSX * pitch + first_next]) : p.GridXTotal;
            off = std::max(off, x0[i] + 1);
            off = std::min(off, p.GridXTotal - (m->np - 1 - i));
        }
        for (unsigned j = done; j < done + (unsigned)cnt[i]; j++) {
            long long v;
            std::memcpy(&v, &soa[j], sizeof(v));
            v &= 0xffffffff00ffffffLL;
            v |= (long long)i << 24;
            std::memcpy(&soa[j], &v, sizeof(v));
        }
        done += (unsigned)cnt[i];
    }
    done = 0;
    for (int i = 0; i < m->np; i++) {
        mpm_handle* h = m->part[i];
        const int gxp = (i < m->np - 1 ? x0[i + 1] : p.GridXTotal) - x0[i];
        if ((unsigned)cnt[i] > h->capacity) return MPM_ERR_CAPACITY;
        int r = mpm_set_partition(h, i, x0[i], gxp, done);
        if (r) return r;
        // the partition's particles as a SoA of their own (28 rows of cnt[i])
        std::vector<double> local((size_t)MPM_N_PTS_ARRAYS * std::max(cnt[i], 1));
        for (int row = 0; row < MPM_N_PTS_ARRAYS; row++)
            std::memcpy(&local[(size_t)row * cnt[i]], &soa[row * pitch + done], sizeof(double) * cnt[i]);
        if ((r = mpm_upload_soa(h, local.data(), (unsigned)cnt[i], (unsigned)cnt[i]))) return r;
        if (cohesion && (r = mpm_upload_cohesion(h, cohesion + done, (unsigned)cnt[i]))) return r;
        if (ids && cnt[i]) {
            CK(h, cudaMemcpyAsync(h->ids, ids->data() + done, sizeof(unsigned) * cnt[i], cudaMemcpyHostToDevice,
                                  h->stream));
            CK(h, cudaStreamSynchronize(h->stream));
        }
        m->disabled[i] = 0;
        done += (unsigned)cnt[i];
    }
    return MPM_OK;
}

// the halo exchange after P2G (gpu_implementation6.cpp:31-112): every
// partition packs its boundary slabs; each receives its neighbours' packed
// slabs of the same columns (a peer copy when they live on another device)
// and adds them (partition_kernel_receive_halos_*). Events order the
// streams; a send buffer is packed again only after both neighbours copied it.
int multi_halo_exchange(mpm_multi* m) {
    const int np = m->np;
    if (np < 2) return MPM_OK;
    for (int i = 0; i < np; i++) {
        mpm_handle* h = m->part[i];
        CK(h, cudaSetDevice(h->device));
        if (i > 0) CK(h, cudaStreamWaitEvent(h->stream, m->ev_received[i - 1], 0));
        if (i < np - 1) CK(h, cudaStreamWaitEvent(h->stream, m->ev_received[i + 1], 0));
        int r;
        if (i > 0 && (r = mpm_halo_pack(h, 0, m->hsend[0][i]))) return r;
        if (i < np - 1 && (r = mpm_halo_pack(h, 1, m->hsend[1][i]))) return r;
        CK(h, cudaEventRecord(m->ev_packed[i], h->stream));
    }
    for (int i = 0; i < np; i++) {
        mpm_handle* h = m->part[i];
        CK(h, cudaSetDevice(h->device));
        const size_t bytes = mpm_halo_bytes(h);
        if (i > 0) {
            mpm_handle* l = m->part[i - 1];
            CK(h, cudaStreamWaitEvent(h->stream, m->ev_packed[i - 1], 0));
            CK(h, cudaMemcpyPeerAsync(m->hrecv[0][i], h->device, m->hsend[1][i - 1], l->device, bytes, h->stream));
        }
        if (i < np - 1) {
            mpm_handle* rr = m->part[i + 1];
            CK(h, cudaStreamWaitEvent(h->stream, m->ev_packed[i + 1], 0));
            CK(h, cudaMemcpyPeerAsync(m->hrecv[1][i], h->device, m->hsend[0][i + 1], rr->device, bytes, h->stream));
        }
        CK(h, cudaEventRecord(m->ev_received[i], h->stream));
        int r;
        if (i > 0 && (r = mpm_halo_add(h, 0, m->hrecv[0][i]))) return r;
        if (i < np - 1 && (r = mpm_halo_add(h, 1, m->hrecv[1][i]))) return r;
    }
    return MPM_OK;
}

// GPU_Implementation6::receive_points (gpu_implementation6.cpp:135-208): the
// records each partition wrote for its neighbours are copied to them and
// appended to their particle lists.
int multi_transfer_points(mpm_multi* m) {
    const int np = m->np;
    if (np < 2) return MPM_OK;
    std::vector<unsigned> nl(np), nr(np);
    for (int i = 0; i < np; i++) {
        mpm_handle* h = m->part[i];
        CK(h, cudaSetDevice(h->device));
        int dev = 0;
        int r = mpm_points_out(h, m->pout[0][i], m->pout[1][i], m->xfer_cap, &nl[i], &nr[i], &dev);
        if (r) return r;
        m->max_deviation = std::max(m->max_deviation, dev);
        m->max_sent = std::max(m->max_sent, (int)std::max(nl[i], nr[i]));
        m->disabled[i] += nl[i] + nr[i];
        CK(h, cudaEventRecord(m->ev_out[i], h->stream));
    }
    const size_t rb = record_bytes(m->part[0]);
    for (int i = 0; i < np; i++) {
        mpm_handle* h = m->part[i];
        CK(h, cudaSetDevice(h->device));
        unsigned k = 0;
        // from the left neighbour (its right-going records), then from the right
        if (i > 0 && nr[i - 1]) {
            CK(h, cudaStreamWaitEvent(h->stream, m->ev_out[i - 1], 0));
            CK(h, cudaMemcpyPeerAsync(m->pin[i], h->device, m->pout[1][i - 1], m->part[i - 1]->device,
                                      rb * nr[i - 1], h->stream));
            k += nr[i - 1];
        }
        if (i < np - 1 && nl[i + 1]) {
            CK(h, cudaStreamWaitEvent(h->stream, m->ev_out[i + 1], 0));
            CK(h, cudaMemcpyPeerAsync(static_cast<char*>(m->pin[i]) + rb * k, h->device, m->pout[0][i + 1],
                                      m->part[i + 1]->device, rb * nl[i + 1], h->stream));
            k += nl[i + 1];
        }
        int r = mpm_points_in(h, m->pin[i], k);
        if (r) return r;
    }
    // the out buffers are written again at the next transfer only after
    // every receiver's copy: wait for them here (transfers are rare)
    for (int i = 0; i < np; i++) {
        mpm_handle* h = m->part[i];
        CK(h, cudaSetDevice(h->device));
        CK(h, cudaStreamSynchronize(h->stream));
    }
    return MPM_OK;
}

int multi_download(mpm_multi* m, std::vector<double>& soa, std::vector<unsigned>& ids,
                   std::vector<double>& cohesion, unsigned& n) {
    n = 0;
    for (mpm_handle* h : m->part) n += h->n;
    soa.assign((size_t)MPM_N_PTS_ARRAYS * std::max(n, 1u), 0.0);
    ids.assign(std::max(n, 1u), 0u);
    cohesion.assign(m->cohesion ? std::max(n, 1u) : 0, 0.0);
    unsigned off = 0;
    std::vector<double> local;
    for (mpm_handle* h : m->part) {
        CK(h, cudaSetDevice(h->device));
        const unsigned k = h->n;
        local.assign((size_t)MPM_N_PTS_ARRAYS * std::max(k, 1u), 0.0);
        unsigned got = 0;
        int r = mpm_download_soa(h, local.data(), std::max(k, 1u), &got);
        if (r) return r;
        for (int row = 0; row < MPM_N_PTS_ARRAYS; row++)
            std::memcpy(&soa[(size_t)row * n + off], &local[(size_t)row * std::max(k, 1u)], sizeof(double) * k);
        if ((r = mpm_download_ids(h, ids.data() + off, &got))) return r;
        if (m->cohesion && k) {
            CK(h, cudaMemcpyAsync(cohesion.data() + off, h->p0, sizeof(double) * k, cudaMemcpyDeviceToHost,
                                  h->stream));
            CK(h, cudaStreamSynchronize(h->stream));
            for (unsigned j = 0; j < k; j++) cohesion[off + j] *= h->prms.DP_tan_phi;   // back to c = p0 tan(phi)
        }
        off += k;
    }
    return MPM_OK;
}

// Model3D::Step's rebalance (model_3d.cpp:99-108): all particles back to the
// host, RemoveDisabledAndSort, split again, upload.
int multi_rebalance(mpm_multi* m) {
    std::vector<double> soa, coh;
    std::vector<unsigned> ids;
    unsigned n = 0;
    int r = multi_download(m, soa, ids, coh, n);
    if (r) return r;
    const std::vector<unsigned> order = sorted_order(m->prms, soa.data(), n, n);
    const unsigned k = (unsigned)order.size();
    std::vector<double> s2((size_t)MPM_N_PTS_ARRAYS * std::max(k, 1u));
    std::vector<double> c2(m->cohesion ? std::max(k, 1u) : 0);
    std::vector<unsigned> i2(std::max(k, 1u));
    for (unsigned j = 0; j < k; j++) {
        const unsigned src = order[j];
        for (int row = 0; row < MPM_N_PTS_ARRAYS; row++) s2[(size_t)row * k + j] = soa[(size_t)row * n + src];
        if (m->cohesion) c2[j] = coh[src];
        i2[j] = ids[src];
    }
    m->rebalances++;
    return multi_split_upload(m, s2, k, k, m->cohesion ? c2.data() : nullptr, &i2);
}

bool multi_needs_rebalance(const mpm_multi* m) {
    const SimParams3D& p = m->prms;
    for (int i = 0; i < m->np; i++) {
        const mpm_handle* h = m->part[i];
        const double n = std::max<double>(h->n, 1.0);
        const double free_share = ((double)h->capacity - (double)h->n) / n;
        const double disabled_share = (double)m->disabled[i] / (double)h->capacity;
        if (free_share < p.RebalanceThresholdFreeSpaceRemaining) return true;
        if (disabled_share > p.RebalanceThresholdDisabledPercentage) return true;
    }
    return false;
}

}  // namespace

extern "C" {

mpm_multi* mpm_multi_create(const SimParams3D* prms, int precision, unsigned capacity, const int* devices,
                            int ndevices, int* status) {
    int st = MPM_OK;
    mpm_multi* m = nullptr;
    do {
        if (!params_valid(prms) || prms->nPartitions < 1 || prms->nPartitions > 256 || !devices || ndevices < 1 ||
            capacity == 0) {
            st = MPM_ERR_ARG;
            break;
        }
        if (prms->nPartitions > 1 && prms->GridHaloSize < 3) { st = MPM_ERR_ARG; break; }
        m = new (std::nothrow) mpm_multi();
        if (!m) { st = MPM_ERR_ARG; break; }
        m->prms = *prms;
        m->precision = precision;
        m->np = prms->nPartitions;
        m->capacity = capacity;
        m->xfer_cap = (unsigned)std::max(prms->VectorCapacity_transfer, 1);
        m->disabled.assign(m->np, 0);
        for (int s = 0; s < 2; s++) {
            m->hsend[s].assign(m->np, nullptr);
            m->hrecv[s].assign(m->np, nullptr);
            m->pout[s].assign(m->np, nullptr);
        }
        m->pin.assign(m->np, nullptr);
        for (int i = 0; i < m->np && st == MPM_OK; i++) {
            // GPU_Implementation6::initialize: partition i on device i % count
            mpm_handle* h = mpm_create(prms, precision, capacity, devices[i % ndevices], &st);
            if (!h) break;
            m->part.push_back(h);
            cudaSetDevice(h->device);
            const size_t hb = mpm_halo_bytes(h), rb = record_bytes(h) * m->xfer_cap;
            cudaEvent_t e[3];
            for (int k = 0; k < 3; k++)
                if (cudaEventCreateWithFlags(&e[k], cudaEventDisableTiming) != cudaSuccess) st = MPM_ERR_CUDA;
            m->ev_packed.push_back(e[0]);
            m->ev_received.push_back(e[1]);
            m->ev_out.push_back(e[2]);
            for (int s = 0; s < 2 && st == MPM_OK; s++) {
                if (cudaMalloc(&m->hsend[s][i], std::max<size_t>(hb, 16)) != cudaSuccess ||
                    cudaMalloc(&m->hrecv[s][i], std::max<size_t>(hb, 16)) != cudaSuccess ||
                    cudaMalloc(&m->pout[s][i], rb) != cudaSuccess)
                    st = MPM_ERR_CUDA;
            }
            if (st == MPM_OK && cudaMalloc(&m->pin[i], 2 * rb) != cudaSuccess) st = MPM_ERR_CUDA;
            // the events start out recorded, so the first waits on them pass
            for (int k = 0; k < 3 && st == MPM_OK; k++)
                if (cudaEventRecord(e[k], h->stream) != cudaSuccess) st = MPM_ERR_CUDA;
        }
        if (st != MPM_OK) break;
        // GPU_Implementation6::enable_peer_access: neighbours on other devices
        for (int i = 0; i + 1 < m->np; i++) {
            const int a = m->part[i]->device, b = m->part[i + 1]->device;
            if (a == b) continue;
            int ok = 0;
            cudaDeviceCanAccessPeer(&ok, a, b);
            if (ok) {
                cudaSetDevice(a);
                cudaDeviceEnablePeerAccess(b, 0);
                cudaSetDevice(b);
                cudaDeviceEnablePeerAccess(a, 0);
                cudaGetLastError();   // "already enabled" is not an error here
            }
        }
    } while (0);
    if (status) *status = st;
    if (st != MPM_OK) {
        if (m) { multi_free(m); delete m; }
        return nullptr;
    }
    return m;
}

void mpm_multi_destroy(mpm_multi* m) {
    if (!m) return;
    for (mpm_handle* h : m->part) {
        cudaSetDevice(h->device);
        cudaStreamSynchronize(h->stream);
    }
    multi_free(m);
    delete m;
}

int mpm_multi_upload_soa(mpm_multi* m, const double* soa, unsigned pitch, unsigned n, const double* cohesion) {
    if (!m || (!soa && n) || pitch < n) return MPM_ERR_ARG;
    const std::vector<unsigned> order = sorted_order(m->prms, soa, pitch, n);
    const unsigned k = (unsigned)order.size();
    std::vector<double> s2((size_t)MPM_N_PTS_ARRAYS * std::max(k, 1u));
    std::vector<double> c2(cohesion ? std::max(k, 1u) : 0);
    std::vector<unsigned> ids(std::max(k, 1u));
    for (unsigned j = 0; j < k; j++) {
        for (int row = 0; row < MPM_N_PTS_ARRAYS; row++) s2[(size_t)row * k + j] = soa[(size_t)row * pitch + order[j]];
        if (cohesion) c2[j] = cohesion[order[j]];
        ids[j] = order[j];
    }
    m->cohesion = cohesion != nullptr;
    m->max_deviation = 0;
    return multi_split_upload(m, s2, k, k, cohesion ? c2.data() : nullptr, &ids);
}

int mpm_multi_step(mpm_multi* m, int nsteps, double* force_hist) {
    if (!m || nsteps < 0) return MPM_ERR_ARG;
    for (mpm_handle* h : m->part)
        if (!h->uploaded) return MPM_ERR_STATE;
    if (nsteps == 0) return MPM_OK;
    SimParams3D& p = m->prms;
    for (mpm_handle* h : m->part) {
        CK(h, cudaSetDevice(h->device));
        if (nsteps > h->force_steps_cap) {
            CK(h, cudaStreamSynchronize(h->stream));
            cudaFree(h->force_steps);
            h->force_steps = nullptr;
            CK(h, cudaMalloc(&h->force_steps, sizeof(double) * 3 * (size_t)nsteps));
            h->force_steps_cap = nsteps;
        }
        CK(h, cudaMemsetAsync(h->force_steps, 0, sizeof(double) * 3 * (size_t)nsteps, h->stream));
    }
    std::vector<double> total((size_t)3 * nsteps, 0.0);
    int done = 0;           // substeps whose forces are in the handles' buffers since the last flush
    auto flush_forces = [&](int upto) -> int {
        std::vector<double> f((size_t)3 * nsteps);
        for (mpm_handle* h : m->part) {
            CK(h, cudaSetDevice(h->device));
            CK(h, cudaMemcpyAsync(f.data(), h->force_steps, sizeof(double) * 3 * (size_t)upto, cudaMemcpyDeviceToHost,
                                  h->stream));
            CK(h, cudaStreamSynchronize(h->stream));
            for (int k = 3 * done; k < 3 * upto; k++) total[k] += f[k];
        }
        done = upto;
        return MPM_OK;
    };
    const int per = std::max(1, p.UpdateEveryNthStep / std::max(1, p.PointTransferFrequency));
    for (int s = 0; s < nsteps; s++) {
        p.SimulationTime += p.InitialTimeStep;
        p.indenter_x = p.indenter_x_initial + p.SimulationTime * p.IndVelocity;
        const int record = (p.SimulationStep % p.UpdateEveryNthStep) == 0;
        const bool transfer = m->np > 1 && (p.SimulationStep % per) == 0;
        const bool last = s == nsteps - 1;
        // v and C reach the mixed state (the fused chain keeps them in
        // registers) where a download can follow: the call's last substep,
        // a point transfer, an animation frame's end (a possible rebalance)
        const bool frame_end = (p.SimulationStep + 1) % p.UpdateEveryNthStep == 0;
        int r;
        for (mpm_handle* h : m->part) {
            CK(h, cudaSetDevice(h->device));
            if ((r = substep_p2g(h))) return r;
        }
        if ((r = multi_halo_exchange(m))) return r;
        for (mpm_handle* h : m->part) {
            CK(h, cudaSetDevice(h->device));
            if ((r = substep_update_g2p(h, p.indenter_x, p.indenter_y, record, last || transfer || frame_end,
                                        h->force_steps + 3 * s)))
                return r;
        }
        p.SimulationStep += 1;
        if (transfer && (r = multi_transfer_points(m))) return r;
        if (p.SimulationStep % p.UpdateEveryNthStep == 0) {
            // the end of an animation frame (model_3d.cpp:72-108): transfer
            // more often if a point strayed past half the halo; rebalance
            // when a partition runs short of room or holds many holes
            if (m->max_deviation > p.GridHaloSize / 2) p.PointTransferFrequency++;
            m->max_deviation = 0;
            if (m->np > 1 && multi_needs_rebalance(m)) {
                if ((r = flush_forces(s + 1))) return r;
                if ((r = multi_rebalance(m))) return r;
            }
        }
    }
    if (int r = flush_forces(nsteps)) return r;
    if (force_hist) std::memcpy(force_hist, total.data(), sizeof(double) * 3 * nsteps);
    int code = 0;
    for (mpm_handle* h : m->part) {
        h->prms.SimulationTime = p.SimulationTime;
        h->prms.SimulationStep = p.SimulationStep;
        h->prms.indenter_x = p.indenter_x;
        h->prms.PointTransferFrequency = p.PointTransferFrequency;
        CK(h, cudaSetDevice(h->device));
        int c = 0;
        int r2 = read_error(h, &c);
        if (r2) return r2;
        if (c && !code) code = c;
    }
    return code;
}

int mpm_multi_download_soa(mpm_multi* m, double* soa, unsigned pitch, unsigned* ids, unsigned* n) {
    if (!m || !n) return MPM_ERR_ARG;
    std::vector<double> all, coh;
    std::vector<unsigned> id;
    unsigned k = 0;
    int r = multi_download(m, all, id, coh, k);
    if (r) return r;
    *n = k;
    if (!soa) return MPM_OK;
    if (pitch < k) return MPM_ERR_ARG;
    for (int row = 0; row < MPM_N_PTS_ARRAYS; row++)
        std::memcpy(soa + (size_t)row * pitch, all.data() + (size_t)row * k, sizeof(double) * k);
    if (ids) std::memcpy(ids, id.data(), sizeof(unsigned) * k);
    return MPM_OK;
}

int mpm_multi_rebalance(mpm_multi* m) {
    if (!m) return MPM_ERR_ARG;
    return multi_rebalance(m);
}

int mpm_multi_info(mpm_multi* m, int i, int* x0, int* gxp, unsigned* n, unsigned* n_disabled) {
    if (!m || i < 0 || i >= m->np) return MPM_ERR_ARG;
    const mpm_handle* h = m->part[i];
    if (x0) *x0 = h->part_x0;
    if (gxp) *gxp = h->part_gxp;
    if (n) *n = h->n;
    if (n_disabled) *n_disabled = m->disabled[i];
    return MPM_OK;
}

int mpm_multi_stats(mpm_multi* m, int* max_sent, int* rebalances, int* point_transfer_frequency) {
    if (!m) return MPM_ERR_ARG;
    if (max_sent) *max_sent = m->max_sent;
    if (rebalances) *rebalances = m->rebalances;
    if (point_transfer_frequency) *point_transfer_frequency = m->prms.PointTransferFrequency;
    return MPM_OK;
}

int mpm_multi_sensors(mpm_multi* m, double* sensor, double total[3]) {
    if (!m) return MPM_ERR_ARG;
    const size_t ns = sensor_count(m->prms);
    std::vector<double> acc(ns, 0.0), one(ns);
    double t[3] = {0, 0, 0};
    for (mpm_handle* h : m->part) {
        CK(h, cudaSetDevice(h->device));
        double tt[3];
        int r = mpm_sensors(h, one.data(), tt);
        if (r) return r;
        for (size_t j = 0; j < ns; j++) acc[j] += one[j];
        for (int k = 0; k < 3; k++) t[k] += tt[k];
    }
    if (sensor) std::memcpy(sensor, acc.data(), sizeof(double) * ns);
    if (total)
        for (int k = 0; k < 3; k++) total[k] = t[k];
    return MPM_OK;
}

int mpm_multi_reset_indenter_force_accumulator(mpm_multi* m) {
    if (!m) return MPM_ERR_ARG;
    for (mpm_handle* h : m->part) {
        CK(h, cudaSetDevice(h->device));
        int r = mpm_reset_indenter_force_accumulator(h);
        if (r) return r;
    }
    return MPM_OK;
}

}  // extern "C"

// ------------------------------------------------------------ test hooks

namespace {
template <class K>
__global__ void k_svd_batch(const double* __restrict__ A, int count, double* __restrict__ U, double* __restrict__ S,
                            double* __restrict__ V) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    typedef typename K::T T;
    T a[3][3], u[3][3], s[3], v[3][3];
    for (int r = 0; r < 3; r++)
        for (int c = 0; c < 3; c++) a[r][c] = (T)A[9 * i + 3 * r + c];
    svd3x3<K>(a, u, s, v);
    for (int r = 0; r < 3; r++) {
        S[3 * i + r] = (double)s[r];
        for (int c = 0; c < 3; c++) {
            U[9 * i + 3 * r + c] = (double)u[r][c];
            V[9 * i + 3 * r + c] = (double)v[r][c];
        }
    }
}
}  // namespace

extern "C" {

int mpm_testing_svd3x3(int mode, const double* A, int count, double* U, double* S, double* V, int device) {
    if (!A || !U || !S || !V || count <= 0 || (mode != 0 && mode != 1)) return MPM_ERR_ARG;
    CK(nullptr, cudaSetDevice(device));
    double *dA = nullptr, *dU = nullptr, *dS = nullptr, *dV = nullptr;
    const size_t m9 = sizeof(double) * 9 * (size_t)count, m3 = sizeof(double) * 3 * (size_t)count;
    int st = MPM_OK;
    if (cudaMalloc(&dA, m9) != cudaSuccess || cudaMalloc(&dU, m9) != cudaSuccess ||
        cudaMalloc(&dS, m3) != cudaSuccess || cudaMalloc(&dV, m9) != cudaSuccess) {
        st = cuda_fail(nullptr, cudaGetLastError(), "svd scratch");
    } else {
        cudaMemcpy(dA, A, m9, cudaMemcpyHostToDevice);
        if (mode == 0) k_svd_batch<SvdF32><<<blocks_for(count, 128), 128>>>(dA, count, dU, dS, dV);
        else k_svd_batch<SvdF64><<<blocks_for(count, 128), 128>>>(dA, count, dU, dS, dV);
        cudaError_t e = cudaDeviceSynchronize();
        if (e != cudaSuccess) st = cuda_fail(nullptr, e, "svd kernel");
        else {
            cudaMemcpy(U, dU, m9, cudaMemcpyDeviceToHost);
            cudaMemcpy(S, dS, m3, cudaMemcpyDeviceToHost);
            cudaMemcpy(V, dV, m9, cudaMemcpyDeviceToHost);
        }
    }
    cudaFree(dA); cudaFree(dU); cudaFree(dS); cudaFree(dV);
    return st;
}

size_t mpm_testing_sizeof_params(void) { return sizeof(SimParams3D); }

int mpm_testing_step_timed(mpm_handle* h, int nsteps, float* ms) {
    if (!h || nsteps <= 0 || !ms) return MPM_ERR_ARG;
    if (!h->uploaded) return MPM_ERR_STATE;
    cudaEvent_t ev[6];
    for (int k = 0; k < 6; k++) CK(h, cudaEventCreate(&ev[k]));
    for (int k = 0; k < 4; k++) ms[k] = 0.f;
    SimParams3D& p = h->prms;
    int r = MPM_OK;
    if (is_mixed(h) && !h->p2g_ready) {
        if ((r = reset_grid(h)) || (r = launch_p2g(h))) return r;
        h->p2g_ready = true;
    }
    if (!h->force_phase) return MPM_ERR_STATE;
    for (int s = 0; s < nsteps && !r; s++) {
        p.SimulationTime += p.InitialTimeStep;
        p.indenter_x = p.indenter_x_initial + p.SimulationTime * p.IndVelocity;
        const int record = (p.SimulationStep % p.UpdateEveryNthStep) == 0;
        cudaEventRecord(ev[0], h->stream);
        if (is_mixed(h)) {
            // ms[0] = 0, ms[1] = return-map kernel, ms[2] = update, ms[3] = fused kernel
            if ((r = launch_update(h, p.indenter_x, p.indenter_y, h->force_phase))) break;
            cudaEventRecord(ev[1], h->stream);
            if ((r = launch_g2p2g_mixed(h, 1, record, s == nsteps - 1))) break;
            cudaEventRecord(ev[2], h->stream);
            if ((r = launch_return_map_mixed(h, 1))) break;
            cudaEventRecord(ev[3], h->stream);
            CK(h, cudaEventSynchronize(ev[3]));
            float t = 0.f;
            cudaEventElapsedTime(&t, ev[0], ev[1]);
            ms[2] += t;
            cudaEventElapsedTime(&t, ev[1], ev[2]);
            ms[3] += t;
            cudaEventElapsedTime(&t, ev[2], ev[3]);
            ms[1] += t;
            p.SimulationStep += 1;
            continue;
        } else {
            if ((r = reset_grid(h))) break;
            cudaEventRecord(ev[1], h->stream);
            if ((r = launch_p2g(h))) break;
            cudaEventRecord(ev[2], h->stream);
            if ((r = launch_update(h, p.indenter_x, p.indenter_y, h->force_phase))) break;
            cudaEventRecord(ev[3], h->stream);
            if ((r = launch_g2p(h, record))) break;
        }
        cudaEventRecord(ev[4], h->stream);
        CK(h, cudaEventSynchronize(ev[4]));
        for (int k = 0; k < 4; k++) {
            float t = 0.f;
            cudaEventElapsedTime(&t, ev[k], ev[k + 1]);
            ms[k] += t;
        }
        p.SimulationStep += 1;
    }
    for (int k = 0; k < 6; k++) cudaEventDestroy(ev[k]);
    return r;
}

int mpm_testing_active_nodes(mpm_handle* h, long long* count) {
    if (!h || !count) return MPM_ERR_ARG;
    const size_t nodes = (size_t)h->dp.nodes;
    long long c = 0;
    if (is_mixed(h) && h->gacc_q) {
        std::vector<unsigned long long> g(4 * nodes);
        CK(h, cudaMemcpyAsync(g.data(), h->gacc_q, sizeof(unsigned long long) * 4 * nodes, cudaMemcpyDeviceToHost,
                              h->stream));
        CK(h, cudaStreamSynchronize(h->stream));
        for (size_t i = 0; i < nodes; i++) c += g[4 * i] != 0ull;
    } else if (is_mixed(h)) {
        std::vector<float4> g(nodes);
        CK(h, cudaMemcpyAsync(g.data(), h->gacc, sizeof(float4) * nodes, cudaMemcpyDeviceToHost, h->stream));
        CK(h, cudaStreamSynchronize(h->stream));
        for (size_t i = 0; i < nodes; i++) c += g[i].x != 0.f;
    } else {
        std::vector<double> m(nodes);
        CK(h, cudaMemcpyAsync(m.data(), h->grid, sizeof(double) * nodes, cudaMemcpyDeviceToHost, h->stream));
        CK(h, cudaStreamSynchronize(h->stream));
        for (size_t i = 0; i < nodes; i++) c += m[i] != 0.0;
    }
    *count = c;
    return MPM_OK;
}

int mpm_testing_download_grid(mpm_handle* h, double* out, int which) {
    if (!h || !out) return MPM_ERR_ARG;
    const size_t nodes = (size_t)h->dp.nodes;
    if (is_mixed(h) && h->gacc_q && !which) {
        std::vector<unsigned long long> g(4 * nodes);
        CK(h, cudaMemcpyAsync(g.data(), h->gacc_q, sizeof(unsigned long long) * 4 * nodes, cudaMemcpyDeviceToHost,
                              h->stream));
        CK(h, cudaStreamSynchronize(h->stream));
        for (size_t i = 0; i < nodes; i++) {
            out[i] = (double)(long long)g[4 * i] * h->dp.q_inv_m;
            for (int c = 1; c < 4; c++) out[c * nodes + i] = (double)(long long)g[4 * i + c] * h->dp.q_inv_p;
        }
        return MPM_OK;
    }
    if (is_mixed(h)) {
        std::vector<float4> g(nodes);
        CK(h, cudaMemcpyAsync(g.data(), which ? h->gvel : h->gacc, sizeof(float4) * nodes, cudaMemcpyDeviceToHost,
                              h->stream));
        CK(h, cudaStreamSynchronize(h->stream));
        for (size_t i = 0; i < nodes; i++) {
            out[i] = which ? 0.0 : g[i].x;
            out[nodes + i] = which ? g[i].x : g[i].y;
            out[2 * nodes + i] = which ? g[i].y : g[i].z;
            out[3 * nodes + i] = which ? g[i].z : g[i].w;
        }
        return MPM_OK;
    }
    for (int c = 0; c < 4; c++)
        CK(h, cudaMemcpyAsync(out + c * nodes, h->grid + c * h->dp.gstride, sizeof(double) * nodes,
                              cudaMemcpyDeviceToHost, h->stream));
    CK(h, cudaStreamSynchronize(h->stream));
    return MPM_OK;
}

}  // extern "C"

// ------------------------------------------- sort without device allocation
//
// Some callers cannot let a library allocate device memory: applications that
// own and plan every byte of the GPU themselves (their own pool, a fixed
// footprint planned at start-up), and loops that cannot afford the latency
// and implicit device-wide synchronisation of a cudaMalloc in the middle of a
// run. mpm_sort_permutation_noalloc serves them: the caller passes its own
// device buffers for input and output, and the sort's scratch lives in the
// fixed array below, which every GPU that loads this library holds until the
// process exits (about 10 MB).

namespace {

constexpr unsigned kNoAllocMaxParticles = 1u << 19;   // 524,288 particles
constexpr unsigned kNoAllocMaxCells = 1u << 20;       // 1,048,576 cell keys incl. the disabled bucket
constexpr unsigned kNoAllocTiles = kNoAllocMaxCells / kScanTile;
// layout (ints): bucket[P] | count[C] | start[C] | tile sums[T] | tile scan[T] | error flag
constexpr size_t kNoAllocOffCount = kNoAllocMaxParticles;
constexpr size_t kNoAllocOffStart = kNoAllocOffCount + kNoAllocMaxCells;
constexpr size_t kNoAllocOffSums = kNoAllocOffStart + kNoAllocMaxCells;
constexpr size_t kNoAllocOffScan = kNoAllocOffSums + kNoAllocTiles;
constexpr size_t kNoAllocOffErr = kNoAllocOffScan + kNoAllocTiles;
constexpr size_t kNoAllocInts = kNoAllocOffErr + 64;
static_assert(kNoAllocTiles <= (unsigned)kScanTile, "one scan level above the tiles");

static __device__ __align__(256) int g_noalloc_sort_scratch[kNoAllocInts];

// Device address of the scratch array per device: looked up once per device
// (with that device current) on the first call made there.
int* noalloc_scratch_for(int device, int* status) {
    static std::mutex mu;
    static int* ptrs[256] = {};
    if (device < 0 || device >= 256) { *status = MPM_ERR_ARG; return nullptr; }
    std::lock_guard<std::mutex> lock(mu);
    if (!ptrs[device]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_sort_scratch);
        if (e != cudaSuccess) {
            *status = cuda_fail(nullptr, e, "cudaGetSymbolAddress(sort scratch)");
            return nullptr;
        }
        ptrs[device] = static_cast<int*>(p);
    }
    *status = MPM_OK;
    return ptrs[device];
}

}  // namespace

extern "C" int mpm_sort_permutation_noalloc(const SimParams3D* prms, const double* soa, unsigned pitch, unsigned n,
                                            unsigned* perm, unsigned* kept, void* stream) {
    if (!params_valid(prms) || (!soa && n) || (!perm && n) || !kept || pitch < n) return MPM_ERR_ARG;
    const long long nb = (long long)(prms->GridXTotal + 2 * prms->GridHaloSize + 1) * prms->GridY * prms->GridZ;
    if (n > kNoAllocMaxParticles || nb + 1 > (long long)kNoAllocMaxCells) return MPM_ERR_NOALLOC_LIMIT;
    int dev = 0;
    CK(nullptr, cudaGetDevice(&dev));
    int st = MPM_OK;
    int* scratch = noalloc_scratch_for(dev, &st);
    if (!scratch) return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int* bucket = scratch;
    int* count = scratch + kNoAllocOffCount;
    int* start = scratch + kNoAllocOffStart;
    int* sums = scratch + kNoAllocOffSums;
    int* scan = scratch + kNoAllocOffScan;
    int* err = scratch + kNoAllocOffErr;
    // the array keeps the previous call's contents: clear what is summed into
    const int nb1 = (int)nb + 1;
    CK(nullptr, cudaMemsetAsync(count, 0, sizeof(int) * nb1, s));
    CK(nullptr, cudaMemsetAsync(err, 0, sizeof(int), s));
    if (n) {
        SortGeom G;
        G.slab = prms->GridY * prms->GridZ;
        G.gz = prms->GridZ;
        G.key_shift = prms->GridHaloSize * G.slab;
        G.nb = (int)nb;
        G.h_inv = prms->cellsize_inv;
        k_sort_keys<<<blocks_for(n, 256), 256, 0, s>>>(G, soa, pitch, (int)n, bucket, count, err);
        CK_LAUNCH(nullptr, "noalloc sort keys");
        const int tiles = (nb1 + kScanTile - 1) / kScanTile;
        k_scan_tiles<<<tiles, kScanBlock, 0, s>>>(count, start, nb1, tiles > 1 ? sums : nullptr);
        CK_LAUNCH(nullptr, "noalloc scan");
        if (tiles > 1) {
            k_scan_tiles<<<1, kScanBlock, 0, s>>>(sums, scan, tiles, nullptr);
            k_scan_add<<<blocks_for(nb1, 256), 256, 0, s>>>(start, nb1, scan);
            CK_LAUNCH(nullptr, "noalloc scan add");
        }
        CK(nullptr, cudaMemsetAsync(count, 0, sizeof(int) * nb1, s));
        k_sort_scatter<<<blocks_for(n, 256), 256, 0, s>>>(bucket, (int)n, start, count, perm);
        k_sort_fix<<<blocks_for(nb, 256), 256, 0, s>>>((int)nb, start, count, perm);
        CK_LAUNCH(nullptr, "noalloc scatter");
    }
    int host[2] = {0, 0};
    if (n) CK(nullptr, cudaMemcpyAsync(&host[0], start + nb, sizeof(int), cudaMemcpyDeviceToHost, s));
    CK(nullptr, cudaMemcpyAsync(&host[1], err, sizeof(int), cudaMemcpyDeviceToHost, s));
    CK(nullptr, cudaStreamSynchronize(s));
    *kept = (unsigned)host[0];
    return host[1];
}

// ------------------------------------------------------------------ adjoint

namespace {

size_t state_bytes(const mpm_handle* h) { return sizeof(double) * MPM_N_PTS_ARRAYS * h->pitch; }

// One FP64 substep of Model3D::Step on the particle rows at h->pts;
// p2g_copy (may be null) receives the grid after P2G (4 x gstride doubles).
int fp64_substep(mpm_handle* h, double* force3, double* p2g_copy = nullptr) {
    SimParams3D& p = h->prms;
    p.SimulationTime += p.InitialTimeStep;
    p.indenter_x = p.indenter_x_initial + p.SimulationTime * p.IndVelocity;
    int r;
    if ((r = reset_grid(h))) return r;
    if ((r = launch_p2g(h))) return r;
    if (p2g_copy)
        CK(h, cudaMemcpyAsync(p2g_copy, h->grid, sizeof(double) * 4 * (size_t)h->dp.gstride, cudaMemcpyDeviceToDevice,
                              h->stream));
    if ((r = launch_update(h, p.indenter_x, p.indenter_y, force3))) return r;
    const int record = (p.SimulationStep % p.UpdateEveryNthStep) == 0;
    if ((r = launch_g2p(h, record))) return r;
    p.SimulationStep += 1;
    return MPM_OK;
}

int ensure_adjoint_buffers(mpm_handle* h, int nsteps, int every) {
    const int nck = (nsteps + every - 1) / every;
    while ((int)h->ckpt.size() < nck) {
        double* b = nullptr;
        CK(h, cudaMalloc(&b, state_bytes(h)));
        h->ckpt.push_back(b);
    }
    while ((int)h->seg.size() < every + 1) {
        double* b = nullptr;
        CK(h, cudaMalloc(&b, state_bytes(h)));
        h->seg.push_back(b);
    }
    while ((int)h->adj_gcache.size() < every) {
        double* b = nullptr;
        CK(h, cudaMalloc(&b, sizeof(double) * 4 * (size_t)h->dp.gstride));
        h->adj_gcache.push_back(b);
    }
    h->ckpt_prms.resize(nck);
    if (!h->adj_A) {
        CK(h, cudaMalloc(&h->adj_A, sizeof(double) * ADJ_ROWS * h->pitch));
        CK(h, cudaMalloc(&h->adj_cgrad, sizeof(double) * h->pitch));
        CK(h, cudaMalloc(&h->adj_Egrad, sizeof(double)));
        CK(h, cudaMalloc(&h->adj_g7, sizeof(double) * 7 * (size_t)h->dp.gstride));
        CK(h, cudaMalloc(&h->adj_gb7, sizeof(double) * 7 * (size_t)h->dp.gstride));
        CK(h, cudaMalloc(&h->adj_rmv, sizeof(double) * 10 * h->pitch));
    }
    return MPM_OK;
}

AdjParams adj_params(const mpm_handle* h) {
    const SimParams3D& p = h->prms;
    AdjParams q;
    q.rc.pmax = p.IceCompressiveStrength;
    q.rc.tensile = p.IceTensileStrength;
    q.rc.shear = p.IceShearStrength;
    q.rc.tan_phi = p.DP_tan_phi;
    const double nu = p.PoissonsRatio;
    q.dmu_dE = 1.0 / (2 * (1 + nu));
    q.dkappa_dE = 2.0 / 3.0 * q.dmu_dE + nu / ((1 + nu) * (1 - 2 * nu));
    q.s4 = 4.0 / (p.cellsize * p.cellsize);
    return q;
}

}  // namespace

namespace {

// While the adjoint recomputes and reverses, a mixed handle is driven as an
// FP64 one with the FP64 SVD, on its FP64 staging rows and FP64 grid.
struct Fp64View {
    mpm_handle* h;
    int saved;
    explicit Fp64View(mpm_handle* hh) : h(hh), saved(hh->precision) {
        if (is_mixed(h)) h->precision = MPM_PRECISION_FP64_SVD64;
    }
    ~Fp64View() { h->precision = saved; }
};

// Mixed forward of the adjoint: the mixed step in segments of ckpt_every
// substeps (each segment's last substep stores v and C), the FP64 staging
// of the state at every segment start as its checkpoint, the force history
// collected in h->adj_force. No sort runs meanwhile (the reverse sweep keeps
// per-particle adjoints by slot).
int adjoint_forward_mixed(mpm_handle* h, int nsteps, int every) {
    const int saved_interval = h->sort_interval;
    h->sort_interval = 0;
    int r = MPM_OK;
    for (int s0 = 0; s0 < nsteps && !r; s0 += every) {
        if ((r = mixed_to_staging(h))) break;
        CK(h, cudaMemcpyAsync(h->ckpt[s0 / every], h->pts, state_bytes(h), cudaMemcpyDeviceToDevice, h->stream));
        h->ckpt_prms[s0 / every] = h->prms;
        const int m = std::min(every, nsteps - s0);
        if ((r = mpm_step(h, m, nullptr))) break;
        CK(h, cudaMemcpyAsync(h->adj_force + 3 * (size_t)s0, h->force_steps, sizeof(double) * 3 * (size_t)m,
                              cudaMemcpyDeviceToDevice, h->stream));
    }
    h->sort_interval = saved_interval;
    return r;
}

}  // namespace

extern "C" int mpm_adjoint_forward(mpm_handle* h, int nsteps, int ckpt_every, double* force_hist) {
    if (!h || nsteps <= 0 || ckpt_every <= 0) return MPM_ERR_ARG;
    if (!h->uploaded) return MPM_ERR_STATE;
    int r = ensure_adjoint_buffers(h, nsteps, ckpt_every);
    if (r) return r;
    if (is_mixed(h)) {
        if (nsteps > h->adj_force_cap) {
            CK(h, cudaStreamSynchronize(h->stream));
            cudaFree(h->adj_force);
            h->adj_force = nullptr;
            CK(h, cudaMalloc(&h->adj_force, sizeof(double) * 3 * (size_t)nsteps));
            h->adj_force_cap = nsteps;
        }
        h->adj_ready = false;
        if ((r = adjoint_forward_mixed(h, nsteps, ckpt_every))) return r;
        if (force_hist)
            CK(h, cudaMemcpyAsync(force_hist, h->adj_force, sizeof(double) * 3 * (size_t)nsteps,
                                  cudaMemcpyDeviceToHost, h->stream));
        CK(h, cudaStreamSynchronize(h->stream));
        h->adj_steps = nsteps;
        h->adj_every = ckpt_every;
        h->adj_ready = true;
        return MPM_OK;
    }
    if (nsteps > h->force_steps_cap) {
        CK(h, cudaStreamSynchronize(h->stream));
        cudaFree(h->force_steps);
        h->force_steps = nullptr;
        CK(h, cudaMalloc(&h->force_steps, sizeof(double) * 3 * (size_t)nsteps));
        h->force_steps_cap = nsteps;
    }
    CK(h, cudaMemsetAsync(h->force_steps, 0, sizeof(double) * 3 * (size_t)nsteps, h->stream));
    for (int s = 0; s < nsteps; s++) {
        if (s % ckpt_every == 0) {
            CK(h, cudaMemcpyAsync(h->ckpt[s / ckpt_every], h->pts, state_bytes(h), cudaMemcpyDeviceToDevice, h->stream));
            h->ckpt_prms[s / ckpt_every] = h->prms;
        }
        if ((r = fp64_substep(h, h->force_steps + 3 * s))) return r;
    }
    if (force_hist)
        CK(h, cudaMemcpyAsync(force_hist, h->force_steps, sizeof(double) * 3 * (size_t)nsteps, cudaMemcpyDeviceToHost,
                              h->stream));
    h->adj_steps = nsteps;
    h->adj_every = ckpt_every;
    h->adj_ready = true;
    int code = 0;
    r = read_error(h, &code);
    return r ? r : code;
}

extern "C" int mpm_adjoint_backward(mpm_handle* h, const double* dL_dforce, double* dL_dcohesion, double* dL_dE) {
    if (!h || !dL_dforce) return MPM_ERR_ARG;
    if (!h->adj_ready) return MPM_ERR_STATE;
    const Fp64View fp64(h);
    const int N = h->adj_steps, k = h->adj_every, n = (int)h->n;
    const DevParams dp = h->dp;
    const AdjParams q = adj_params(h);
    const size_t gs = (size_t)dp.gstride;
    CK(h, cudaMemsetAsync(h->adj_A, 0, sizeof(double) * ADJ_ROWS * h->pitch, h->stream));
    CK(h, cudaMemsetAsync(h->adj_cgrad, 0, sizeof(double) * h->pitch, h->stream));
    CK(h, cudaMemsetAsync(h->adj_Egrad, 0, sizeof(double), h->stream));
    double* const pts_final = h->pts;
    const SimParams3D prms_final = h->prms;
    int r = MPM_OK;
    const int nseg = (N + k - 1) / k;
    for (int j = nseg - 1; j >= 0 && !r; j--) {
        const int s0 = j * k, s1 = std::min(N, s0 + k);
        // recompute the segment's states from its checkpoint
        std::vector<SimParams3D> sp(s1 - s0);
        CK(h, cudaMemcpyAsync(h->seg[0], h->ckpt[j], state_bytes(h), cudaMemcpyDeviceToDevice, h->stream));
        h->prms = h->ckpt_prms[j];
        for (int s = s0; s < s1 && !r; s++) {
            double* next = h->seg[s - s0 + 1];
            CK(h, cudaMemcpyAsync(next, h->seg[s - s0], state_bytes(h), cudaMemcpyDeviceToDevice, h->stream));
            h->pts = next;
            r = fp64_substep(h, h->force_phase, h->adj_gcache[s - s0]);
            sp[s - s0] = h->prms;   // holds this substep's indenter position
        }
        h->pts = pts_final;
        if (r) break;
        // reverse the segment
        for (int s = s1 - 1; s >= s0; s--) {
            const double* Sn = h->seg[s - s0];
            const double* Sn1 = h->seg[s - s0 + 1];
            const double ix = sp[s - s0].indenter_x, iy = sp[s - s0].indenter_y;
            // the substep's P2G grid, as the recompute produced it
            CK(h, cudaMemcpyAsync(h->adj_g7, h->adj_gcache[s - s0], sizeof(double) * 4 * gs, cudaMemcpyDeviceToDevice,
                                  h->stream));
            k_adj_update_record<256><<<blocks_for(dp.nodes, 256), 256, 0, h->stream>>>(dp, h->adj_g7, ix, iy);
            CK(h, cudaMemsetAsync(h->adj_gb7, 0, sizeof(double) * 7 * gs, h->stream));
            k_adj_rm_vjp<128><<<blocks_for(n, 128), 128, 0, h->stream>>>(dp, q, Sn, Sn1, h->pitch, n, h->p0, h->adj_A,
                                                                        h->adj_rmv, h->adj_cgrad, h->adj_Egrad);
            k_adj_g2p_rev<128><<<blocks_for(n, 128), 128, 0, h->stream>>>(dp, q, Sn, Sn1, h->pitch, n, h->adj_g7,
                                                                         h->adj_rmv, h->adj_A, h->adj_gb7);
            k_adj_node_rev<256><<<blocks_for(dp.nodes, 256), 256, 0, h->stream>>>(
                dp, h->adj_g7, h->adj_gb7, ix, iy, dL_dforce[3 * s], dL_dforce[3 * s + 1], dL_dforce[3 * s + 2]);
            k_adj_p2g_rev<128><<<blocks_for(n, 128), 128, 0, h->stream>>>(dp, q, Sn, h->pitch, n, h->adj_gb7, h->adj_A,
                                                                         h->adj_Egrad);
            CK_LAUNCH(h, "adjoint kernels");
        }
    }
    h->pts = pts_final;
    h->prms = prms_final;
    if (r) return r;
    if (dL_dcohesion && n)
        CK(h, cudaMemcpyAsync(dL_dcohesion, h->adj_cgrad, sizeof(double) * n, cudaMemcpyDeviceToHost, h->stream));
    double eg = 0;
    CK(h, cudaMemcpyAsync(&eg, h->adj_Egrad, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CK(h, cudaStreamSynchronize(h->stream));
    if (dL_dE) *dL_dE = eg;
    return MPM_OK;
}

extern "C" int mpm_adjoint_state(mpm_handle* h, double* adj, unsigned pitch) {
    if (!h || !adj || pitch < h->n) return MPM_ERR_ARG;
    if (!h->adj_ready || !h->adj_A) return MPM_ERR_STATE;
    if (h->n)
        CK(h, cudaMemcpy2DAsync(adj, sizeof(double) * pitch, h->adj_A, sizeof(double) * h->pitch, sizeof(double) * h->n,
                                ADJ_ROWS, cudaMemcpyDeviceToHost, h->stream));
    CK(h, cudaStreamSynchronize(h->stream));
    return MPM_OK;
}

extern "C" int mpm_adjoint(mpm_handle* h, int nsteps, int ckpt_every, const double* dL_dforce, double* dL_dcohesion,
                           double* dL_dE) {
    if (!h || !dL_dforce) return MPM_ERR_ARG;
    const int r = mpm_adjoint_forward(h, nsteps, ckpt_every, nullptr);
    if (r) return r;
    return mpm_adjoint_backward(h, dL_dforce, dL_dcohesion, dL_dE);
}
