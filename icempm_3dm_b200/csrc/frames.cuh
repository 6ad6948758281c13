// Animation-frame records of SnapshotManager::SaveFrame
// (simulation/snapshotmanager.cpp:116-293, converter/visualpoint.{h,cpp}),
// built on the device.
//
// A full frame stores every non-disabled point as a VisualPoint (float
// position, velocity, Jp_inv, status byte = partition id | 0x80 if crushed)
// and keeps that visual state, with the frame of each point's last position
// refresh. A partial frame compares each non-disabled point (visual index =
// its rank among the non-disabled points) with the visual state:
//   - |pos - (vpos + vvel * (float)(dt * elapsed * UpdateEveryNthStep))| >
//     animation_threshold_pos  -> UpdatePos record {rank, pos, vel}, and the
//     point's refresh frame becomes this frame;
//   - |vJp_inv - Jp_inv| > 1e-2 -> UpdateJp record {rank, Jp_inv};
//   - status byte changed       -> UpdateStatus record {rank, status}.
// Records appear in point order (stable compaction by prefix sums). As in
// the reference, where the loop modifies a copy of visual_state[count]
// (snapshotmanager.cpp:177), a partial frame changes only the refresh frame:
// the stored positions, velocities, Jp_inv and status bytes stay those of
// the last full frame.
//
// The float arithmetic is that of the reference's host code (Eigen on
// Vector3f, no fused multiply-add): products and sums are rounded one by one
// (__fmul_rn / __fadd_rn), the norm is sqrt((x*x + y*y) + z*z).
#pragma once
#include "device_common.cuh"
#include "kernels_mixed.cuh"

namespace icempm {

struct VisualPointRec {     // VisualPoint (converter/visualpoint.h:7-11), 32 bytes
    float pos[3], vel[3], jp_inv;
    unsigned char status, pad[3];
};
struct UpdPosRec {           // std::pair<int, std::array<float, 6>>, 28 bytes
    int idx;
    float pv[6];
};
struct UpdJpRec {            // std::pair<int, float>, 8 bytes
    int idx;
    float jp_inv;
};
struct UpdStatusRec {        // std::pair<int, uint8_t>, 8 bytes
    int idx;
    unsigned char status, pad[3];
};
static_assert(sizeof(VisualPointRec) == 32 && sizeof(UpdPosRec) == 28 && sizeof(UpdJpRec) == 8 &&
                  sizeof(UpdStatusRec) == 8,
              "record layouts of the reference");

struct FramePoint {
    float pos[3], vel[3], jp;
    unsigned char status;
    bool keep;
};

__device__ __forceinline__ unsigned char frame_status_byte(long long u) {
    // ProxyPoint3D::getPartition (proxypoint3d.cpp:112-118) | crushed bit
    return (unsigned char)(((u >> 24) & 0xff) | ((u & kCrushed) ? 0x80 : 0));
}

// FP64 modes: the 28-row SoA, values cast to float as pos.cast<float>() does.
struct FramePointsF64 {
    const double* pts;
    size_t pitch;
    __device__ __forceinline__ void get(int i, FramePoint& q) const {
        const long long u = __double_as_longlong(pts[(size_t)MPM_IDX_UTILITY * pitch + i]);
        q.keep = !(u & kDisabled);
#pragma unroll
        for (int d = 0; d < 3; d++) {
            q.pos[d] = (float)pts[(size_t)(MPM_POSX + d) * pitch + i];
            q.vel[d] = (float)pts[(size_t)(MPM_VELX + d) * pitch + i];
        }
        q.jp = (float)pts[(size_t)MPM_IDX_JP_INV * pitch + i];
        q.status = frame_status_byte(u);
    }
};

// Mixed mode: the same double values mpm_download_soa produces (position
// = X * 2^-20 * h, Jp_inv = 1 + (Jp_inv - 1)), cast to float.
struct FramePointsMixed {
    MixedState s;
    double h;
    __device__ __forceinline__ void get(int i, FramePoint& q) const {
        const int st = s.status[i];
        q.keep = !(st & (int)kDisabled);
#pragma unroll
        for (int d = 0; d < 3; d++) {
            q.pos[d] = (float)((double)s.X[d * s.pitch + i] * (1.0 / (double)(1 << kFixBits)) * h);
            q.vel[d] = s.v[d * s.pitch + i];
        }
        q.jp = (float)(1.0 + (double)s.Jpm1[i]);
        q.status = frame_status_byte((long long)(unsigned)st);
    }
};

// The kept visual state, rows of `cap` entries indexed by visual index.
struct FrameVis {
    float* pos;              // 3 rows
    float* vel;              // 3 rows
    float* jp;
    unsigned char* status;
    int* last;               // frame of the last position refresh
    size_t cap;
};

template <class Pts>
__global__ void __launch_bounds__(256) k_frame_keep(Pts pts, int n, int* __restrict__ keep) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    FramePoint q;
    pts.get(i, q);
    keep[i] = q.keep ? 1 : 0;
}

template <class Pts>
__global__ void __launch_bounds__(256) k_frame_full(Pts pts, int n, const int* __restrict__ rank, FrameVis v,
                                                    int frame, VisualPointRec* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    FramePoint q;
    pts.get(i, q);
    if (!q.keep) return;
    const int c = rank[i];
    VisualPointRec r;
#pragma unroll
    for (int d = 0; d < 3; d++) {
        r.pos[d] = q.pos[d];
        r.vel[d] = q.vel[d];
        v.pos[d * v.cap + c] = q.pos[d];
        v.vel[d * v.cap + c] = q.vel[d];
    }
    r.jp_inv = q.jp;
    r.status = q.status;
    r.pad[0] = r.pad[1] = r.pad[2] = 0;
    v.jp[c] = q.jp;
    v.status[c] = q.status;
    v.last[c] = frame;
    out[c] = r;
}

// flags[k * stride + i], k = 0 position/velocity, 1 Jp_inv, 2 status
// (stride > n: each row ends with a zero sentinel the caller sets)
template <class Pts>
__global__ void __launch_bounds__(256) k_frame_flags(Pts pts, int n, const int* __restrict__ rank, FrameVis v,
                                                     int frame, double dt, int coeff, double threshold_pos,
                                                     int* __restrict__ flags, size_t stride) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    FramePoint q;
    pts.get(i, q);
    int fpv = 0, fjp = 0, fst = 0;
    if (q.keep) {
        const int c = rank[i];
        const int elapsed = frame - v.last[c];
        const float f = (float)(dt * (double)elapsed * (double)coeff);
        float e[3];
#pragma unroll
        for (int d = 0; d < 3; d++) {
            const float pred = __fadd_rn(v.pos[d * v.cap + c], __fmul_rn(v.vel[d * v.cap + c], f));
            e[d] = __fsub_rn(q.pos[d], pred);
        }
        const float n2 = __fadd_rn(__fadd_rn(__fmul_rn(e[0], e[0]), __fmul_rn(e[1], e[1])), __fmul_rn(e[2], e[2]));
        if ((double)__fsqrt_rn(n2) > threshold_pos) {
            fpv = 1;
            v.last[c] = frame;
        }
        fjp = fabsf(__fsub_rn(v.jp[c], q.jp)) > 1e-2f;
        fst = v.status[c] != q.status;
    }
    flags[i] = fpv;
    flags[stride + i] = fjp;
    flags[2 * stride + i] = fst;
}

template <class Pts>
__global__ void __launch_bounds__(256) k_frame_emit(Pts pts, int n, const int* __restrict__ rank,
                                                    const int* __restrict__ flags, const int* __restrict__ offs,
                                                    size_t m, UpdPosRec* __restrict__ upv,
                                                    UpdJpRec* __restrict__ ujp, UpdStatusRec* __restrict__ ust) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int f0 = flags[i], f1 = flags[m + i], f2 = flags[2 * m + i];
    if (!(f0 | f1 | f2)) return;
    FramePoint q;
    pts.get(i, q);
    const int c = rank[i];
    if (f0) {
        UpdPosRec r;
        r.idx = c;
#pragma unroll
        for (int d = 0; d < 3; d++) { r.pv[d] = q.pos[d]; r.pv[3 + d] = q.vel[d]; }
        upv[offs[i]] = r;
    }
    if (f1) {
        UpdJpRec r;
        r.idx = c;
        r.jp_inv = q.jp;
        ujp[offs[m + i]] = r;
    }
    if (f2) {
        UpdStatusRec r;
        r.idx = c;
        r.status = q.status;
        r.pad[0] = r.pad[1] = r.pad[2] = 0;
        ust[offs[2 * m + i]] = r;
    }
}

}  // namespace icempm
