// Hand-written adjoint (reverse mode) of the FP64 substep, for gradients of
// an indenter-force loss with respect to per-particle cohesion and Young's
// modulus.
//
// Forward substep n (state S_n = x, v, C, F, Jp, status):
//   P2G   m_i = sum_p w_ip m,  P_i = sum_p w_ip (m v_p + Q_p d_ip),
//         Q_p = m C_p - k tau(F_p), k = dt V Dp^-1, d_ip = x_i - x_p
//   node  v1 = P_i/m_i - dt g e_y, speed clamp, cylinder contact
//         v3 = v2 - n (n.(v2 - v_ind)) with force f_i = (v2 - v3) m_i / dt,
//         wall masks; f_n = sum_i f_i
//   G2P   v' = sum_i w v_i, C' = 4/h^2 sum_i w v_i d_ip^T, x' = x + dt v',
//         F_tr = (I + dt C') F, F' = RM(F_tr, Jp, p0, mu, kappa) if crushed
// The reverse of one substep runs three kernels, after recomputing the grid
// of substep n from S_n:
//   k_adj_g2p_rev   particles: adjoint of G2P (including the weight
//                   gradients and the return map), velocity adjoints
//                   scattered to the nodes
//   k_adj_node_rev  nodes: adjoint of the node update (masks, contact
//                   projection, force, clamp, division by the mass)
//   k_adj_p2g_rev   particles: adjoint of P2G as a gather over each
//                   particle's 27 nodes (no atomics), including the
//                   Kirchhoff stress
// The return map's vector-Jacobian product uses the local Jacobian taken by
// forward-mode dual numbers through the same FP64 SVD and projection code
// (one direction per input), so it follows every branch the forward took.
#pragma once

#include "device_common.cuh"
#include "physics_f64.cuh"
#include "svd3.cuh"

namespace icempm {

// ------------------------------------------------------------- dual numbers

struct Dual1 {
    double v, d;
    __device__ Dual1() {}
    __device__ Dual1(double x) : v(x), d(0.0) {}
    __device__ Dual1(double x, double dx) : v(x), d(dx) {}
};
__device__ __forceinline__ Dual1 operator+(Dual1 a, Dual1 b) { return Dual1(a.v + b.v, a.d + b.d); }
__device__ __forceinline__ Dual1 operator-(Dual1 a, Dual1 b) { return Dual1(a.v - b.v, a.d - b.d); }
__device__ __forceinline__ Dual1 operator-(Dual1 a) { return Dual1(-a.v, -a.d); }
__device__ __forceinline__ Dual1 operator*(Dual1 a, Dual1 b) { return Dual1(a.v * b.v, a.d * b.v + a.v * b.d); }
__device__ __forceinline__ Dual1 operator/(Dual1 a, Dual1 b) {
    return Dual1(a.v / b.v, (a.d * b.v - a.v * b.d) / (b.v * b.v));
}
__device__ __forceinline__ bool operator<(Dual1 a, Dual1 b) { return a.v < b.v; }
__device__ __forceinline__ bool operator<=(Dual1 a, Dual1 b) { return a.v <= b.v; }
__device__ __forceinline__ bool operator>(Dual1 a, Dual1 b) { return a.v > b.v; }
__device__ __forceinline__ bool operator>=(Dual1 a, Dual1 b) { return a.v >= b.v; }

__device__ __forceinline__ double gsqrt(double x) { return sqrt(x); }
__device__ __forceinline__ double gcbrt(double x) { return cbrt(x); }
__device__ __forceinline__ double grcbrt(double x) { return rcbrt(x); }
__device__ __forceinline__ double gfmin(double a, double b) { return fmin(a, b); }
__device__ __forceinline__ double gval(double x) { return x; }
__device__ __forceinline__ Dual1 gsqrt(Dual1 x) {
    const double s = sqrt(x.v);
    return Dual1(s, s > 0 ? 0.5 * x.d / s : 0.0);
}
__device__ __forceinline__ Dual1 gcbrt(Dual1 x) {
    const double c = cbrt(x.v);
    return Dual1(c, x.v != 0 ? x.d * c / (3.0 * x.v) : 0.0);
}
__device__ __forceinline__ Dual1 grcbrt(Dual1 x) {
    const double c = rcbrt(x.v);
    return Dual1(c, -x.d * c / (3.0 * x.v));
}
__device__ __forceinline__ Dual1 gfmin(Dual1 a, Dual1 b) { return a.v <= b.v ? a : b; }
__device__ __forceinline__ double gval(Dual1 x) { return x.v; }

// SVD arithmetic on dual numbers (same algorithm and sweeps as SvdF64)
struct SvdDual {
    typedef Dual1 T;
    static constexpr int kSweeps = 8;
    __device__ static __forceinline__ T add(T a, T b) { return a + b; }
    __device__ static __forceinline__ T sub(T a, T b) { return a - b; }
    __device__ static __forceinline__ T mul(T a, T b) { return a * b; }
    __device__ static __forceinline__ T rsqrt(T a) { return Dual1(1.0) / gsqrt(a); }
    __device__ static __forceinline__ T fmax_(T a, T b) { return a.v >= b.v ? a : b; }
    __device__ static __forceinline__ T tiny() { return Dual1(1.e-40); }
    __device__ static __forceinline__ T small() { return Dual1(1.e-40); }
    __device__ static __forceinline__ T four_gamma_sq() { return Dual1(5.828427124746190); }
    __device__ static __forceinline__ T sin_pi8() { return Dual1(0.38268343236508977); }
    __device__ static __forceinline__ T cos_pi8() { return Dual1(0.92387953251128674); }
};

// Material constants of the return map that are not differentiated.
struct RMConst {
    double pmax, tensile, shear, tan_phi;
};

template <class T>
__device__ __forceinline__ T det3g(const T a[3][3]) {
    return a[0][0] * (a[1][1] * a[2][2] - a[2][1] * a[1][2]) - a[1][0] * (a[0][1] * a[2][2] - a[2][1] * a[0][2]) +
           a[2][0] * (a[0][1] * a[1][2] - a[1][1] * a[0][2]);
}

// ComputePQ + ComputeSVD + Wolper_Drucker_Prager (mpm_kernels.cuh:477-544)
// on a generic scalar: F in/out, Jp in/out.
template <class T, class K>
__device__ __forceinline__ void rm_generic(const RMConst& c, T F[3][3], T& Jp, T p0, T mu, T kappa) {
    const T Je = det3g(F);
    const T Jsq = Je * Je;
    const T p_tr = -(T(0.5) * kappa) * (Jsq - T(1.0));
    T b[3][3];
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) b[i][j] = F[i][0] * F[j][0] + F[i][1] * F[j][1] + F[i][2] * F[j][2];
    const T tr3 = (b[0][0] + b[1][1] + b[2][2]) / T(3.0);
    T sq = T(0.0);
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            const T d = (i == j) ? b[i][j] - tr3 : b[i][j];
            sq = sq + d * d;
        }
    const T q_tr = T(kCoeff1) * mu * grcbrt(Jsq) * gsqrt(sq);

    T U[3][3], S[3], V[3][3];
    svd3x3<K>(F, U, S, V);
    T sig2[3];
#pragma unroll
    for (int i = 0; i < 3; i++) sig2[i] = S[i] * S[i];

    T d[3];
    if (gval(p_tr) < -gval(p0) || gval(Jp) < 1.0) {
        const T Je_new = gsqrt(T(2.0) * p0 / kappa + T(1.0));
        const T cc = gcbrt(Je_new);
        d[0] = d[1] = d[2] = cc;
        Jp = Jp * Je_new / Je;
    } else {
        T q_n_1;
        if (gval(p_tr) > c.pmax) {
            q_n_1 = T(0.0);
        } else {
            const T q_from_dp = (p_tr + p0) * T(c.tan_phi);
            const double pmin = -c.tensile;
            const T q_fs = T(2.0) * gsqrt((T(c.pmax) - p_tr) * (p_tr - T(pmin))) * T(c.shear) / T(c.pmax - pmin);
            q_n_1 = gfmin(q_fs, q_from_dp);
        }
        if (!(gval(q_tr) >= gval(q_n_1))) return;   // inside the yield surface: F unchanged
        const T mean = (sig2[0] + sig2[1] + sig2[2]) / T(3.0);
        const T sfac = mu * grcbrt(Jsq);
        T sh[3];
#pragma unroll
        for (int i = 0; i < 3; i++) sh[i] = sfac * (sig2[i] - mean);
        const T nrm = gsqrt(sh[0] * sh[0] + sh[1] * sh[1] + sh[2] * sh[2]);
        const T coef = (q_n_1 * T(kCoeff1Inv)) * gcbrt(Jsq) / mu;
#pragma unroll
        for (int i = 0; i < 3; i++) d[i] = gsqrt(coef * (gval(nrm) > 0 ? sh[i] / nrm : T(0.0)) + mean);
    }
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) F[i][j] = U[i][0] * d[0] * V[j][0] + U[i][1] * d[1] * V[j][1] + U[i][2] * d[2] * V[j][2];
}

// Vector-Jacobian product of the return map: inputs (F_tr[9], Jp, p0, mu,
// kappa), output adjoints (Fb[9], Jpb); one dual pass per input.
__device__ __noinline__ void rm_vjp(const RMConst c, const double Ftr[9], double Jp, double p0, double mu, double kappa,
                                    const double Fb[9], double Jpb, double gin[13]) {
#pragma unroll 1
    for (int j = 0; j < 13; j++) {
        Dual1 F[3][3];
        for (int k = 0; k < 9; k++) F[k / 3][k % 3] = Dual1(Ftr[k], j == k ? 1.0 : 0.0);
        Dual1 J(Jp, j == 9 ? 1.0 : 0.0);
        rm_generic<Dual1, SvdDual>(c, F, J, Dual1(p0, j == 10 ? 1.0 : 0.0), Dual1(mu, j == 11 ? 1.0 : 0.0),
                                   Dual1(kappa, j == 12 ? 1.0 : 0.0));
        double g = Jpb * J.d;
        for (int k = 0; k < 9; k++) g += Fb[k] * F[k / 3][k % 3].d;
        gin[j] = g;
    }
}

// Forward value of the return map on doubles (the FP64-SVD forward).
__device__ __noinline__ void rm_value(const RMConst c, double F[9], double& Jp, double p0, double mu, double kappa) {
    double G[3][3];
    for (int k = 0; k < 9; k++) G[k / 3][k % 3] = F[k];
    rm_generic<double, SvdF64>(c, G, Jp, p0, mu, kappa);
    for (int k = 0; k < 9; k++) F[k] = G[k / 3][k % 3];
}

// quadratic B-spline weights and their derivatives in cell units
__device__ __forceinline__ void quad_w_dw(const double fx[3], double w[3][3], double dw[3][3]) {
#pragma unroll
    for (int d = 0; d < 3; d++) {
        const double v0 = 1.5 - fx[d], v1 = fx[d] - 1.0, v2 = fx[d] - 0.5;
        w[0][d] = 0.5 * v0 * v0;
        w[1][d] = 0.75 - v1 * v1;
        w[2][d] = 0.5 * v2 * v2;
        dw[0][d] = -v0;
        dw[1][d] = -2.0 * v1;
        dw[2][d] = v2;
    }
}

// cofactor matrix: d det(F) / dF
__device__ __forceinline__ void cofactor(const double F[3][3], double cof[3][3]) {
    cof[0][0] = F[1][1] * F[2][2] - F[1][2] * F[2][1];
    cof[0][1] = F[1][2] * F[2][0] - F[1][0] * F[2][2];
    cof[0][2] = F[1][0] * F[2][1] - F[1][1] * F[2][0];
    cof[1][0] = F[0][2] * F[2][1] - F[0][1] * F[2][2];
    cof[1][1] = F[0][0] * F[2][2] - F[0][2] * F[2][0];
    cof[1][2] = F[0][1] * F[2][0] - F[0][0] * F[2][1];
    cof[2][0] = F[0][1] * F[1][2] - F[0][2] * F[1][1];
    cof[2][1] = F[0][2] * F[1][0] - F[0][0] * F[1][2];
    cof[2][2] = F[0][0] * F[1][1] - F[0][1] * F[1][0];
}

// Adjoint of the Kirchhoff stress tau = mu J^(-2/3) dev(F F^T) + kappa/2 (J^2-1) I:
// Fb += dtau/dF^T : taub, mub += dtau/dmu : taub, kappab += dtau/dkappa : taub.
__device__ __forceinline__ void kirchhoff_vjp(double mu, double kappa, const double F[3][3], const double tb[3][3],
                                              double Fb[3][3], double& mub, double& kappab) {
    const double J = det3(F);
    const double a = rcbrt(J * J);
    double b[3][3];
    ffT(F, b);
    const double trb = (b[0][0] + b[1][1] + b[2][2]) / 3;
    const double trt = tb[0][0] + tb[1][1] + tb[2][2];
    double s1 = 0;   // taub : dev(b)
    double D[3][3];  // dev(taub)
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            s1 += tb[i][j] * (b[i][j] - (i == j ? trb : 0.0));
            D[i][j] = tb[i][j] - (i == j ? trt / 3 : 0.0);
        }
    // mu a dev(db), db = dF F^T + F dF^T  ->  mu a (D + D^T) F
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            double acc = 0;
#pragma unroll
            for (int k = 0; k < 3; k++) acc += (D[i][k] + D[k][i]) * F[k][j];
            Fb[i][j] += mu * a * acc;
        }
    // through J: d(J^-2/3) = -2/3 J^-2/3 dJ / J, d(J^2) = 2 J dJ, dJ = cof(F) : dF
    const double Jb = mu * s1 * (-2.0 / 3.0) * a / J + kappa * J * trt;
    double cof[3][3];
    cofactor(F, cof);
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) Fb[i][j] += Jb * cof[i][j];
    mub += a * s1;
    kappab += 0.5 * (J * J - 1.0) * trt;
}

// Rows of the particle adjoint buffer A (pitch doubles per row).
enum { ADJ_X = 0, ADJ_V = 3, ADJ_C = 6, ADJ_F = 15, ADJ_JP = 24, ADJ_ROWS = 25 };

__device__ __forceinline__ void block_add_double(double v, double* out) {
    __shared__ double red[32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) red[warp] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) s += red[w];
        if (s != 0) atomicAdd(out, s);
    }
}

// -------------------------------------------------- node update (recording)

// The node update of k_update_f64 for the reverse sweep: reads m and P
// (arrays 0..3 of a 7-array grid), writes the final velocity to arrays 4..6
// and leaves the momentum in place.
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_adj_update_record(DevParams P, double* __restrict__ g7, double ind_x,
                                                             double ind_y) {
    const long long idx = (long long)blockIdx.x * BLOCK + threadIdx.x;
    if (idx >= P.nodes) return;
    const long long gs = P.gstride;
    const double mass = g7[idx];
    double v[3] = {0, 0, 0};
    if (mass != 0) {
        v[0] = g7[gs + idx] / mass;
        v[1] = g7[2 * gs + idx] / mass;
        v[2] = g7[3 * gs + idx] / mass;
        const int idx_z = (int)(idx % P.Gz), idx_y = (int)((idx / P.Gz) % P.Gy), idx_x = (int)(idx / P.slab);
        const int gx = idx_x - P.halo, gy = idx_y, gz = idx_z;
        v[1] -= P.dt_gravity;
        const double vsq = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
        if (vsq > P.vmax_sq) {
            const double nv = sqrt(vsq);
            for (int k = 0; k < 3; k++) v[k] = v[k] / nv * P.vmax;
        }
        if (P.setup_type != 2) {
            double n0 = gx * P.h - ind_x, n1 = gy * P.h - ind_y;
            const double nsq = n0 * n0 + n1 * n1;
            if (nsq < P.ind_rsq) {
                if (nsq > 0) { const double nn = sqrt(nsq); n0 /= nn; n1 /= nn; }
                const double vn = (v[0] - P.ind_velocity) * n0 + v[1] * n1;
                if (vn < 0) { v[0] -= n0 * vn; v[1] -= n1 * vn; }
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
        if (P.setup_type == 2 && P.drag != 0)
            for (int k = 0; k < 3; k++) v[k] *= (1 - P.drag);
    }
    g7[4 * gs + idx] = v[0];
    g7[5 * gs + idx] = v[1];
    g7[6 * gs + idx] = v[2];
}

// ----------------------------------------------------------- reverse G2P

struct AdjParams {
    RMConst rc;
    double dmu_dE, dkappa_dE;
    double s4;   // 4 / h^2
};

// Vector-Jacobian product of the return map (mpm_kernels.cuh:494-544) for
// the points crushed in this substep, ahead of k_adj_g2p_rev: rmv rows 0-8
// receive dL/dF_tr, row 9 dL/dJp_inv; the cohesion and E terms go to cgrad
// and Egrad. Kept apart from k_adj_g2p_rev so that the dual-number sweep's
// registers do not set that kernel's occupancy.
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_adj_rm_vjp(DevParams P, AdjParams Q, const double* __restrict__ S0,
                                                      const double* __restrict__ S1, size_t pitch, int n,
                                                      const double* __restrict__ p0arr, const double* __restrict__ A,
                                                      double* __restrict__ rmv, double* __restrict__ cgrad,
                                                      double* __restrict__ Egrad) {
    const int i = blockIdx.x * BLOCK + threadIdx.x;
    double eg = 0;
    const long long util = i < n ? __double_as_longlong(S0[i]) : kDisabled;
    if (!(util & kDisabled) && !(util & kLiquid) && (__double_as_longlong(S1[i]) & kCrushed)) {
        const double dt = P.dt;
        double F[3][3], Am[3][3], Ftr9[9], Fb1[9], g[13];
        for (int r = 0; r < 3; r++)
            for (int c = 0; c < 3; c++) {
                F[r][c] = S0[(MPM_FE00 + 3 * r + c) * pitch + i];
                Am[r][c] = (r == c ? 1.0 : 0.0) + dt * S1[(MPM_BP00 + 3 * r + c) * pitch + i];
            }
        for (int r = 0; r < 3; r++)
            for (int c = 0; c < 3; c++) Ftr9[3 * r + c] = Am[r][0] * F[0][c] + Am[r][1] * F[1][c] + Am[r][2] * F[2][c];
        for (int k = 0; k < 9; k++) Fb1[k] = A[(ADJ_F + k) * pitch + i];
        const double Jpb1 = A[ADJ_JP * pitch + i];
        const double p0 = p0arr ? p0arr[i] : P.p0;
        rm_vjp(Q.rc, Ftr9, S0[MPM_IDX_JP_INV * pitch + i], p0, P.mu, P.kappa, Fb1, Jpb1, g);
        for (int k = 0; k < 10; k++) rmv[k * pitch + i] = g[k];
        cgrad[i] += g[10] / Q.rc.tan_phi;
        eg = g[11] * Q.dmu_dE + g[12] * Q.dkappa_dE;
    }
    block_add_double(eg, Egrad);
}

template <int BLOCK>
__global__ void __launch_bounds__(BLOCK, 3) k_adj_g2p_rev(DevParams P, AdjParams Q, const double* __restrict__ S0,
                                                       const double* __restrict__ S1, size_t pitch, int n,
                                                       const double* __restrict__ g7,
                                                       const double* __restrict__ rmv, double* __restrict__ A,
                                                       double* __restrict__ gadj) {
    const int i = blockIdx.x * BLOCK + threadIdx.x;
    const long long util = i < n ? __double_as_longlong(S0[i]) : kDisabled;
    if (!(util & kDisabled)) {
        const long long util1 = __double_as_longlong(S1[i]);
        const bool liquid = (util & kLiquid) != 0;
        const bool crushed = !liquid && (util1 & kCrushed);
        const double h = P.h, dt = P.dt, s4 = Q.s4;
        double x[3], F[3][3];
#pragma unroll
        for (int d = 0; d < 3; d++) x[d] = S0[(MPM_POSX + d) * pitch + i];
#pragma unroll
        for (int r = 0; r < 3; r++)
#pragma unroll
            for (int c = 0; c < 3; c++) F[r][c] = S0[(MPM_FE00 + 3 * r + c) * pitch + i];
        const double Jp = S0[MPM_IDX_JP_INV * pitch + i];
        int base[3];
        double fx[3], w[3][3], dw[3][3];
#pragma unroll
        for (int d = 0; d < 3; d++) {
            base[d] = (int)(x[d] * P.h_inv - 0.5);
            fx[d] = x[d] * P.h_inv - (double)base[d];
        }
        quad_w_dw(fx, w, dw);
        double dwh[3][3];   // weight derivatives per unit length (d/dx = d/dfx / h)
#pragma unroll
        for (int k = 0; k < 3; k++)
#pragma unroll
            for (int d = 0; d < 3; d++) dwh[k][d] = dw[k][d] * P.h_inv;
        // C' of this substep: the G2P that produced S1 stored it (the Bp rows)
        double Cp[3][3];
#pragma unroll
        for (int r = 0; r < 3; r++)
#pragma unroll
            for (int c = 0; c < 3; c++) Cp[r][c] = S1[(MPM_BP00 + 3 * r + c) * pitch + i];
        double Am[3][3], Ftr[3][3];
#pragma unroll
        for (int r = 0; r < 3; r++)
#pragma unroll
            for (int c = 0; c < 3; c++) Am[r][c] = (r == c ? 1.0 : 0.0) + dt * Cp[r][c];
#pragma unroll
        for (int r = 0; r < 3; r++)
#pragma unroll
            for (int c = 0; c < 3; c++) Ftr[r][c] = Am[r][0] * F[0][c] + Am[r][1] * F[1][c] + Am[r][2] * F[2][c];
        // adjoints of S_{n+1}
        double xb[3], vb[3], Cb[3][3], Fb1[9], Jpb1;
#pragma unroll
        for (int d = 0; d < 3; d++) { xb[d] = A[(ADJ_X + d) * pitch + i]; vb[d] = A[(ADJ_V + d) * pitch + i]; }
#pragma unroll
        for (int k = 0; k < 9; k++) { Cb[k / 3][k % 3] = A[(ADJ_C + k) * pitch + i]; Fb1[k] = A[(ADJ_F + k) * pitch + i]; }
        Jpb1 = A[ADJ_JP * pitch + i];
        // return map (and liquid volume update)
        double Ftrb[3][3], Jpb0 = Jpb1, Ab[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
#pragma unroll
        for (int k = 0; k < 9; k++) Ftrb[k / 3][k % 3] = Fb1[k];
        if (crushed) {
            // the return map's VJP, from k_adj_rm_vjp (which also took its
            // cohesion and E terms)
#pragma unroll
            for (int k = 0; k < 9; k++) Ftrb[k / 3][k % 3] = rmv[k * pitch + i];
            Jpb0 = rmv[9 * pitch + i];
        } else if (liquid) {
            const double detA = det3(Am);
            double cof[3][3];
            cofactor(Am, cof);
            Jpb0 = Jpb1 * detA;
#pragma unroll
            for (int r = 0; r < 3; r++)
#pragma unroll
                for (int c = 0; c < 3; c++) Ab[r][c] += Jpb1 * Jp * cof[r][c];
        }
        // F_tr = A F
        double Fb0[3][3];
#pragma unroll
        for (int r = 0; r < 3; r++)
#pragma unroll
            for (int c = 0; c < 3; c++) {
                Ab[r][c] += Ftrb[r][0] * F[c][0] + Ftrb[r][1] * F[c][1] + Ftrb[r][2] * F[c][2];
                Fb0[r][c] = Am[0][r] * Ftrb[0][c] + Am[1][r] * Ftrb[1][c] + Am[2][r] * Ftrb[2][c];
            }
        double Cbt[3][3], vbt[3];
#pragma unroll
        for (int r = 0; r < 3; r++) {
            vbt[r] = vb[r] + dt * xb[r];
#pragma unroll
            for (int c = 0; c < 3; c++) Cbt[r][c] = Cb[r][c] + dt * Ab[r][c];
        }
        // gather adjoint: node velocity adjoints and x-gradients
        double xb0[3] = {xb[0], xb[1], xb[2]};
#pragma unroll
        for (int a = 0; a < 3; a++)
#pragma unroll
            for (int b = 0; b < 3; b++)
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    const int nx = base[0] + a, ny = base[1] + b, nz = base[2] + c;
                    if (!node_inside(P, nx, ny, nz)) continue;
                    const long long ni = node_index(P, nx, ny, nz);
                    const double wt = w[a][0] * w[b][1] * w[c][2];
                    const double gw[3] = {dwh[a][0] * w[b][1] * w[c][2], w[a][0] * dwh[b][1] * w[c][2],
                                          w[a][0] * w[b][1] * dwh[c][2]};
                    const double nv[3] = {g7[4 * P.gstride + ni], g7[5 * P.gstride + ni], g7[6 * P.gstride + ni]};
                    const double dd[3] = {(a - fx[0]) * h, (b - fx[1]) * h, (c - fx[2]) * h};
                    double gsc = 0;
#pragma unroll
                    for (int r = 0; r < 3; r++) {
                        const double cd = Cbt[r][0] * dd[0] + Cbt[r][1] * dd[1] + Cbt[r][2] * dd[2];
                        atomicAdd(gadj + r * P.gstride + ni, wt * vbt[r] + s4 * wt * cd);
                        gsc += nv[r] * (vbt[r] + s4 * cd);
                    }
#pragma unroll
                    for (int d = 0; d < 3; d++) {
                        const double ctv = Cbt[0][d] * nv[0] + Cbt[1][d] * nv[1] + Cbt[2][d] * nv[2];
                        xb0[d] += gw[d] * gsc - s4 * wt * ctv;
                    }
                }
#pragma unroll
        for (int d = 0; d < 3; d++) {
            A[(ADJ_X + d) * pitch + i] = xb0[d];
            A[(ADJ_V + d) * pitch + i] = 0.0;
        }
#pragma unroll
        for (int k = 0; k < 9; k++) {
            A[(ADJ_C + k) * pitch + i] = 0.0;
            A[(ADJ_F + k) * pitch + i] = Fb0[k / 3][k % 3];
        }
        A[ADJ_JP * pitch + i] = Jpb0;
    }
}

// ---------------------------------------------------------- reverse node

template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_adj_node_rev(DevParams P, const double* __restrict__ g7,
                                                        double* __restrict__ gadj, double ind_x, double ind_y,
                                                        double fb0, double fb1, double fb2) {
    const long long idx = (long long)blockIdx.x * BLOCK + threadIdx.x;
    if (idx >= P.nodes) return;
    const long long gs = P.gstride;
    const double mass = g7[idx];
    double mb = 0, Pb[3] = {0, 0, 0};
    if (mass != 0) {
        const double Pm[3] = {g7[gs + idx], g7[2 * gs + idx], g7[3 * gs + idx]};
        double v1[3] = {Pm[0] / mass, Pm[1] / mass - P.dt_gravity, Pm[2] / mass};
        const int idx_z = (int)(idx % P.Gz), idx_y = (int)((idx / P.Gz) % P.Gy), idx_x = (int)(idx / P.slab);
        const int gx = idx_x - P.halo, gy = idx_y, gz = idx_z;
        const double vsq = v1[0] * v1[0] + v1[1] * v1[1] + v1[2] * v1[2];
        const bool clamped = vsq > P.vmax_sq;
        const double nv1 = sqrt(vsq);
        double v2[3];
        for (int k = 0; k < 3; k++) v2[k] = clamped ? v1[k] / nv1 * P.vmax : v1[k];
        bool contact = false;
        double n0 = 0, n1 = 0, vn = 0;
        double v3[3] = {v2[0], v2[1], v2[2]};
        if (P.setup_type != 2) {
            n0 = gx * P.h - ind_x;
            n1 = gy * P.h - ind_y;
            const double nsq = n0 * n0 + n1 * n1;
            if (nsq < P.ind_rsq) {
                if (nsq > 0) { const double nn = sqrt(nsq); n0 /= nn; n1 /= nn; }
                vn = (v2[0] - P.ind_velocity) * n0 + v2[1] * n1;
                if (vn < 0) {
                    contact = true;
                    v3[0] -= n0 * vn;
                    v3[1] -= n1 * vn;
                }
            }
        }
        // wall masks as in the forward (on v3)
        double mk[3] = {1, 1, 1};
        if (P.setup_type != 2) {
            if (gy <= 2) mk[0] = mk[1] = mk[2] = 0;
        } else {
            if (gy <= 2 && v3[1] < 0) mk[1] = 0;
        }
        if (gy >= P.Gy - 3 && v3[1] > 0) mk[1] = 0;
        if (gx <= 2 && v3[0] < 0) mk[0] = 0;
        else if (gx >= P.Gx - 3 && v3[0] > 0) mk[0] = 0;
        if (gz <= 2 && v3[2] < 0) mk[2] = 0;
        else if (gz >= P.Gz - 3 && v3[2] > 0) mk[2] = 0;
        const double drag = (P.setup_type == 2 && P.drag != 0) ? (1 - P.drag) : 1.0;
        double vb3[3];
        for (int k = 0; k < 3; k++) vb3[k] = mk[k] * drag * gadj[k * gs + idx];
        double vb2[3] = {vb3[0], vb3[1], vb3[2]};
        if (contact) {
            const double nb = n0 * vb3[0] + n1 * vb3[1];
            vb2[0] -= n0 * nb;
            vb2[1] -= n1 * nb;
            // force f = n vn m / dt
            const double fn = n0 * fb0 + n1 * fb1;
            vb2[0] += fn * mass / P.dt * n0;
            vb2[1] += fn * mass / P.dt * n1;
            mb += fn * vn / P.dt;
        }
        (void)fb2;
        double vb1[3];
        if (clamped) {
            const double vh[3] = {v1[0] / nv1, v1[1] / nv1, v1[2] / nv1};
            const double dot = vh[0] * vb2[0] + vh[1] * vb2[1] + vh[2] * vb2[2];
            for (int k = 0; k < 3; k++) vb1[k] = P.vmax / nv1 * (vb2[k] - vh[k] * dot);
        } else {
            for (int k = 0; k < 3; k++) vb1[k] = vb2[k];
        }
        for (int k = 0; k < 3; k++) {
            Pb[k] = vb1[k] / mass;
            mb -= vb1[k] * Pm[k] / (mass * mass);
        }
    }
    gadj[3 * gs + idx] = mb;
    gadj[4 * gs + idx] = Pb[0];
    gadj[5 * gs + idx] = Pb[1];
    gadj[6 * gs + idx] = Pb[2];
}

// ----------------------------------------------------------- reverse P2G

template <int BLOCK>
__global__ void __launch_bounds__(BLOCK, 4) k_adj_p2g_rev(DevParams P, AdjParams Q, const double* __restrict__ S0,
                                                       size_t pitch, int n, const double* __restrict__ gadj,
                                                       double* __restrict__ A, double* __restrict__ Egrad) {
    const int i = blockIdx.x * BLOCK + threadIdx.x;
    double eg = 0;
    const long long util = i < n ? __double_as_longlong(S0[i]) : kDisabled;
    if (!(util & kDisabled)) {
        const bool liquid = (util & kLiquid) != 0;
        const double h = P.h;
        const double mass = liquid ? P.liquid_mass : P.particle_mass;
        double x[3], v[3], C[3][3], F[3][3];
#pragma unroll
        for (int d = 0; d < 3; d++) {
            x[d] = S0[(MPM_POSX + d) * pitch + i];
            v[d] = S0[(MPM_VELX + d) * pitch + i];
        }
#pragma unroll
        for (int r = 0; r < 3; r++)
#pragma unroll
            for (int c = 0; c < 3; c++) {
                C[r][c] = S0[(MPM_BP00 + 3 * r + c) * pitch + i];
                F[r][c] = S0[(MPM_FE00 + 3 * r + c) * pitch + i];
            }
        const double Jp = S0[MPM_IDX_JP_INV * pitch + i];
        double tau[3][3];
        if (liquid) {
            const double pw = water_pressure(P, Jp);
#pragma unroll
            for (int r = 0; r < 3; r++)
#pragma unroll
                for (int c = 0; c < 3; c++) tau[r][c] = r == c ? pw : 0.0;
        } else {
            kirchhoff_wolper(P, F, tau);
        }
        double Qm[3][3];
#pragma unroll
        for (int r = 0; r < 3; r++)
#pragma unroll
            for (int c = 0; c < 3; c++) Qm[r][c] = mass * C[r][c] - P.dt_vol_Dpinv * tau[r][c];
        int base[3];
        double fx[3], w[3][3], dw[3][3];
#pragma unroll
        for (int d = 0; d < 3; d++) {
            base[d] = (int)(x[d] * P.h_inv - 0.5);
            fx[d] = x[d] * P.h_inv - (double)base[d];
        }
        quad_w_dw(fx, w, dw);
        double dwh[3][3];   // weight derivatives per unit length (d/dx = d/dfx / h)
#pragma unroll
        for (int k = 0; k < 3; k++)
#pragma unroll
            for (int d = 0; d < 3; d++) dwh[k][d] = dw[k][d] * P.h_inv;
        double xb[3] = {0, 0, 0}, sP[3] = {0, 0, 0}, Qb[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
#pragma unroll
        for (int a = 0; a < 3; a++)
#pragma unroll
            for (int b = 0; b < 3; b++)
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    const int nx = base[0] + a, ny = base[1] + b, nz = base[2] + c;
                    if (!node_inside(P, nx, ny, nz)) continue;
                    const long long ni = node_index(P, nx, ny, nz);
                    const double wt = w[a][0] * w[b][1] * w[c][2];
                    const double gw[3] = {dwh[a][0] * w[b][1] * w[c][2], w[a][0] * dwh[b][1] * w[c][2],
                                          w[a][0] * w[b][1] * dwh[c][2]};
                    const double mb = gadj[3 * P.gstride + ni];
                    const double Pb[3] = {gadj[4 * P.gstride + ni], gadj[5 * P.gstride + ni], gadj[6 * P.gstride + ni]};
                    const double dd[3] = {(a - fx[0]) * h, (b - fx[1]) * h, (c - fx[2]) * h};
                    double g = mass * mb;
#pragma unroll
                    for (int r = 0; r < 3; r++) {
                        const double cr = mass * v[r] + Qm[r][0] * dd[0] + Qm[r][1] * dd[1] + Qm[r][2] * dd[2];
                        g += Pb[r] * cr;
                        sP[r] += wt * Pb[r];
#pragma unroll
                        for (int k = 0; k < 3; k++) Qb[r][k] += wt * Pb[r] * dd[k];
                    }
#pragma unroll
                    for (int d = 0; d < 3; d++) {
                        const double qtp = Qm[0][d] * Pb[0] + Qm[1][d] * Pb[1] + Qm[2][d] * Pb[2];
                        xb[d] += gw[d] * g - wt * qtp;
                    }
                }
        // Q = m C - k tau
        double Fb[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}}, tb[3][3];
#pragma unroll
        for (int r = 0; r < 3; r++)
#pragma unroll
            for (int c = 0; c < 3; c++) tb[r][c] = -P.dt_vol_Dpinv * Qb[r][c];
        double mub = 0, kb = 0, Jpb = 0;
        if (liquid) {
            const double trt = tb[0][0] + tb[1][1] + tb[2][2];
            Jpb = P.kappa * 3.0 * pow(Jp, -4.0) * trt;
            kb += (1.0 - pow(Jp, -3.0)) * trt;
        } else {
            kirchhoff_vjp(P.mu, P.kappa, F, tb, Fb, mub, kb);
        }
        eg += mub * Q.dmu_dE + kb * Q.dkappa_dE;
#pragma unroll
        for (int d = 0; d < 3; d++) {
            A[(ADJ_X + d) * pitch + i] += xb[d];
            A[(ADJ_V + d) * pitch + i] = mass * sP[d];
        }
#pragma unroll
        for (int k = 0; k < 9; k++) {
            A[(ADJ_C + k) * pitch + i] = mass * Qb[k / 3][k % 3];
            A[(ADJ_F + k) * pitch + i] += Fb[k / 3][k % 3];
        }
        A[ADJ_JP * pitch + i] += Jpb;
    }
    block_add_double(eg, Egrad);
}

}  // namespace icempm
