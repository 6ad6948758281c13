// CPU ORACLE — test infrastructure, not product code.
//
// Restatement, in plain C++ with explicit 3x3 arithmetic (the reference uses
// Eigen in device code), of the single-partition step of
// simulation/mpm_kernels.cuh. Each function cites the lines it follows. The
// parity status of this file is described in mpm_oracle.h: the whole step is
// pinned against the reference's own kernels compiled on the host, the SVD
// bit for bit.
//
// The per-particle and per-node functions are templated on the scalar type:
// double is the oracle proper; Dual (dual.h) runs the same arithmetic with a
// tangent attached, the FP64 forward-mode derivative of the step
// (or_dual_steps) that checks the product's hand-written adjoint.
//
// Deviations from the reference, all on invalid input only:
//   - a particle whose stencil leaves the grid raises the error code as the
//     reference does (mpm_kernels.cuh:70-75) but its out-of-grid stencil
//     nodes are skipped (the reference writes/reads outside its buffer);
//   - G2P applies the same bounds check (the reference has none there).

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "dual.h"
#include "mpm_oracle.h"

namespace {

const double kCoeff1 = 1.224744871391589;      // sqrt(3/2), mpm_kernels.cuh:11
const double kCoeff1Inv = 0.8164965809277260;  // mpm_kernels.cuh:12

template <class T> struct M3 { T a[3][3]; };

template <class T> inline M3<T> zero3() {
    M3<T> m;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) m.a[i][j] = 0.0;
    return m;
}
template <class T> inline M3<T> eye3() { M3<T> m = zero3<T>(); m.a[0][0] = m.a[1][1] = m.a[2][2] = 1.0; return m; }

template <class T> inline M3<T> mul(const M3<T>& A, const M3<T>& B) {
    M3<T> C;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++)
            C.a[i][j] = A.a[i][0] * B.a[0][j] + A.a[i][1] * B.a[1][j] + A.a[i][2] * B.a[2][j];
    return C;
}
template <class T> inline M3<T> mul_abt(const M3<T>& A, const M3<T>& B) {  // A * B^T
    M3<T> C;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++)
            C.a[i][j] = A.a[i][0] * B.a[j][0] + A.a[i][1] * B.a[j][1] + A.a[i][2] * B.a[j][2];
    return C;
}
// Eigen's 3x3 determinant: expansion along the first row.
template <class T> inline T det3(const M3<T>& m) {
    const T (*a)[3] = m.a;
    return a[0][0] * (a[1][1] * a[2][2] - a[2][1] * a[1][2])
         - a[1][0] * (a[0][1] * a[2][2] - a[2][1] * a[0][2])
         + a[2][0] * (a[0][1] * a[1][2] - a[1][1] * a[0][2]);
}
template <class T> inline T trace3(const M3<T>& m) { return m.a[0][0] + m.a[1][1] + m.a[2][2]; }
// dev(A) = A - tr(A)/3 I   (mpm_kernels.cuh:569-572)
template <class T> inline M3<T> dev3(const M3<T>& A) {
    M3<T> D = A;
    T t = trace3(A) / 3;
    for (int i = 0; i < 3; i++) D.a[i][i] -= t;
    return D;
}
template <class T> inline T fro_norm(const M3<T>& A) {
    T s = 0.0;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) s += A.a[i][j] * A.a[i][j];
    return sc::sqrt(s);
}
template <class T> inline T rcbrt_h(const T& x) { return 1.0 / sc::cbrt(x); }

inline long long util_bits(double d) { long long v; std::memcpy(&v, &d, 8); return v; }
inline double util_double(long long v) { double d; std::memcpy(&d, &v, 8); return d; }

// The elastic moduli, the only parameters carrying a tangent (d/dE) in the
// forward-mode derivative. For T = double they are prms.mu and prms.kappa.
template <class T> struct Elastic { T mu, kappa; };

// KirchhoffStress_Wolper (mpm_kernels.cuh:547-557)
template <class T> M3<T> kirchhoff_wolper(const Elastic<T>& E, const M3<T>& F) {
    T Je = det3(F);
    M3<T> b = mul_abt(F, F);
    M3<T> d = dev3(b);
    T s = E.mu * rcbrt_h(Je * Je);
    T hyd = E.kappa * 0.5 * (Je * Je - 1.);
    M3<T> t;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) t.a[i][j] = s * d.a[i][j] + (i == j ? hyd : T(0.0));
    return t;
}

// Water (mpm_kernels.cuh:559-566)
template <class T> M3<T> water(const Elastic<T>& E, const T& J) {
    M3<T> t = zero3<T>();
    T v = E.kappa * (1. - sc::pow(J, -3.0));
    t.a[0][0] = t.a[1][1] = t.a[2][2] = v;
    return t;
}

template <class T> struct PointState {
    T pos[3], vel[3];
    M3<T> Fe, Bp;
    T Jp_inv;
    short grain;
    T p_tr, q_tr, Je_tr;
    M3<T> U, V;
    T vSigma[3], vSigmaSquared[3], v_s_hat_tr[3];
    long long utility;
};

// GetParametersForGrain (mpm_kernels.cuh:434-450)
void grain_params(const SimParams3D& P, short grain, double& pmin, double& pmax, double& qmax,
                  double& beta, double& mSq, double& pmin2) {
    double var2 = 1.0 + P.GrainVariability * 0.033 * (-15 + (grain + 3) % 30);
    double var3 = 1.0 + P.GrainVariability * 0.1 * (-10 + (grain + 4) % 11);
    pmax = P.IceCompressiveStrength;
    pmin = -P.IceTensileStrength;
    qmax = P.IceShearStrength * var3;
    pmin2 = -P.IceTensileStrength2 * var2;
    beta = P.NACC_beta;
    mSq = (4 * qmax * qmax * (1 + 2 * beta)) / ((pmax - pmin) * (pmax - pmin));
}

// CheckIfPointIsInsideFailureSurface (mpm_kernels.cuh:453-474)
template <class T> void check_failure_surface(const SimParams3D& P, PointState<T>& p) {
    double beta, M_sq, pmin, pmax, qmax, pmin2;
    grain_params(P, p.grain, pmin, pmax, qmax, beta, M_sq, pmin2);
    if (p.p_tr < 0) {
        if (p.p_tr < pmin2) { p.utility |= MPM_STATUS_CRUSHED; return; }
        double q0 = 2 * std::sqrt(-pmax * pmin) * qmax / (pmax - pmin);
        double k = -q0 / pmin2;
        T q_limit = k * (p.p_tr - pmin2);
        if (p.q_tr > q_limit) { p.utility |= MPM_STATUS_CRUSHED; return; }
    } else {
        T y = (1. + 2. * beta) * p.q_tr * p.q_tr + M_sq * (p.p_tr + beta * pmax) * (p.p_tr - pmax);
        if (y > 0) p.utility |= MPM_STATUS_CRUSHED;
    }
}

// ComputePQ (mpm_kernels.cuh:477-484)
template <class T> void compute_pq(const Elastic<T>& E, PointState<T>& p) {
    p.Je_tr = det3(p.Fe);
    T Jsq = p.Je_tr * p.Je_tr;
    p.p_tr = -(0.5 * E.kappa) * (Jsq - 1.);
    p.q_tr = kCoeff1 * E.mu * rcbrt_h(Jsq) * fro_norm(dev3(mul_abt(p.Fe, p.Fe)));
}

inline void svd_call(const double A[9], double U[9], double S[3], double V[9], int svd_mode) {
    if (svd_mode == 0) or_svd3x3_f32(A, U, S, V);
    else or_svd3x3_f64(A, U, S, V, 8);
}
// The forward-mode derivative differentiates the FP64 SVD (svd_mode 1).
inline void svd_call(const Dual A[9], Dual U[9], Dual S[3], Dual V[9], int) {
    double a[9], da[9], u[9], du[9], s[3], ds[3], v[9], dv[9];
    for (int k = 0; k < 9; k++) { a[k] = A[k].v; da[k] = A[k].d; }
    or_svd3x3_dual(a, da, u, du, s, ds, v, dv, 8);
    for (int k = 0; k < 9; k++) { U[k] = Dual(u[k], du[k]); V[k] = Dual(v[k], dv[k]); }
    for (int k = 0; k < 3; k++) S[k] = Dual(s[k], ds[k]);
}

// ComputeSVD (mpm_kernels.cuh:486-492) with svd3x3 (:585-601)
template <class T> void compute_svd(const Elastic<T>& E, PointState<T>& p, int svd_mode) {
    T A[9], U[9], S[3], V[9];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) A[3 * i + j] = p.Fe.a[i][j];
    svd_call(A, U, S, V, svd_mode);
    for (int i = 0; i < 3; i++) {
        p.vSigma[i] = S[i];
        for (int j = 0; j < 3; j++) { p.U.a[i][j] = U[3 * i + j]; p.V.a[i][j] = V[3 * i + j]; }
    }
    for (int i = 0; i < 3; i++) p.vSigmaSquared[i] = p.vSigma[i] * p.vSigma[i];
    T Je_tr_sq = p.Je_tr * p.Je_tr;
    T mean = (p.vSigmaSquared[0] + p.vSigmaSquared[1] + p.vSigmaSquared[2]) / 3;   // dev_d, :578-581
    T s = E.mu * rcbrt_h(Je_tr_sq);
    for (int i = 0; i < 3; i++) p.v_s_hat_tr[i] = s * (p.vSigmaSquared[i] - mean);
}

template <class T> inline M3<T> u_diag_vt(const M3<T>& U, const T d[3], const M3<T>& V) {
    M3<T> R;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++)
            R.a[i][j] = U.a[i][0] * d[0] * V.a[j][0] + U.a[i][1] * d[1] * V.a[j][1] + U.a[i][2] * d[2] * V.a[j][2];
    return R;
}

// Wolper_Drucker_Prager (mpm_kernels.cuh:494-544); p0 = apex shift
// (DP_threshold_p of the reference, per particle where cohesion is given).
template <class T> void wolper_drucker_prager(const SimParams3D& P, const Elastic<T>& E, PointState<T>& p, const T& p0) {
    const T mu = E.mu, kappa = E.kappa;
    const double tan_phi = P.DP_tan_phi;
    const double pmax = P.IceCompressiveStrength, qmax = P.IceShearStrength;
    if (p.p_tr < -p0 || p.Jp_inv < 1) {
        T p_new = -p0;
        T Je_new = sc::sqrt(-2. * p_new / kappa + 1.);
        T c = sc::cbrt(Je_new);
        T d[3] = {c, c, c};
        p.Fe = u_diag_vt(p.U, d, p.V);
        p.Jp_inv *= Je_new / p.Je_tr;
    } else {
        T q_n_1;
        if (p.p_tr > pmax) {
            q_n_1 = 0.0;
        } else {
            T q_from_dp = (p.p_tr + p0) * tan_phi;
            const double pmin = -P.IceTensileStrength;
            T q_from_failure_surface = 2 * sc::sqrt((pmax - p.p_tr) * (p.p_tr - pmin)) * qmax / (pmax - pmin);
            q_n_1 = sc::fmin(q_from_failure_surface, q_from_dp);
        }
        if (p.q_tr >= q_n_1) {
            T s_hat_n_1_norm = q_n_1 * kCoeff1Inv;
            T Je_tr_sq = p.Je_tr * p.Je_tr;
            T nrm = sc::sqrt(p.v_s_hat_tr[0] * p.v_s_hat_tr[0] + p.v_s_hat_tr[1] * p.v_s_hat_tr[1] +
                             p.v_s_hat_tr[2] * p.v_s_hat_tr[2]);
            T dir[3] = {0.0, 0.0, 0.0};
            if (nrm > 0) for (int i = 0; i < 3; i++) dir[i] = p.v_s_hat_tr[i] / nrm;   // Eigen normalized()
            T coef = s_hat_n_1_norm * sc::cbrt(Je_tr_sq) / mu;
            T tr3 = (p.vSigmaSquared[0] + p.vSigmaSquared[1] + p.vSigmaSquared[2]) / 3;
            T sig[3];
            for (int i = 0; i < 3; i++) sig[i] = sc::sqrt(coef * dir[i] + tr3);
            p.Fe = u_diag_vt(p.U, sig, p.V);
        }
    }
}

template <class T> inline void quad_weights(const T fx[3], T ww[3][3]) {
    // mpm_kernels.cuh:78-81 : ww[i][dim]
    for (int d = 0; d < 3; d++) {
        T v0 = 1.5 - fx[d], v1 = fx[d] - 1.0, v2 = fx[d] - 0.5;
        ww[0][d] = 0.5 * v0 * v0;
        ww[1][d] = 0.75 - v1 * v1;
        ww[2][d] = 0.5 * v2 * v2;
    }
}

// Bounds check of mpm_kernels.cuh:70-75 for one partition (gridX_offset 0,
// gridX = GridXTotal): the last failing test sets the code.
inline int stencil_error(const SimParams3D& P, const int b[3]) {
    int e = 0;
    const int halo = P.GridHaloSize;
    if (b[0] < -halo) e = 70;
    if (b[1] < 0) e = 71;
    if (b[2] < 0) e = 72;
    if (b[0] > P.GridXTotal + halo - 3) e = 73;
    if (b[1] > P.GridY - 3) e = 74;
    if (b[2] > P.GridZ - 3) e = 75;
    return e;
}

inline long long node_index(const SimParams3D& P, int x, int y, int z) {
    return ((long long)(x + P.GridHaloSize) * P.GridY + y) * P.GridZ + z;
}

template <class T> inline void load_point(const T* soa, unsigned pitch, unsigned i, PointState<T>& p) {
    p.utility = util_bits(sc::val(soa[(size_t)pitch * MPM_IDX_UTILITY + i]));
    for (int d = 0; d < 3; d++) {
        p.pos[d] = soa[(size_t)pitch * (MPM_POSX + d) + i];
        p.vel[d] = soa[(size_t)pitch * (MPM_VELX + d) + i];
        for (int e = 0; e < 3; e++) {
            p.Fe.a[d][e] = soa[(size_t)pitch * (MPM_FE00 + 3 * d + e) + i];
            p.Bp.a[d][e] = soa[(size_t)pitch * (MPM_BP00 + 3 * d + e) + i];
        }
    }
    p.Jp_inv = soa[(size_t)pitch * MPM_IDX_JP_INV + i];
    p.grain = (short)p.utility;
}

inline void grid_add(double* a, double v, bool atomic) {
    if (atomic) {
#pragma omp atomic
        *a += v;
    } else {
        *a += v;
    }
}
inline void grid_add(Dual* a, const Dual& v, bool) { *a += v; }

// The particle part of partition_kernel_p2g (mpm_kernels.cuh:24-99) writing
// into a grid window whose buffer slab 0 is grid column `xlo`.
template <class T>
int p2g_particle(const SimParams3D& P, const Elastic<T>& E, const T* soa, unsigned pitch, unsigned i,
                 T* win, long long win_nodes, int xlo, bool atomic) {
    long long util = util_bits(sc::val(soa[(size_t)pitch * MPM_IDX_UTILITY + i]));
    if (util & MPM_STATUS_DISABLED) return 0;
    const double h = P.cellsize, h_inv = P.cellsize_inv;
    const int isLiquid = (int)((util & MPM_STATUS_LIQUID) >> 18);
    const double particle_mass = isLiquid ? P.LiquidParticleMass : P.ParticleMass;

    PointState<T> p;
    load_point(soa, pitch, i, p);
    M3<T> PFt = isLiquid ? water(E, p.Jp_inv) : kirchhoff_wolper(E, p.Fe);
    M3<T> sub;
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) sub.a[a][b] = particle_mass * p.Bp.a[a][b] - P.dt_vol_Dpinv * PFt.a[a][b];

    int base[3];
    T fx[3];
    for (int d = 0; d < 3; d++) base[d] = (int)sc::val(p.pos[d] * h_inv - 0.5);
    for (int d = 0; d < 3; d++) fx[d] = p.pos[d] * h_inv - (double)base[d];
    int err = stencil_error(P, base);

    T ww[3][3];
    quad_weights(fx, ww);
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++)
            for (int c = 0; c < 3; c++) {
                int nx = base[0] + a, ny = base[1] + b, nz = base[2] + c;
                if (nx < -P.GridHaloSize || nx >= P.GridXTotal + P.GridHaloSize || ny < 0 || ny >= P.GridY ||
                    nz < 0 || nz >= P.GridZ)
                    continue;
                T Wip = ww[a][0] * ww[b][1] * ww[c][2];
                T dpos[3] = {(a - fx[0]) * h, (b - fx[1]) * h, (c - fx[2]) * h};
                T incV[3];
                for (int m = 0; m < 3; m++)
                    incV[m] = Wip * (p.vel[m] * particle_mass +
                                     (sub.a[m][0] * dpos[0] + sub.a[m][1] * dpos[1] + sub.a[m][2] * dpos[2]));
                T incM = Wip * particle_mass;
                long long idx = ((long long)(nx - xlo) * P.GridY + ny) * P.GridZ + nz;
                grid_add(&win[idx], incM, atomic);
                for (int m = 0; m < 3; m++) grid_add(&win[(m + 1) * win_nodes + idx], incV[m], atomic);
            }
    return err;
}

// One node of partition_kernel_update_nodes (mpm_kernels.cuh:138-232), one
// partition. sensor (double, may be NULL) and fsum accumulate the indenter force.
template <class T>
void update_node(const SimParams3D& P, T* grid, long long nodes, long long idx, double ind_x, double ind_y,
                 double* sensor, T fsum[3]) {
    const int halo = P.GridHaloSize, gridY = P.GridY, gridZ = P.GridZ, gridXTotal = P.GridXTotal;
    const double indRsq = P.IndRSq, dt = P.InitialTimeStep, cellsize = P.cellsize;
    const double vmax = P.vmax, vmax_squared = P.vmax_squared;
    const double vco[3] = {P.IndVelocity, 0, 0};
    T mass = grid[idx];
    if (mass == 0) return;
    T v[3];
    for (int i = 0; i < 3; i++) v[i] = grid[(i + 1) * nodes + idx];
    int idx_z = (int)(idx % gridZ);
    int idx_y = (int)((idx / gridZ) % gridY);
    int idx_x = (int)(idx / ((long long)gridZ * gridY));
    int gi[3] = {idx_x - halo, idx_y, idx_z};
    double gnpos[3] = {gi[0] * cellsize, gi[1] * cellsize, gi[2] * cellsize};

    for (int i = 0; i < 3; i++) v[i] /= mass;
    v[1] -= P.dt_Gravity;
    T vsq = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
    if (vsq > vmax_squared) {
        T nv = sc::sqrt(vsq);
        for (int i = 0; i < 3; i++) v[i] = v[i] / nv * vmax;
    }

    if (P.SetupType != 2) {
        double n[2] = {gnpos[0] - ind_x, gnpos[1] - ind_y};
        double nsq = n[0] * n[0] + n[1] * n[1];
        if (nsq < indRsq) {
            T vrel[3] = {v[0] - vco[0], v[1] - vco[1], v[2] - vco[2]};
            double nn = std::sqrt(nsq);
            if (nsq > 0) { n[0] /= nn; n[1] /= nn; }
            T vn = vrel[0] * n[0] + vrel[1] * n[1] + vrel[2] * 0.0;
            if (vn < 0) {
                T vt[3] = {vrel[0] - n[0] * vn, vrel[1] - n[1] * vn, vrel[2] - 0.0 * vn};
                T prev[3] = {v[0], v[1], v[2]};
                for (int i = 0; i < 3; i++) v[i] = vco[i] + vt[i];
                T force[3];
                for (int i = 0; i < 3; i++) force[i] = (prev[i] - v[i]) * mass / dt;
                float angle = std::atan2((float)n[0], (float)n[1]);
                angle += MPM_PI;
                angle *= P.IndenterSubdivisions / (2 * MPM_PI);
                int index_angle = std::min(std::max((int)angle, 0), P.IndenterSubdivisions - 1);
                int index_z = std::min(std::max(idx_z, 0), gridZ - 1);
                int index = index_z + index_angle * gridZ;
                for (int i = 0; i < 3; i++) {
                    if (sensor) sensor[i + 3 * index] += sc::val(force[i]);
                    fsum[i] += force[i];
                }
            }
        }
    }

    if (P.SetupType != 2) {
        if (gi[1] <= 2) v[0] = v[1] = v[2] = 0.0;
    } else {
        if (gi[1] <= 2 && v[1] < 0) v[1] = 0.0;
    }
    if (gi[1] >= gridY - 3 && v[1] > 0) v[1] = 0.0;
    if (gi[0] <= 2 && v[0] < 0) v[0] = 0.0;
    else if (gi[0] >= gridXTotal - 3 && v[0] > 0) v[0] = 0.0;
    if (gi[2] <= 2 && v[2] < 0) v[2] = 0.0;
    else if (gi[2] >= gridZ - 3 && v[2] > 0) v[2] = 0.0;

    if (P.SetupType == 2 && P.DragGlobal != 0)
        for (int i = 0; i < 3; i++) v[i] *= (1 - P.DragGlobal);

    for (int i = 0; i < 3; i++) grid[(i + 1) * nodes + idx] = v[i];
}

// One particle of partition_kernel_g2p (mpm_kernels.cuh:237-351), no migration.
template <class T>
int g2p_particle(const SimParams3D& P, const Elastic<T>& E, T* soa, unsigned pitch, unsigned i, const T* grid,
                 long long nodes, int record_pq, const T& p0, int svd_mode) {
    const double h_inv = P.cellsize_inv, dt = P.InitialTimeStep;
    PointState<T> p;
    p.utility = util_bits(sc::val(soa[(size_t)pitch * MPM_IDX_UTILITY + i]));
    if (p.utility & MPM_STATUS_DISABLED) return 0;
    p.p_tr = p.q_tr = p.Je_tr = 0.0;
    bool isLiquid = (p.utility & MPM_STATUS_LIQUID) != 0;
    load_point(soa, pitch, i, p);

    int base[3];
    T fx[3];
    for (int d = 0; d < 3; d++) base[d] = (int)sc::val(p.pos[d] * h_inv - 0.5);
    for (int d = 0; d < 3; d++) fx[d] = p.pos[d] * h_inv - (double)base[d];
    int err = stencil_error(P, base);
    T ww[3][3];
    quad_weights(fx, ww);

    T vel[3] = {0.0, 0.0, 0.0};
    M3<T> Bp = zero3<T>();
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++)
            for (int c = 0; c < 3; c++) {
                int nx = base[0] + a, ny = base[1] + b, nz = base[2] + c;
                if (nx < -P.GridHaloSize || nx >= P.GridXTotal + P.GridHaloSize || ny < 0 || ny >= P.GridY ||
                    nz < 0 || nz >= P.GridZ)
                    continue;
                T dpos[3] = {a - fx[0], b - fx[1], c - fx[2]};
                T weight = ww[a][0] * ww[b][1] * ww[c][2];
                long long idx = node_index(P, nx, ny, nz);
                T nv[3];
                for (int m = 0; m < 3; m++) nv[m] = grid[(1 + m) * nodes + idx];
                for (int m = 0; m < 3; m++) vel[m] += weight * nv[m];
                T s = (4. * h_inv) * weight;
                for (int r = 0; r < 3; r++)
                    for (int q = 0; q < 3; q++) Bp.a[r][q] += s * (nv[r] * dpos[q]);
            }
    for (int m = 0; m < 3; m++) p.vel[m] = vel[m];
    p.Bp = Bp;

    for (int d = 0; d < 3; d++) p.pos[d] += p.vel[d] * dt;
    M3<T> A = eye3<T>();
    for (int r = 0; r < 3; r++)
        for (int q = 0; q < 3; q++) A.a[r][q] += dt * p.Bp.a[r][q];
    p.Fe = mul(A, p.Fe);

    if (isLiquid) {
        p.Jp_inv *= det3(A);
    } else {
        compute_pq(E, p);
        if (!(p.utility & MPM_STATUS_CRUSHED)) check_failure_surface(P, p);
        if (p.utility & MPM_STATUS_CRUSHED) {
            compute_svd(E, p, svd_mode);
            wolper_drucker_prager(P, E, p, p0);
        }
    }

    for (int d = 0; d < 3; d++) {
        soa[(size_t)pitch * (MPM_POSX + d) + i] = p.pos[d];
        soa[(size_t)pitch * (MPM_VELX + d) + i] = p.vel[d];
        for (int q = 0; q < 3; q++) {
            soa[(size_t)pitch * (MPM_FE00 + 3 * d + q) + i] = p.Fe.a[d][q];
            soa[(size_t)pitch * (MPM_BP00 + 3 * d + q) + i] = p.Bp.a[d][q];
        }
    }
    soa[(size_t)pitch * MPM_IDX_JP_INV + i] = p.Jp_inv;
    soa[(size_t)pitch * MPM_IDX_UTILITY + i] = util_double(p.utility);
    if (record_pq) {
        soa[(size_t)pitch * MPM_IDX_P + i] = p.p_tr;
        soa[(size_t)pitch * MPM_IDX_Q + i] = p.q_tr;
    }
    return err;
}

inline Elastic<double> elastic_of(const SimParams3D& P) { return Elastic<double>{P.mu, P.kappa}; }

}  // namespace

extern "C" {

long long or_grid_nodes(const SimParams3D* P) {
    return (long long)(P->GridXTotal + 2 * P->GridHaloSize) * P->GridY * P->GridZ;
}

int or_cell_key(const SimParams3D* P, double x, double y, double z) {
    const double hinv = P->cellsize_inv;
    int ix = (int)(x * hinv + 0.5), iy = (int)(y * hinv + 0.5), iz = (int)(z * hinv + 0.5);
    return ix * P->GridY * P->GridZ + iy * P->GridZ + iz;
}

unsigned or_sort_permutation(const SimParams3D* P, const double* soa, unsigned pitch, unsigned n,
                             unsigned* perm) {
    std::vector<std::pair<int, unsigned>> keyed;
    keyed.reserve(n);
    for (unsigned i = 0; i < n; i++) {
        long long util = util_bits(soa[(size_t)pitch * MPM_IDX_UTILITY + i]);
        if ((util & MPM_STATUS_DISABLED) == MPM_STATUS_DISABLED) continue;
        int key = or_cell_key(P, soa[(size_t)pitch * MPM_POSX + i], soa[(size_t)pitch * (MPM_POSX + 1) + i],
                              soa[(size_t)pitch * (MPM_POSX + 2) + i]);
        keyed.push_back({key, i});
    }
    std::stable_sort(keyed.begin(), keyed.end(),
                     [](const std::pair<int, unsigned>& a, const std::pair<int, unsigned>& b) {
                         return a.first < b.first;
                     });
    for (size_t k = 0; k < keyed.size(); k++) perm[k] = keyed[k].second;
    return (unsigned)keyed.size();
}

int or_p2g(const SimParams3D* P, const double* soa, unsigned pitch, unsigned n, double* grid, int nthreads) {
    const long long nodes = or_grid_nodes(P);
    const int xlo = -P->GridHaloSize;
    const Elastic<double> E = elastic_of(*P);
    int err = 0;
    if (nthreads <= 1) {
        for (unsigned i = 0; i < n; i++) {
            int e = p2g_particle(*P, E, soa, pitch, i, grid, nodes, xlo, false);
            if (e) err = e;
        }
        return err;
    }
#ifdef _OPENMP
    // Contiguous particle chunks (cell-sorted input keeps their x-range small)
    // accumulate into private slab windows, then windows are summed in
    // chunk order, node by node.
    const long long slab = (long long)P->GridY * P->GridZ;
    std::vector<int> wlo(nthreads), whi(nthreads);
    std::vector<std::vector<double>> win(nthreads);
    std::vector<int> errs(nthreads, 0);
    long long total_win = 0;
    for (int t = 0; t < nthreads; t++) {
        unsigned a = (unsigned)((unsigned long long)n * t / nthreads), b = (unsigned)((unsigned long long)n * (t + 1) / nthreads);
        int lo = P->GridXTotal + P->GridHaloSize, hi = -P->GridHaloSize - 1;
        for (unsigned i = a; i < b; i++) {
            int bx = (int)(soa[(size_t)pitch * MPM_POSX + i] * P->cellsize_inv - 0.5);
            lo = std::min(lo, bx);
            hi = std::max(hi, bx + 2);
        }
        lo = std::max(lo, -P->GridHaloSize);
        hi = std::min(hi, P->GridXTotal + P->GridHaloSize - 1);
        if (hi < lo) hi = lo - 1;
        wlo[t] = lo; whi[t] = hi;
        total_win += (long long)(hi - lo + 1) * slab;
    }
    const bool use_windows = total_win <= 3 * nodes;
    if (!use_windows) {
#pragma omp parallel for num_threads(nthreads) schedule(static)
        for (long long i = 0; i < (long long)n; i++) {
            int e = p2g_particle(*P, E, soa, pitch, (unsigned)i, grid, nodes, xlo, true);
            if (e) errs[omp_get_thread_num()] = e;
        }
    } else {
#pragma omp parallel num_threads(nthreads)
        {
            int t = omp_get_thread_num();
            long long wn = (long long)(whi[t] - wlo[t] + 1) * slab;
            win[t].assign((size_t)(4 * std::max(wn, 1LL)), 0.0);
            unsigned a = (unsigned)((unsigned long long)n * t / nthreads), b = (unsigned)((unsigned long long)n * (t + 1) / nthreads);
            for (unsigned i = a; i < b; i++) {
                int e = p2g_particle(*P, E, soa, pitch, i, win[t].data(), wn, wlo[t], false);
                if (e) errs[t] = e;
            }
#pragma omp barrier
#pragma omp for schedule(static)
            for (long long node = 0; node < nodes; node++) {
                int gx = (int)(node / slab) - P->GridHaloSize;
                long long rem = node % slab;
                for (int u = 0; u < nthreads; u++) {
                    if (gx < wlo[u] || gx > whi[u]) continue;
                    long long wnu = (long long)(whi[u] - wlo[u] + 1) * slab;
                    long long li = (long long)(gx - wlo[u]) * slab + rem;
                    for (int m = 0; m < 4; m++) grid[m * nodes + node] += win[u][m * wnu + li];
                }
            }
        }
    }
    for (int t = 0; t < nthreads; t++) if (errs[t]) err = errs[t];
    return err;
#else
    return or_p2g(P, soa, pitch, n, grid, 1);
#endif
}

// partition_kernel_update_nodes (mpm_kernels.cuh:138-232), one partition.
void or_update_nodes(const SimParams3D* P, double* grid, double ind_x, double ind_y, double* sensor,
                     double force3[3], int nthreads) {
    const long long nodes = or_grid_nodes(P);
    double fsum[3] = {0, 0, 0};
    (void)nthreads;
    // Sensor accumulation is serial (node order) so the oracle is deterministic.
    for (long long idx = 0; idx < nodes; idx++) update_node(*P, grid, nodes, idx, ind_x, ind_y, sensor, fsum);
    if (force3) for (int i = 0; i < 3; i++) force3[i] = fsum[i];
}

// partition_kernel_g2p (mpm_kernels.cuh:237-351), no migration.
int or_g2p(const SimParams3D* P, double* soa, unsigned pitch, unsigned n, const double* grid, int record_pq,
           const double* p0, int svd_mode, int nthreads) {
    const long long nodes = or_grid_nodes(P);
    const Elastic<double> E = elastic_of(*P);
    int err = 0;
#pragma omp parallel for num_threads(nthreads > 1 ? nthreads : 1) schedule(static) reduction(max : err)
    for (long long ii = 0; ii < (long long)n; ii++) {
        unsigned i = (unsigned)ii;
        int e = g2p_particle(*P, E, soa, pitch, i, grid, nodes, record_pq, p0 ? p0[i] : P->DP_threshold_p, svd_mode);
        if (e > err) err = e;
    }
    return err;
}

int or_step(SimParams3D* P, double* soa, unsigned pitch, unsigned n, double* grid, double* sensor,
            double force3[3], const double* p0, int svd_mode, int nthreads) {
    P->SimulationTime += P->InitialTimeStep;
    P->indenter_x = P->indenter_x_initial + P->SimulationTime * P->IndVelocity;
    const long long nodes = or_grid_nodes(P);
    std::memset(grid, 0, sizeof(double) * 4 * (size_t)nodes);
    int e1 = or_p2g(P, soa, pitch, n, grid, nthreads);
    or_update_nodes(P, grid, P->indenter_x, P->indenter_y, sensor, force3, nthreads);
    const int isZeroStep = (P->SimulationStep % P->UpdateEveryNthStep) == 0;
    int e2 = or_g2p(P, soa, pitch, n, grid, isZeroStep, p0, svd_mode, nthreads);
    P->SimulationStep += 1;
    return e1 ? e1 : e2;
}

int or_dual_steps(SimParams3D* P, double* soa, double* dsoa, unsigned pitch, unsigned n, const double* p0,
                  const double* dp0, double dE, int nsteps, double* force_hist, double* dforce_hist) {
    // d mu / dE and d kappa / dE of mpm_params_compute_lame (parameters_sim_3d.cpp:65-70):
    // mu = E / (2 (1 + nu)), lambda = E nu / ((1 + nu)(1 - 2 nu)), kappa = 2/3 mu + lambda
    const double nu = P->PoissonsRatio;
    const double dmu = dE / (2 * (1 + nu));
    const double dkappa = dmu * 2. / 3. + dE * nu / ((1 + nu) * (1 - 2 * nu));
    const Elastic<Dual> E{Dual(P->mu, dmu), Dual(P->kappa, dkappa)};
    const long long nodes = or_grid_nodes(P);
    std::vector<Dual> s((size_t)MPM_N_PTS_ARRAYS * pitch), g((size_t)4 * nodes), c(n);
    for (size_t k = 0; k < s.size(); k++) s[k] = Dual(soa[k], dsoa[k]);
    for (unsigned i = 0; i < n; i++) c[i] = Dual(p0 ? p0[i] : P->DP_threshold_p, dp0 ? dp0[i] : 0.0);
    int err = 0;
    for (int step = 0; step < nsteps && !err; step++) {
        P->SimulationTime += P->InitialTimeStep;
        P->indenter_x = P->indenter_x_initial + P->SimulationTime * P->IndVelocity;
        std::fill(g.begin(), g.end(), Dual(0.0));
        for (unsigned i = 0; i < n; i++) {
            int e = p2g_particle(*P, E, s.data(), pitch, i, g.data(), nodes, -P->GridHaloSize, false);
            if (e) err = e;
        }
        Dual fsum[3] = {0.0, 0.0, 0.0};
        for (long long idx = 0; idx < nodes; idx++)
            update_node(*P, g.data(), nodes, idx, P->indenter_x, P->indenter_y, nullptr, fsum);
        for (int k = 0; k < 3; k++) {
            force_hist[3 * step + k] = fsum[k].v;
            dforce_hist[3 * step + k] = fsum[k].d;
        }
        const int isZeroStep = (P->SimulationStep % P->UpdateEveryNthStep) == 0;
        for (unsigned i = 0; i < n; i++) {
            int e = g2p_particle(*P, E, s.data(), pitch, i, g.data(), nodes, isZeroStep, c[i], 1);
            if (e > err) err = e;
        }
        P->SimulationStep += 1;
    }
    for (size_t k = 0; k < s.size(); k++) { soa[k] = s[k].v; dsoa[k] = s[k].d; }
    return err;
}

}  // extern "C"
