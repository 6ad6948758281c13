// FP64 per-particle and per-node physics of the step: Kirchhoff stress,
// trial p/q, failure surface, Drucker-Prager return map. Each function names
// the reference lines (simulation/mpm_kernels.cuh) whose mathematics it
// carries out.
#pragma once

#include "device_common.cuh"
#include "svd3.cuh"

namespace icempm {

__device__ __forceinline__ double det3(const double a[3][3]) {
    return a[0][0] * (a[1][1] * a[2][2] - a[2][1] * a[1][2])
         - a[1][0] * (a[0][1] * a[2][2] - a[2][1] * a[0][2])
         + a[2][0] * (a[0][1] * a[1][2] - a[1][1] * a[0][2]);
}

// b = F F^T
__device__ __forceinline__ void ffT(const double F[3][3], double b[3][3]) {
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) b[i][j] = F[i][0] * F[j][0] + F[i][1] * F[j][1] + F[i][2] * F[j][2];
}

// KirchhoffStress_Wolper (mpm_kernels.cuh:547-557):
// tau = mu J^(-2/3) dev(F F^T) + kappa/2 (J^2 - 1) I
__device__ __forceinline__ void kirchhoff_wolper(const DevParams& P, const double F[3][3], double tau[3][3]) {
    double Je = det3(F);
    double b[3][3];
    ffT(F, b);
    double tr3 = (b[0][0] + b[1][1] + b[2][2]) / 3;
    double s = P.mu * rcbrt(Je * Je);
    double hyd = P.kappa * 0.5 * (Je * Je - 1.);
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) tau[i][j] = s * (b[i][j] - (i == j ? tr3 : 0.0)) + (i == j ? hyd : 0.0);
}

// Water (mpm_kernels.cuh:559-566): kappa (1 - J^-3), times I
__device__ __forceinline__ double water_pressure(const DevParams& P, double J) {
    return P.kappa * (1. - pow(J, -3.0));
}

// ComputePQ (mpm_kernels.cuh:477-484); PP: DevParams or DPParams
template <class PP>
__device__ __forceinline__ void trial_pq(const PP& P, const double F[3][3], double& Je, double& p_tr,
                                         double& q_tr) {
    Je = det3(F);
    double Jsq = Je * Je;
    p_tr = -(0.5 * P.kappa) * (Jsq - 1.);
    double b[3][3];
    ffT(F, b);
    double tr3 = (b[0][0] + b[1][1] + b[2][2]) / 3;
    double sq = 0;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            double d = b[i][j] - (i == j ? tr3 : 0.0);
            sq += d * d;
        }
    q_tr = kCoeff1 * P.mu * rcbrt(Jsq) * sqrt(sq);
}

// GetParametersForGrain + CheckIfPointIsInsideFailureSurface
// (mpm_kernels.cuh:434-474). True if the point crushes now.
__device__ __forceinline__ bool outside_failure_surface(const DevParams& P, short grain, double p_tr, double q_tr) {
    const double var2 = 1.0 + P.grain_var * 0.033 * (-15 + (grain + 3) % 30);
    const double var3 = 1.0 + P.grain_var * 0.1 * (-10 + (grain + 4) % 11);
    const double pmax = P.pmax;
    const double pmin = -P.tensile;
    const double qmax = P.shear * var3;
    const double pmin2 = -P.tensile2 * var2;
    const double beta = P.beta;
    if (p_tr < 0) {
        if (p_tr < pmin2) return true;
        double q0 = 2 * sqrt(-pmax * pmin) * qmax / (pmax - pmin);
        double k = -q0 / pmin2;
        return q_tr > k * (p_tr - pmin2);
    }
    const double mSq = (4 * qmax * qmax * (1 + 2 * beta)) / ((pmax - pmin) * (pmax - pmin));
    double y = (1. + 2. * beta) * q_tr * q_tr + mSq * (p_tr + beta * pmax) * (p_tr - pmax);
    return y > 0;
}

// F = U diag(d) V^T
__device__ __forceinline__ void compose_usv(const double U[3][3], const double d[3], const double V[3][3],
                                            double F[3][3]) {
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++)
            F[i][j] = U[i][0] * d[0] * V[j][0] + U[i][1] * d[1] * V[j][1] + U[i][2] * d[2] * V[j][2];
}

// ComputeSVD (mpm_kernels.cuh:486-492) + Wolper_Drucker_Prager (:494-544)
// for a crushed point. p0 is the apex shift (DP_threshold_p, or the
// per-particle cohesion / tan(phi)). K selects the SVD arithmetic.
// The material constants the return map reads (a small by-value copy for
// out-of-line callers).
struct DPParams {
    double mu, kappa, pmax, tensile, shear, tan_phi;
};

__device__ __forceinline__ DPParams dp_params(const DevParams& P) {
    DPParams d;
    d.mu = P.mu; d.kappa = P.kappa; d.pmax = P.pmax; d.tensile = P.tensile; d.shear = P.shear; d.tan_phi = P.tan_phi;
    return d;
}

template <class K, class PP>
__device__ __forceinline__ void drucker_prager_return(const PP& P, double F[3][3], double& Jp_inv,
                                                      double Je_tr, double p_tr, double q_tr, double p0) {
    typedef typename K::T T;
    T A[3][3], Uk[3][3], Sk[3], Vk[3][3];
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) A[i][j] = (T)F[i][j];
    svd3x3<K>(A, Uk, Sk, Vk);
    double U[3][3], V[3][3], sig2[3];
#pragma unroll
    for (int i = 0; i < 3; i++) {
        double s = (double)Sk[i];
        sig2[i] = s * s;
#pragma unroll
        for (int j = 0; j < 3; j++) { U[i][j] = (double)Uk[i][j]; V[i][j] = (double)Vk[i][j]; }
    }
    const double mu = P.mu, kappa = P.kappa;
    if (p_tr < -p0 || Jp_inv < 1) {
        // tension cut-off / recompaction: project to the apex
        double p_new = -p0;
        double Je_new = sqrt(-2. * p_new / kappa + 1.);
        double c = cbrt(Je_new);
        double d[3] = {c, c, c};
        compose_usv(U, d, V, F);
        Jp_inv *= Je_new / Je_tr;
        return;
    }
    double q_n_1;
    if (p_tr > P.pmax) {
        q_n_1 = 0;
    } else {
        double q_from_dp = (p_tr + p0) * P.tan_phi;
        const double pmin = -P.tensile;
        double q_from_failure_surface = 2 * sqrt((P.pmax - p_tr) * (p_tr - pmin)) * P.shear / (P.pmax - pmin);
        q_n_1 = fmin(q_from_failure_surface, q_from_dp);
    }
    if (q_tr >= q_n_1) {
        const double Je_tr_sq = Je_tr * Je_tr;
        const double mean = (sig2[0] + sig2[1] + sig2[2]) / 3;
        const double sfac = mu * rcbrt(Je_tr_sq);
        double sh[3];
#pragma unroll
        for (int i = 0; i < 3; i++) sh[i] = sfac * (sig2[i] - mean);      // v_s_hat_tr
        double nrm = sqrt(sh[0] * sh[0] + sh[1] * sh[1] + sh[2] * sh[2]);
        const double coef = (q_n_1 * kCoeff1Inv) * cbrt(Je_tr_sq) / mu;
        double sig[3];
#pragma unroll
        for (int i = 0; i < 3; i++) sig[i] = sqrt(coef * (nrm > 0 ? sh[i] / nrm : 0.0) + mean);
        compose_usv(U, sig, V, F);
    }
}

}  // namespace icempm
