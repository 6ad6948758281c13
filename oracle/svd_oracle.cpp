// CPU ORACLE — test infrastructure, not product code.
//
// Restatement of the 3x3 SVD the reference performs (simulation/helper_math.cuh:24-1120,
// called through svd3x3, mpm_kernels.cuh:585-601). The algorithm is the one
// published by McAdams, Selle, Tamstorf, Teran and Sifakis, "Computing the
// Singular Value Decomposition of 3x3 matrices with minimal branching and
// elementary floating point operations" (UW-Madison CS TR1690, 2011):
//   1. B = A^T A (symmetric);
//   2. 4 cyclic Jacobi sweeps over the pairs (1,2), (2,3), (3,1) with the
//      "approximate Givens" quaternion (sh, ch) = (a_pq/2, a_pp - a_qq),
//      replaced by the pi/8 rotation when ch^2 <= (3+2*sqrt 2) sh^2,
//      accumulating V as a quaternion;
//   3. quaternion normalised with one Newton step on rsqrt, turned into V;
//   4. A V, columns sorted by decreasing norm (swaps negate a column so V
//      stays a rotation);
//   5. QR of A V by three Givens rotations -> U and the diagonal S.
// The float variant carries out every step with the same sequence of IEEE
// float operations as the reference (each add/sub separately rounded, no
// fused multiply-add: this file is compiled with -ffp-contract=off), so its
// output is bit-identical to the reference's. Compile-time type T selects the
// float variant (reference semantics) or a double variant (more sweeps).

#include <cmath>
#include <cstdint>
#include <cstring>
#include "dual.h"
#include "mpm_oracle.h"

namespace {

// Correctly rounded 1/sqrt(x) in float: the reciprocal square root is taken
// in 64-bit extended precision and rounded once to float.
inline float rsqrt_rn(float x) { return (float)(1.0L / sqrtl((long double)x)); }
inline double rsqrt_rn(double x) { return 1.0 / std::sqrt(x); }
inline Dual rsqrt_rn(const Dual& x) {
    double r = 1.0 / std::sqrt(x.v);
    return Dual(r, -0.5 * r * r * r * x.d);
}

template <typename T> struct SvdConst;
template <> struct SvdConst<float> {
    static float tiny() { return 1.e-20f; }
    static float small() { return 1.e-12f; }
    // 3 + 2 sqrt(2), sin(pi/8) and cos(pi/8) as the float values the
    // reference uses (helper_math.cuh:10-16); its cos(pi/8) is one ulp above
    // the correctly rounded value, and bit-exact parity needs that value.
    static float four_gamma_sq() { return 0x1.7504f4p+2f; }
    static float sin_pi8() { return 0x1.87de2ap-2f; }
    static float cos_pi8() { return 0x1.d906bep-1f; }
};
template <> struct SvdConst<double> {
    static double tiny() { return 1.e-40; }
    static double small() { return 1.e-40; }
    static double four_gamma_sq() { return 3.0 + 2.0 * std::sqrt(2.0); }
    static double sin_pi8() { return std::sin(MPM_PI / 8.0); }
    static double cos_pi8() { return std::cos(MPM_PI / 8.0); }
};
// Forward-mode derivative of the double variant: the constants carry no tangent.
template <> struct SvdConst<Dual> {
    static Dual tiny() { return SvdConst<double>::tiny(); }
    static Dual small() { return SvdConst<double>::small(); }
    static Dual four_gamma_sq() { return SvdConst<double>::four_gamma_sq(); }
    static Dual sin_pi8() { return SvdConst<double>::sin_pi8(); }
    static Dual cos_pi8() { return SvdConst<double>::cos_pi8(); }
};

// Symmetric 3x3 stored as s[i][j] (both halves kept in sync by writing the
// lower-triangle entry through a reference).
template <typename T>
struct Quat { T s, x, y, z; };

// One approximate-Givens Jacobi conjugation on the pair (p, q); r is the
// third index. a_pp, a_qq, a_pq, a_rp, a_rq, a_rr are references into the
// symmetric matrix; q_p, q_q, q_r the quaternion vector components along
// the axes p, q, r.
template <typename T>
void jacobi_conjugate(T& a_pp, T& a_qq, T& a_pq, T& a_rp, T& a_rq, T& a_rr,
                      T& qs, T& q_p, T& q_q, T& q_r) {
    typedef SvdConst<T> K;
    T sh = a_pq * (T)0.5;
    T d = a_pp - a_qq;
    T ch;
    if (sh * sh >= K::tiny()) { ch = d; } else { sh = (T)0; ch = (T)1; }

    T sh2 = sh * sh;
    T ch2 = ch * ch;
    T w = rsqrt_rn(sh2 + ch2);
    sh = w * sh;
    ch = w * ch;
    if (ch2 <= K::four_gamma_sq() * sh2) { sh = K::sin_pi8(); ch = K::cos_pi8(); }

    sh2 = sh * sh;
    ch2 = ch * ch;
    T c = ch2 - sh2;
    T s = ch * sh;
    s = s + s;

    // The quaternion (ch, sh) need not be unit length here; the rotation is
    // scaled by |q|^2 = sh2 + ch2, applied to the entries coupling r.
    T scale = sh2 + ch2;
    a_rr = a_rr * scale;
    a_rp = a_rp * scale;
    a_rq = a_rq * scale;
    a_rr = a_rr * scale;

    T t1 = s * a_rp;
    T t2 = s * a_rq;
    a_rp = c * a_rp;
    a_rq = c * a_rq;
    a_rp = t2 + a_rp;
    a_rq = a_rq - t1;

    T ss = s * s;
    T qq_s = a_qq * ss;
    T pp_s = a_pp * ss;
    T cc = c * c;
    a_pp = a_pp * cc;
    a_qq = a_qq * cc;
    a_pp = a_pp + qq_s;
    a_qq = a_qq + pp_s;
    T c2s2 = cc - ss;
    T pq2 = a_pq + a_pq;
    a_pq = a_pq * c2s2;
    T cs = c * s;
    pq2 = pq2 * cs;
    d = d * cs;
    a_pp = a_pp + pq2;
    a_pq = a_pq - d;
    a_qq = a_qq - pq2;

    // cumulative rotation: q <- q * (ch + sh e_r)
    T u_p = sh * q_p;
    T u_q = sh * q_q;
    T u_r = sh * q_r;
    T u_s = sh * qs;
    qs = ch * qs;
    q_p = ch * q_p;
    q_q = ch * q_q;
    q_r = ch * q_r;
    q_r = q_r + u_s;
    qs = qs - u_r;
    q_p = q_p + u_q;
    q_q = q_q - u_p;
}

// Newton-refined reciprocal square root: r <- r + r/2 - n*r^3/2.
template <typename T>
T refined_rsqrt(T n) {
    T r = rsqrt_rn(n);
    T h = r * (T)0.5;
    T t = r * h;
    t = r * t;
    t = n * t;
    r = r + h;
    r = r - t;
    return r;
}

// Givens rotation of rows (i, j) of B (3x3) zeroing B[j][i_col], accumulated
// into the columns (i, j) of U.
template <typename T>
void qr_givens(T B[3][3], T U[3][3], int i, int j, int col) {
    typedef SvdConst<T> K;
    T a = B[i][col];            // pivot entry (row i)
    T b = B[j][col];                                            // entry to annihilate
    T sh = (b * b >= K::small()) ? b : (T)0;
    T ch = sc::fmax((T)0 - a, a);
    ch = sc::fmax(ch, K::small());
    bool pos = a >= (T)0;

    T t2 = ch * ch;
    T t1 = sh * sh;
    t2 = t2 + t1;
    T r = refined_rsqrt(t2);
    r = r * t2;                 // ~ sqrt(ch^2 + sh^2)
    ch = ch + r;
    if (!pos) { T tmp = ch; ch = sh; sh = tmp; }

    t2 = ch * ch;
    t1 = sh * sh;
    t2 = t2 + t1;
    r = refined_rsqrt(t2);
    ch = ch * r;
    sh = sh * r;

    T c = ch * ch;
    T s = sh * sh;
    c = c - s;
    s = sh * ch;
    s = s + s;

    for (int k = 0; k < 3; k++) {
        T u = s * B[i][k];
        T v = s * B[j][k];
        B[i][k] = c * B[i][k];
        B[j][k] = c * B[j][k];
        B[i][k] = B[i][k] + v;
        B[j][k] = B[j][k] - u;
    }
    for (int k = 0; k < 3; k++) {
        T u = s * U[k][i];
        T v = s * U[k][j];
        U[k][i] = c * U[k][i];
        U[k][j] = c * U[k][j];
        U[k][i] = U[k][i] + v;
        U[k][j] = U[k][j] - u;
    }
}

template <typename T>
void swap_columns_if(T B[3][3], T V[3][3], T rho[3], int a, int b, int negate) {
    if (rho[a] < rho[b]) {
        for (int k = 0; k < 3; k++) {
            T t = B[k][a]; B[k][a] = B[k][b]; B[k][b] = t;
            t = V[k][a]; V[k][a] = V[k][b]; V[k][b] = t;
        }
        T t = rho[a]; rho[a] = rho[b]; rho[b] = t;
        for (int k = 0; k < 3; k++) { B[k][negate] = -B[k][negate]; V[k][negate] = -V[k][negate]; }
    }
}

template <typename T>
void svd_mcadams(const T A[3][3], T U[3][3], T S[3], T V[3][3], int sweeps) {
    // 1. normal equations: s_ij = sum_k a_ki a_kj, summed k = 0, 1, 2 as
    //    (a0i a0j + a1i a1j) + a2i a2j
    T s[3][3];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j <= i; j++) {
            T acc = A[0][j] * A[0][i];
            T t = A[1][j] * A[1][i];
            acc = t + acc;
            t = A[2][j] * A[2][i];
            acc = t + acc;
            s[i][j] = acc;
        }

    // 2. Jacobi sweeps; lower-triangle entries hold the symmetric matrix
    Quat<T> q = {(T)1, (T)0, (T)0, (T)0};
    for (int it = 0; it < sweeps; it++) {
        // pair (1,2), r = 3 (axis z)
        jacobi_conjugate<T>(s[0][0], s[1][1], s[1][0], s[2][0], s[2][1], s[2][2], q.s, q.x, q.y, q.z);
        // pair (2,3), r = 1 (axis x)
        jacobi_conjugate<T>(s[1][1], s[2][2], s[2][1], s[1][0], s[2][0], s[0][0], q.s, q.y, q.z, q.x);
        // pair (3,1), r = 2 (axis y)
        jacobi_conjugate<T>(s[2][2], s[0][0], s[2][0], s[2][1], s[1][0], s[1][1], q.s, q.z, q.x, q.y);
    }

    // 3. normalise, quaternion -> V
    T n = q.s * q.s;
    T t = q.x * q.x;
    n = t + n;
    t = q.y * q.y;
    n = t + n;
    t = q.z * q.z;
    n = t + n;
    T r = refined_rsqrt(n);
    q.s = q.s * r; q.x = q.x * r; q.y = q.y * r; q.z = q.z * r;

    T xx = q.x * q.x, yy = q.y * q.y, zz = q.z * q.z;
    T ss = q.s * q.s;
    T d2 = ss - xx;           // s^2 - x^2
    T v33 = d2 - yy;
    v33 = v33 + zz;
    T v22 = d2 + yy;
    v22 = v22 - zz;
    T v11 = ss + xx;
    v11 = v11 - yy;
    v11 = v11 - zz;
    T x2 = q.x + q.x, y2 = q.y + q.y, z2 = q.z + q.z;
    T sx = q.s * x2, sy = q.s * y2, sz = q.s * z2;
    T xy = q.y * x2, yz = q.z * y2, zx = q.x * z2;
    V[0][0] = v11; V[1][1] = v22; V[2][2] = v33;
    V[0][1] = xy - sz; V[1][0] = xy + sz;
    V[1][2] = yz - sx; V[2][1] = yz + sx;
    V[2][0] = zx - sy; V[0][2] = zx + sy;

    // 4. B = A V, row by row: B_rc = (a_r0 v_0c + a_r1 v_1c) + a_r2 v_2c
    T B[3][3];
    for (int row = 0; row < 3; row++)
        for (int col = 0; col < 3; col++) {
            T acc = V[0][col] * A[row][0];
            T u = V[1][col] * A[row][1];
            acc = acc + u;
            u = V[2][col] * A[row][2];
            acc = acc + u;
            B[row][col] = acc;
        }

    T rho[3];
    for (int col = 0; col < 3; col++) {
        T acc = B[0][col] * B[0][col];
        T u = B[1][col] * B[1][col];
        acc = acc + u;
        u = B[2][col] * B[2][col];
        acc = acc + u;
        rho[col] = acc;
    }
    swap_columns_if<T>(B, V, rho, 0, 1, 1);
    swap_columns_if<T>(B, V, rho, 0, 2, 0);
    swap_columns_if<T>(B, V, rho, 1, 2, 2);

    // 5. QR by Givens rotations
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) U[i][j] = (i == j) ? (T)1 : (T)0;
    qr_givens<T>(B, U, 0, 1, 0);
    qr_givens<T>(B, U, 0, 2, 0);
    qr_givens<T>(B, U, 1, 2, 1);
    S[0] = B[0][0]; S[1] = B[1][1]; S[2] = B[2][2];
}

template <typename T>
void svd_entry(const double Ain[9], double Uout[9], double Sout[3], double Vout[9], int sweeps) {
    T A[3][3], U[3][3], S[3], V[3][3];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) A[i][j] = (T)Ain[3 * i + j];
    svd_mcadams<T>(A, U, S, V, sweeps);
    for (int i = 0; i < 3; i++) {
        Sout[i] = (double)S[i];
        for (int j = 0; j < 3; j++) {
            Uout[3 * i + j] = (double)U[i][j];
            Vout[3 * i + j] = (double)V[i][j];
        }
    }
}

}  // namespace

extern "C" void or_svd3x3_f32(const double A[9], double U[9], double S[3], double V[9]) {
    svd_entry<float>(A, U, S, V, 4);
}

extern "C" void or_svd3x3_f64(const double A[9], double U[9], double S[3], double V[9], int sweeps) {
    svd_entry<double>(A, U, S, V, sweeps);
}

// Forward-mode derivative of or_svd3x3_f64: the same iteration carried out in
// dual numbers, A + eps dA -> (U, S, V) + eps (dU, dS, dV).
extern "C" void or_svd3x3_dual(const double A[9], const double dA[9], double U[9], double dU[9], double S[3],
                               double dS[3], double V[9], double dV[9], int sweeps) {
    Dual a[3][3], u[3][3], s[3], v[3][3];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) a[i][j] = Dual(A[3 * i + j], dA[3 * i + j]);
    svd_mcadams<Dual>(a, u, s, v, sweeps);
    for (int i = 0; i < 3; i++) {
        S[i] = s[i].v;
        dS[i] = s[i].d;
        for (int j = 0; j < 3; j++) {
            U[3 * i + j] = u[i][j].v; dU[3 * i + j] = u[i][j].d;
            V[3 * i + j] = v[i][j].v; dV[3 * i + j] = v[i][j].d;
        }
    }
}
