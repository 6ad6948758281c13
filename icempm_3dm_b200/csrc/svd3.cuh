// 3x3 singular value decomposition for the Drucker-Prager return map.
//
// Algorithm of McAdams, Selle, Tamstorf, Teran and Sifakis, "Computing the
// Singular Value Decomposition of 3x3 matrices with minimal branching and
// elementary floating point operations" (UW-Madison CS TR1690, 2011): Jacobi
// eigen-analysis of A^T A with approximate Givens quaternions, sorting of
// the columns of A V, QR of A V by Givens rotations.
//
// The reference calls this algorithm through helper_math.cuh:24-1120 with
// its inputs narrowed to float. SvdF32 reproduces that computation: every
// add, subtract and multiply is a separately rounded IEEE float operation
// (__fadd_rn/__fsub_rn/__fmul_rn are never fused into FMA), __frsqrt_rn is
// correctly rounded, and the three constants are the reference's float
// values, so the result is bit-identical to the reference's on the same
// input. SvdF64 runs the same steps in double with more sweeps; it is the
// "FP64 SVD" of the mixed-precision and FP64-SVD modes.
#pragma once

#include <cuda_runtime.h>

namespace icempm {

struct SvdF32 {
    typedef float T;
    static constexpr int kSweeps = 4;
    __device__ static __forceinline__ T add(T a, T b) { return __fadd_rn(a, b); }
    __device__ static __forceinline__ T sub(T a, T b) { return __fsub_rn(a, b); }
    __device__ static __forceinline__ T mul(T a, T b) { return __fmul_rn(a, b); }
    __device__ static __forceinline__ T rsqrt(T a) { return __frsqrt_rn(a); }
    __device__ static __forceinline__ T fmax_(T a, T b) { return fmaxf(a, b); }
    __device__ static __forceinline__ T tiny() { return 1.e-20f; }
    __device__ static __forceinline__ T small() { return 1.e-12f; }
    __device__ static __forceinline__ T four_gamma_sq() { return 0x1.7504f4p+2f; }
    __device__ static __forceinline__ T sin_pi8() { return 0x1.87de2ap-2f; }
    __device__ static __forceinline__ T cos_pi8() { return 0x1.d906bep-1f; }
};

struct SvdF64 {
    typedef double T;
    static constexpr int kSweeps = 8;
    __device__ static __forceinline__ T add(T a, T b) { return __dadd_rn(a, b); }
    __device__ static __forceinline__ T sub(T a, T b) { return __dsub_rn(a, b); }
    __device__ static __forceinline__ T mul(T a, T b) { return __dmul_rn(a, b); }
    __device__ static __forceinline__ T rsqrt(T a) { return 1.0 / sqrt(a); }
    __device__ static __forceinline__ T fmax_(T a, T b) { return fmax(a, b); }
    __device__ static __forceinline__ T tiny() { return 1.e-40; }
    __device__ static __forceinline__ T small() { return 1.e-40; }
    __device__ static __forceinline__ T four_gamma_sq() { return 5.828427124746190; }   // 3 + 2 sqrt 2
    __device__ static __forceinline__ T sin_pi8() { return 0.38268343236508977; }
    __device__ static __forceinline__ T cos_pi8() { return 0.92387953251128674; }
};

namespace svd_detail {

// Jacobi conjugation of the symmetric matrix on the pair (p, q), r the third
// index; the cumulative rotation quaternion is (qs, q_p, q_q, q_r) in the
// axes of p, q, r.
template <class K>
__device__ __forceinline__ void conjugate(typename K::T& a_pp, typename K::T& a_qq, typename K::T& a_pq,
                                          typename K::T& a_rp, typename K::T& a_rq, typename K::T& a_rr,
                                          typename K::T& qs, typename K::T& q_p, typename K::T& q_q,
                                          typename K::T& q_r) {
    typedef typename K::T T;
    T sh = K::mul(a_pq, (T)0.5);
    T d = K::sub(a_pp, a_qq);
    const bool rotate = K::mul(sh, sh) >= K::tiny();
    T ch = rotate ? d : (T)1;
    sh = rotate ? sh : (T)0;

    T sh2 = K::mul(sh, sh);
    T ch2 = K::mul(ch, ch);
    T w = K::rsqrt(K::add(sh2, ch2));
    sh = K::mul(w, sh);
    ch = K::mul(w, ch);
    const bool eighth = ch2 <= K::mul(K::four_gamma_sq(), sh2);
    sh = eighth ? K::sin_pi8() : sh;
    ch = eighth ? K::cos_pi8() : ch;

    sh2 = K::mul(sh, sh);
    ch2 = K::mul(ch, ch);
    T c = K::sub(ch2, sh2);
    T s = K::mul(ch, sh);
    s = K::add(s, s);

    T scale = K::add(sh2, ch2);
    a_rr = K::mul(a_rr, scale);
    a_rp = K::mul(a_rp, scale);
    a_rq = K::mul(a_rq, scale);
    a_rr = K::mul(a_rr, scale);

    T t1 = K::mul(s, a_rp);
    T t2 = K::mul(s, a_rq);
    a_rp = K::add(t2, K::mul(c, a_rp));
    a_rq = K::sub(K::mul(c, a_rq), t1);

    T ss = K::mul(s, s);
    T qq_s = K::mul(a_qq, ss);
    T pp_s = K::mul(a_pp, ss);
    T cc = K::mul(c, c);
    a_pp = K::add(K::mul(a_pp, cc), qq_s);
    a_qq = K::add(K::mul(a_qq, cc), pp_s);
    T c2s2 = K::sub(cc, ss);
    T pq2 = K::add(a_pq, a_pq);
    a_pq = K::mul(a_pq, c2s2);
    T cs = K::mul(c, s);
    pq2 = K::mul(pq2, cs);
    d = K::mul(d, cs);
    a_pp = K::add(a_pp, pq2);
    a_pq = K::sub(a_pq, d);
    a_qq = K::sub(a_qq, pq2);

    T u_p = K::mul(sh, q_p);
    T u_q = K::mul(sh, q_q);
    T u_r = K::mul(sh, q_r);
    T u_s = K::mul(sh, qs);
    q_r = K::add(K::mul(ch, q_r), u_s);
    qs = K::sub(K::mul(ch, qs), u_r);
    q_p = K::add(K::mul(ch, q_p), u_q);
    q_q = K::sub(K::mul(ch, q_q), u_p);
}

// rsqrt with one Newton step: r + r/2 - n r^3 / 2
template <class K>
__device__ __forceinline__ typename K::T refined_rsqrt(typename K::T n) {
    typedef typename K::T T;
    T r = K::rsqrt(n);
    T h = K::mul(r, (T)0.5);
    T t = K::mul(r, h);
    t = K::mul(r, t);
    t = K::mul(n, t);
    return K::sub(K::add(r, h), t);
}

// Givens rotation on rows (i, j) of B annihilating B[j][col]; U accumulates
// it in its columns (i, j).
template <class K>
__device__ __forceinline__ void qr_givens(typename K::T B[3][3], typename K::T U[3][3], int i, int j, int col) {
    typedef typename K::T T;
    T a = B[i][col];
    T b = B[j][col];
    T sh = K::mul(b, b) >= K::small() ? b : (T)0;
    T ch = K::fmax_(K::sub((T)0, a), a);
    ch = K::fmax_(ch, K::small());
    const bool pos = a >= (T)0;

    T n = K::add(K::mul(ch, ch), K::mul(sh, sh));
    T r = K::mul(refined_rsqrt<K>(n), n);
    ch = K::add(ch, r);
    T ch_s = pos ? ch : sh;
    T sh_s = pos ? sh : ch;

    n = K::add(K::mul(ch_s, ch_s), K::mul(sh_s, sh_s));
    r = refined_rsqrt<K>(n);
    ch = K::mul(ch_s, r);
    sh = K::mul(sh_s, r);

    T c = K::sub(K::mul(ch, ch), K::mul(sh, sh));
    T s = K::mul(sh, ch);
    s = K::add(s, s);

#pragma unroll
    for (int k = 0; k < 3; k++) {
        T u = K::mul(s, B[i][k]);
        T v = K::mul(s, B[j][k]);
        B[i][k] = K::add(K::mul(c, B[i][k]), v);
        B[j][k] = K::sub(K::mul(c, B[j][k]), u);
    }
#pragma unroll
    for (int k = 0; k < 3; k++) {
        T u = K::mul(s, U[k][i]);
        T v = K::mul(s, U[k][j]);
        U[k][i] = K::add(K::mul(c, U[k][i]), v);
        U[k][j] = K::sub(K::mul(c, U[k][j]), u);
    }
}

template <class K>
__device__ __forceinline__ void sort_pair(typename K::T B[3][3], typename K::T V[3][3], typename K::T rho[3],
                                          int a, int b, int negate) {
    typedef typename K::T T;
    const bool sw = rho[a] < rho[b];
#pragma unroll
    for (int k = 0; k < 3; k++) {
        T ba = B[k][a], bb = B[k][b], va = V[k][a], vb = V[k][b];
        B[k][a] = sw ? bb : ba;
        B[k][b] = sw ? ba : bb;
        V[k][a] = sw ? vb : va;
        V[k][b] = sw ? va : vb;
    }
    T ra = rho[a], rb = rho[b];
    rho[a] = sw ? rb : ra;
    rho[b] = sw ? ra : rb;
#pragma unroll
    for (int k = 0; k < 3; k++) {
        B[k][negate] = sw ? -B[k][negate] : B[k][negate];
        V[k][negate] = sw ? -V[k][negate] : V[k][negate];
    }
}

}  // namespace svd_detail

// A = U diag(S) V^T; A, U, V row-major 3x3 in the working type of K.
template <class K>
__device__ __forceinline__ void svd3x3(const typename K::T A[3][3], typename K::T U[3][3], typename K::T S[3],
                                       typename K::T V[3][3]) {
    typedef typename K::T T;
    using namespace svd_detail;
    // normal equations, s_ij = (a0i a0j + a1i a1j) + a2i a2j
    T s00, s10, s11, s20, s21, s22;
    {
        T m[3][3];
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = 0; j <= i; j++) {
                T acc = K::mul(A[0][j], A[0][i]);
                acc = K::add(K::mul(A[1][j], A[1][i]), acc);
                acc = K::add(K::mul(A[2][j], A[2][i]), acc);
                m[i][j] = acc;
            }
        s00 = m[0][0]; s10 = m[1][0]; s11 = m[1][1]; s20 = m[2][0]; s21 = m[2][1]; s22 = m[2][2];
    }
    T qs = (T)1, qx = (T)0, qy = (T)0, qz = (T)0;
#pragma unroll 1
    for (int it = 0; it < K::kSweeps; it++) {
        conjugate<K>(s00, s11, s10, s20, s21, s22, qs, qx, qy, qz);   // (1,2), axis z
        conjugate<K>(s11, s22, s21, s10, s20, s00, qs, qy, qz, qx);   // (2,3), axis x
        conjugate<K>(s22, s00, s20, s21, s10, s11, qs, qz, qx, qy);   // (3,1), axis y
    }

    T n = K::mul(qs, qs);
    n = K::add(K::mul(qx, qx), n);
    n = K::add(K::mul(qy, qy), n);
    n = K::add(K::mul(qz, qz), n);
    T r = refined_rsqrt<K>(n);
    qs = K::mul(qs, r); qx = K::mul(qx, r); qy = K::mul(qy, r); qz = K::mul(qz, r);

    T xx = K::mul(qx, qx), yy = K::mul(qy, qy), zz = K::mul(qz, qz), ss = K::mul(qs, qs);
    T d2 = K::sub(ss, xx);
    V[2][2] = K::add(K::sub(d2, yy), zz);
    V[1][1] = K::sub(K::add(d2, yy), zz);
    V[0][0] = K::sub(K::sub(K::add(ss, xx), yy), zz);
    T x2 = K::add(qx, qx), y2 = K::add(qy, qy), z2 = K::add(qz, qz);
    T sx = K::mul(qs, x2), sy = K::mul(qs, y2), sz = K::mul(qs, z2);
    T xy = K::mul(qy, x2), yz = K::mul(qz, y2), zx = K::mul(qx, z2);
    V[0][1] = K::sub(xy, sz); V[1][0] = K::add(xy, sz);
    V[1][2] = K::sub(yz, sx); V[2][1] = K::add(yz, sx);
    V[2][0] = K::sub(zx, sy); V[0][2] = K::add(zx, sy);

    T B[3][3];
#pragma unroll
    for (int row = 0; row < 3; row++)
#pragma unroll
        for (int col = 0; col < 3; col++) {
            T acc = K::mul(V[0][col], A[row][0]);
            acc = K::add(acc, K::mul(V[1][col], A[row][1]));
            acc = K::add(acc, K::mul(V[2][col], A[row][2]));
            B[row][col] = acc;
        }
    T rho[3];
#pragma unroll
    for (int col = 0; col < 3; col++) {
        T acc = K::mul(B[0][col], B[0][col]);
        acc = K::add(acc, K::mul(B[1][col], B[1][col]));
        acc = K::add(acc, K::mul(B[2][col], B[2][col]));
        rho[col] = acc;
    }
    sort_pair<K>(B, V, rho, 0, 1, 1);
    sort_pair<K>(B, V, rho, 0, 2, 0);
    sort_pair<K>(B, V, rho, 1, 2, 2);

#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) U[i][j] = (i == j) ? (T)1 : (T)0;
    qr_givens<K>(B, U, 0, 1, 0);
    qr_givens<K>(B, U, 0, 2, 0);
    qr_givens<K>(B, U, 1, 2, 1);
    S[0] = B[0][0]; S[1] = B[1][1]; S[2] = B[2][2];
}

}  // namespace icempm
