// fm_lie.cuh — 3x3 matrix functions of the element state update, in FP64,
// on the reference's Matrix3x3 data layout (CORE/lie_operator.hpp:
// data[c*3 + r], column-major; the products below are its matrix_multiply).
//
// Published methods, restated step for step as the reference applies them
// (CORE/lie_operator.cpp) so that branch decisions (scaling exponents,
// square-root counts, Newton clean-up) fall the same way:
//   expm  scaling and squaring with the [3/3] Pade approximant (Higham,
//         "Functions of Matrices", 2008, sec. 10.3; theta_3 = 1.495585...),
//         one extra squaring when the 1-norm condition estimate exceeds
//         1e8, then det(R) rescaled to exp(tr A) by a cube root (:95-152);
//   sqrtm Denman-Beavers iteration (Higham 2008, sec. 6.3), stopped when
//         ||Y^2 - A||_F < 4e-16, at most 20 steps (:164-184);
//   logm  inverse scaling and squaring: square roots until ||B - I||_inf <
//         0.125, then the Gregory series log B = 2 atanh((B-I)(B+I)^-1)
//         to 33 terms, rescaled by 2^k, and up to 4 Newton corrections
//         L += (A - e^L) e^-L kept while they reduce ||A - e^L||_F (:200-268);
//   sl3   retraction exp(log G + V), rescaled to det 1 (:300-311).
// exp, log2, cbrt and sqrt are CUDA's own.
#pragma once

#include <math.h>

#include <cuda_runtime.h>

// device code; also host code so that a CPU build can check it against the
// oracle's restatement
#ifdef __CUDACC__
#define FM_LIE_FN __host__ __device__ __forceinline__
#define FM_LIE_NOINLINE __host__ __device__ __noinline__
#else
#define FM_LIE_FN inline
#define FM_LIE_NOINLINE inline
#endif

namespace fm {
namespace lie {

struct M3 {
    double a[9];
};

FM_LIE_FN M3 ident() {
    M3 r;
#pragma unroll
    for (int i = 0; i < 9; ++i) r.a[i] = (i % 4 == 0) ? 1.0 : 0.0;
    return r;
}
FM_LIE_FN M3 zero() {
    M3 r;
#pragma unroll
    for (int i = 0; i < 9; ++i) r.a[i] = 0.0;
    return r;
}
FM_LIE_FN M3 add(const M3& A, const M3& B) {
    M3 r;
#pragma unroll
    for (int i = 0; i < 9; ++i) r.a[i] = A.a[i] + B.a[i];
    return r;
}
FM_LIE_FN M3 sub(const M3& A, const M3& B) {
    M3 r;
#pragma unroll
    for (int i = 0; i < 9; ++i) r.a[i] = A.a[i] - B.a[i];
    return r;
}
FM_LIE_FN M3 scale(const M3& A, double s) {
    M3 r;
#pragma unroll
    for (int i = 0; i < 9; ++i) r.a[i] = A.a[i] * s;
    return r;
}
// C = A B, column-major: C(r,c) = sum_k A(r,k) B(k,c)
FM_LIE_FN M3 mul(const M3& A, const M3& B) {
    M3 C;
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int r = 0; r < 3; ++r)
            C.a[3 * c + r] =
                A.a[r] * B.a[3 * c] + A.a[3 + r] * B.a[3 * c + 1] + A.a[6 + r] * B.a[3 * c + 2];
    return C;
}
FM_LIE_FN double trace(const M3& A) { return A.a[0] + A.a[4] + A.a[8]; }
FM_LIE_FN double frob_sq(const M3& A) {
    double s = 0.0;
#pragma unroll
    for (int i = 0; i < 9; ++i) s += A.a[i] * A.a[i];
    return s;
}
FM_LIE_FN double frob(const M3& A) { return sqrt(frob_sq(A)); }
// max row sum / max column sum of |a| in the column-major layout
FM_LIE_FN double inf_norm(const M3& A) {
    double m = 0.0;
#pragma unroll
    for (int r = 0; r < 3; ++r) m = fmax(m, fabs(A.a[r]) + fabs(A.a[3 + r]) + fabs(A.a[6 + r]));
    return m;
}
FM_LIE_FN double one_norm(const M3& A) {
    double m = 0.0;
#pragma unroll
    for (int c = 0; c < 3; ++c)
        m = fmax(m, fabs(A.a[3 * c]) + fabs(A.a[3 * c + 1]) + fabs(A.a[3 * c + 2]));
    return m;
}
FM_LIE_FN double det(const M3& A) {
    return A.a[0] * (A.a[4] * A.a[8] - A.a[7] * A.a[5]) -
           A.a[3] * (A.a[1] * A.a[8] - A.a[7] * A.a[2]) +
           A.a[6] * (A.a[1] * A.a[5] - A.a[4] * A.a[2]);
}
// cofactor inverse; |det| < 1e-15 gives the identity (the reference's guard)
FM_LIE_FN M3 inv(const M3& A) {
    const double a00 = A.a[0], a10 = A.a[1], a20 = A.a[2];
    const double a01 = A.a[3], a11 = A.a[4], a21 = A.a[5];
    const double a02 = A.a[6], a12 = A.a[7], a22 = A.a[8];
    const double c00 = a11 * a22 - a21 * a12, c10 = -(a01 * a22 - a21 * a02),
                 c20 = a01 * a12 - a11 * a02;
    const double c01 = -(a10 * a22 - a20 * a12), c11 = a00 * a22 - a20 * a02,
                 c21 = -(a00 * a12 - a10 * a02);
    const double c02 = a10 * a21 - a20 * a11, c12 = -(a00 * a21 - a20 * a01),
                 c22 = a00 * a11 - a10 * a01;
    const double d = a00 * c00 + a10 * c10 + a20 * c20;
    if (fabs(d) < 1.0e-15) return ident();
    const double id = 1.0 / d;
    M3 r;
    r.a[0] = c00 * id;
    r.a[1] = c01 * id;
    r.a[2] = c02 * id;
    r.a[3] = c10 * id;
    r.a[4] = c11 * id;
    r.a[5] = c12 * id;
    r.a[6] = c20 * id;
    r.a[7] = c21 * id;
    r.a[8] = c22 * id;
    return r;
}
FM_LIE_FN double cond_estimate(const M3& A) {
    if (fabs(det(A)) < 1.0e-15) return 1.0e18;
    return fmin(one_norm(A) * one_norm(inv(A)), 1.0e18);
}

FM_LIE_NOINLINE M3 expm(const M3& A) {
    constexpr double b1 = 0.5, b2 = 0.1, b3 = 1.0 / 120.0;
    constexpr double theta3 = 1.495585217958292;
    const double nrm = inf_norm(A);
    if (!isfinite(nrm)) return ident();
    int s = 0;
    if (nrm > theta3) s = (int)ceil(log2(nrm / theta3));
    if (cond_estimate(A) > 1.0e8 && s < 8) ++s;
    const double sc = 1.0 / (double)(1ll << s);
    const M3 X = scale(A, sc);
    const M3 X2 = mul(X, X);
    const M3 X3 = mul(X2, X);
    const M3 I = ident();
    const M3 P = add(add(I, scale(X, b1)), add(scale(X2, b2), scale(X3, b3)));
    const M3 Q = add(add(I, scale(X, -b1)), add(scale(X2, b2), scale(X3, -b3)));
    M3 R = mul(inv(Q), P);
    for (int i = 0; i < s; ++i) R = mul(R, R);
    const double dR = det(R), target = exp(trace(A));
    if (isfinite(dR) && isfinite(target) && dR > 1.0e-300 && target > 1.0e-300)
        R = scale(R, cbrt(target / dR));
    return R;
}

FM_LIE_NOINLINE M3 sqrtm_db(const M3& A) {
    M3 Y = A, Z = ident();
    for (int it = 0; it < 20; ++it) {
        if (frob(sub(mul(Y, Y), A)) < 4.0e-16) break;
        const M3 Yi = inv(Y), Zi = inv(Z);
        const M3 Yn = scale(add(Y, Zi), 0.5);
        const M3 Zn = scale(add(Z, Yi), 0.5);
        Y = Yn;
        Z = Zn;
    }
    return Y;
}

FM_LIE_NOINLINE M3 logm(const M3& A) {
    if (!isfinite(frob_sq(A))) return zero();
    const M3 I = ident();
    {
        const M3 E = sub(A, I);
        if (inf_norm(E) < 1.0e-7) {
            const M3 E2 = mul(E, E);
            const M3 E3 = mul(E2, E);
            return add(sub(E, scale(E2, 0.5)), scale(E3, 1.0 / 3.0));
        }
    }
    M3 B = A;
    int roots = 0;
    for (int k = 0; k < 16; ++k) {
        if (inf_norm(sub(B, I)) < 0.125) break;
        B = sqrtm_db(B);
        ++roots;
    }
    const M3 Z = mul(sub(B, I), inv(add(B, I)));
    const M3 Z2 = mul(Z, Z);
    M3 Zp = Z, sum = Z;
    for (int k = 1; k <= 32; ++k) {
        Zp = mul(Zp, Z2);
        sum = add(sum, scale(Zp, 1.0 / (double)(2 * k + 1)));
    }
    M3 L = scale(scale(sum, 2.0), (double)(1ll << roots));
    M3 best = L;
    double best_rel = INFINITY;
    const double denom = fmax(frob(A), 1.0e-30);
    for (int it = 0; it < 4; ++it) {
        const M3 eL = expm(L);
        const M3 res = sub(A, eL);
        const double rel = frob(res) / denom;
        if (isfinite(rel) && rel < best_rel) {
            best_rel = rel;
            best = L;
        }
        if (rel < 1.0e-12) break;
        const M3 corr = mul(res, inv(eL));
        const double cn = frob(corr);
        if (!isfinite(cn) || cn > 0.25) break;
        L = add(L, corr);
    }
    return best;
}

// exp(log G + V) with V = 0, rescaled to det 1
FM_LIE_FN M3 sl3_retraction(const M3& G) {
    M3 R = expm(add(logm(G), zero()));
    const double d = det(R);
    if (fabs(d) > 1.0e-15) R = scale(R, 1.0 / cbrt(d));
    return R;
}

}  // namespace lie
}  // namespace fm
