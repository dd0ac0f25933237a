// fm_device.cuh — device helpers shared by the FlexMesh kernels:
// warp reductions, acquire/release flags with bounded waits, the
// deterministic last-block reduction, and the tetrahedron kinematics and
// Neo-Hookean constitutive evaluation.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "fm_api.h"

namespace fm {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kWarp = 32;
// Bounded device waits: a wait that sees no progress for this many SM clock
// cycles (about 1 s at B200 clocks) records FM_FLAG_TIMEOUT and returns.
// A context can set another limit (fm_set_wait_limit): it travels in the
// word after every status word the library hands to kernels, in units of
// 1024 cycles (0: this default).
constexpr long long kWaitCycles = 2000000000ll;
// Reference constants (FEM/adaptive_fem_engine.hpp:102,141,170,308-309).
constexpr double kJSafe = 0.01;
constexpr double kPivotThreshold = 1e-12;
constexpr double kPivotPerturb = 1e-8;

// Scalars shared by solver kernels, resident in device memory.
struct DevScalars {
    double rr;       // r.r after r = b - A x0
    double rz;       // current r.z
    double rz_new;   // r.z after the latest preconditioner apply
    double pAp;      // p.Ap
    double bb;       // b.b
    double relres;   // sqrt(rz_new / max(b.b, 1e-300))
    double norm2;    // generic reduction output
    double scale;    // rhs scaling for the FP32 inner solve
    double guess_xb, guess_xkx;  // x_prev . b and x_prev . K x_prev (initial guess)
    unsigned stop;   // 1: |pAp| < 1e-60 breakdown
    unsigned status; // FM_FLAG_* bits
    unsigned wait_budget;  // bounded-wait limit in 1024 cycles (0: kWaitCycles); follows status
    unsigned counter[8];  // last-block counters (one per reduction site)
    unsigned never;       // a flag no kernel sets (fm_check_wait waits on it)
    unsigned state_counts[2];   // element state update: |det F_sl3 - 1| > 1e-8, non-finite
};

constexpr int kRedBlocks = 296;  // 2 x 148 SMs: fixed grid => fixed summation order

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
    return v;
}

__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release(unsigned* p, unsigned v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned ld_volatile_u32(const unsigned* p) {
    return *reinterpret_cast<const volatile unsigned*>(p);
}
// L2-coherent loads of values produced by other SMs during the same kernel
__device__ __forceinline__ double ld_cg(const double* p) { return __ldcg(p); }
__device__ __forceinline__ float ld_cg(const float* p) { return __ldcg(p); }

__device__ __forceinline__ void raise_flag(unsigned* status, unsigned bits) {
    atomicOr(status, bits);
}

// The wait limit in SM cycles that travels with a status word (the next word).
__device__ __forceinline__ long long wait_limit(const unsigned* status) {
    const unsigned b = ld_volatile_u32(status + 1);
    return b ? (long long)b << 10 : kWaitCycles;
}

// Spin until *flag == epoch.  Returns false (and sets FM_FLAG_TIMEOUT) when
// the wait exceeds kWaitCycles or another thread already timed out, so no
// wait can run unbounded.
__device__ __forceinline__ bool wait_flag(const unsigned* flag, unsigned epoch,
                                          unsigned* status) {
    if (ld_acquire(flag) == epoch) return true;
    const long long t0 = clock64(), limit = wait_limit(status);
    for (unsigned it = 1;; ++it) {
        if (ld_acquire(flag) == epoch) return true;
        if ((it & 31u) == 0) {
            if (ld_volatile_u32(status) & FM_FLAG_TIMEOUT) return false;
            if (clock64() - t0 > limit) {
                raise_flag(status, FM_FLAG_TIMEOUT);
                return false;
            }
        }
    }
}

// Warp-uniform bounded wait: every lane with `need` waits for *flag ==
// epoch (acquire loads); all lanes leave together (the exit test is a warp
// vote), so the warp never splits into separately spinning lanes.  A
// caller's __syncwarp after it extends each lane's acquire to the whole
// warp.  After 16 polls the loop sleeps between polls, doubling from 32 ns
// up to sleep_ns (0: never sleeps).  Returns false (FM_FLAG_TIMEOUT set)
// when the wait exceeds kWaitCycles or another wait already timed out.
__device__ __forceinline__ bool wait_flags_warp(const unsigned* flag, bool need, unsigned epoch,
                                                unsigned* status, unsigned sleep_ns) {
    bool ok = !need || ld_acquire(flag) == epoch;
    if (__all_sync(kFull, ok)) return true;
    const long long t0 = clock64(), limit = wait_limit(status);
    unsigned ns = 32;
    for (unsigned it = 1;; ++it) {
        if (sleep_ns && it > 16) {
            __nanosleep(ns);
            if (ns < sleep_ns) ns <<= 1;
        }
        if (!ok) ok = ld_acquire(flag) == epoch;
        if (__all_sync(kFull, ok)) return true;
        if ((it & 31u) == 0 &&
            __any_sync(kFull, (ld_volatile_u32(status) & FM_FLAG_TIMEOUT) ||
                                  clock64() - t0 > limit)) {
            if ((threadIdx.x & 31) == 0) raise_flag(status, FM_FLAG_TIMEOUT);
            return false;
        }
    }
}

// Block-wide sum (blockDim.x multiple of 32, <= 1024).
template <typename T>
__device__ __forceinline__ T block_sum(T v, T* sbuf) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    v = warp_sum(v);
    __syncthreads();
    if (lane == 0) sbuf[w] = v;
    __syncthreads();
    T r = (threadIdx.x < nw) ? sbuf[threadIdx.x] : T(0);
    if (w == 0) r = warp_sum(r);
    return r;  // valid in thread 0
}

// Deterministic grid reduction: each block writes its partial; the last
// block to arrive sums the partials in block order and calls fin(total).
// Works for any grid size <= number of partial slots.
template <typename T, typename Fin>
__device__ __forceinline__ void grid_reduce_finish(T block_total, T* partials, unsigned* counter,
                                                   Fin fin) {
    __shared__ bool last;
    __syncthreads();  // a previous call's readers of `last` are done
    if (threadIdx.x == 0) {
        partials[blockIdx.x] = block_total;
        __threadfence();
        unsigned t = atomicAdd(counter, 1u);
        last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (last) {
        __threadfence();
        T s = T(0);
        // fixed order: thread t sums partials t, t+blockDim, ... then tree
        for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x) s += ld_cg(partials + b);
        __shared__ T sbuf[32];
        s = block_sum(s, sbuf);
        if (threadIdx.x == 0) {
            fin(s);
            *counter = 0u;
        }
    }
}

// ---------------------------------------------------------------------------
// Tetrahedron kinematics and constitutive law
// ---------------------------------------------------------------------------
// Shape-function gradients dN_a = J^-T dN_xi(a) of the linear tet, the
// deformation gradient F = I + sum_a u_a (x) dN_a and J = det F, as in
// tet_element_stiffness_rigorous (FEM/adaptive_fem_engine.hpp:519-580).
struct TetKin {
    double d[4][3];
    double F[9];
    double J;
    double vol;
};

__device__ __forceinline__ bool tet_kinematics(const double x[12], const double u[12], TetKin& k) {
    double m[9];
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        m[r * 3 + 0] = x[3 + r] - x[r];
        m[r * 3 + 1] = x[6 + r] - x[r];
        m[r * 3 + 2] = x[9 + r] - x[r];
    }
    const double c0 = m[4] * m[8] - m[7] * m[5];
    const double c1 = m[1] * m[8] - m[7] * m[2];
    const double c2 = m[1] * m[5] - m[4] * m[2];
    const double det = m[0] * c0 - m[3] * c1 + m[6] * c2;
    k.vol = fabs(det) / 6.0;
    if (!(k.vol >= 1e-30)) return false;
    const double inv = 1.0 / det;
    double ji[9];
    ji[0] = c0 * inv;
    ji[1] = -c1 * inv;
    ji[2] = c2 * inv;
    ji[3] = -(m[3] * m[8] - m[6] * m[5]) * inv;
    ji[4] = (m[0] * m[8] - m[6] * m[2]) * inv;
    ji[5] = -(m[0] * m[5] - m[3] * m[2]) * inv;
    ji[6] = (m[3] * m[7] - m[6] * m[4]) * inv;
    ji[7] = -(m[0] * m[7] - m[6] * m[1]) * inv;
    ji[8] = (m[0] * m[4] - m[3] * m[1]) * inv;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        k.d[1][c] = ji[c];
        k.d[2][c] = ji[3 + c];
        k.d[3][c] = ji[6 + c];
        k.d[0][c] = -ji[c] - ji[3 + c] - ji[6 + c];
    }
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b) {
            double s = u[a] * k.d[0][b];
            s += u[3 + a] * k.d[1][b];
            s += u[6 + a] * k.d[2][b];
            s += u[9 + a] * k.d[3][b];
            k.F[a * 3 + b] = (a == b) ? 1.0 + s : s;
        }
    const double* F = k.F;
    k.J = F[0] * (F[4] * F[8] - F[7] * F[5]) - F[3] * (F[1] * F[8] - F[7] * F[2]) +
          F[6] * (F[1] * F[5] - F[4] * F[2]);
    return true;
}

// g = dN_a for a runtime local index a, by selects (indexing the register
// array with a runtime value would move it to local memory)
__device__ __forceinline__ void grad_of(const TetKin& k, int a, double g[3]) {
#pragma unroll
    for (int c = 0; c < 3; ++c)
        g[c] = a == 0 ? k.d[0][c] : a == 1 ? k.d[1][c] : a == 2 ? k.d[2][c] : k.d[3][c];
}

// Mandel stress M = C S with S = mu (I - C^-1) + lam ln(max(J,0.01)) C^-1
// (neo_hookean_response, FEM/adaptive_fem_engine.hpp:79-129), evaluated in
// the closed form M = mu (C - I) + lam lnJ I that C C^-1 = I gives; the
// reference's Voigt round trip M01*sqrt2/sqrt2 is the identity up to one
// rounding.  A degenerate C (det C = J^2 < 1e-30) takes the reference's
// guarded inverse instead.  Out: symmetric M as (00,11,22,01,02,12) and lnJ.
struct Mandel {
    double m00, m11, m22, m01, m02, m12;
    double lnJ;
};

// |det C| < 1e-30 for C = F^T F, each operation rounded as the reference's
// neo_hookean_response and matrix_3x3_inv round it (:88-96, :53-56)
static __device__ __noinline__ bool degenerate_c(double f0, double f1, double f2, double f3,
                                                  double f4, double f5, double f6, double f7,
                                                  double f8) {
    const double F[9] = {f0, f1, f2, f3, f4, f5, f6, f7, f8};
    double C[9];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            double acc = 0.0;
            for (int k = 0; k < 3; ++k) acc = __dadd_rn(acc, __dmul_rn(F[k * 3 + i], F[k * 3 + j]));
            C[i * 3 + j] = acc;
        }
    const double t0 = __dsub_rn(__dmul_rn(C[4], C[8]), __dmul_rn(C[7], C[5]));
    const double t1 = __dsub_rn(__dmul_rn(C[1], C[8]), __dmul_rn(C[7], C[2]));
    const double t2 = __dsub_rn(__dmul_rn(C[1], C[5]), __dmul_rn(C[4], C[2]));
    const double det =
        __dadd_rn(__dsub_rn(__dmul_rn(C[0], t0), __dmul_rn(C[3], t1)), __dmul_rn(C[6], t2));
    return fabs(det) < 1e-30;
}

__device__ __forceinline__ Mandel mandel_stress(const double F[9], double J, double mu, double lam) {
    Mandel M;
    const double c00 = F[0] * F[0] + F[3] * F[3] + F[6] * F[6];
    const double c11 = F[1] * F[1] + F[4] * F[4] + F[7] * F[7];
    const double c22 = F[2] * F[2] + F[5] * F[5] + F[8] * F[8];
    const double c01 = F[0] * F[1] + F[3] * F[4] + F[6] * F[7];
    const double c02 = F[0] * F[2] + F[3] * F[5] + F[6] * F[8];
    const double c12 = F[1] * F[2] + F[4] * F[5] + F[7] * F[8];
    const double Js = J < kJSafe ? kJSafe : J;
    M.lnJ = log(Js);
    const double vol = lam * M.lnJ;
    // det C = J^2 below matrix_3x3_inv's 1e-30 guard (:56-60) makes the
    // reference's C^-1 1e30 I, S = (mu (1 - 1e30) + lam lnJ 1e30) I and
    // M = C S.  Near a singular F the guard sees det C through its own
    // rounding, so there the decision is taken on det C formed as the
    // reference forms it (C_ij = sum_k F_ki F_kj, cofactor expansion,
    // no fused operations)
    if (J * J < 1e-10 && degenerate_c(F[0], F[1], F[2], F[3], F[4], F[5], F[6], F[7], F[8])) {
        const double s = mu * (1.0 - 1e30) + vol * 1e30;
        M.m00 = s * c00;
        M.m11 = s * c11;
        M.m22 = s * c22;
        M.m01 = s * c01;
        M.m02 = s * c02;
        M.m12 = s * c12;
        return M;
    }
    M.m00 = mu * (c00 - 1.0) + vol;
    M.m11 = mu * (c11 - 1.0) + vol;
    M.m22 = mu * (c22 - 1.0) + vol;
    M.m01 = mu * c01;
    M.m02 = mu * c02;
    M.m12 = mu * c12;
    return M;
}

// The reference's 6x6 Voigt tangent (neo_hookean_tangent, :135-187) has the
// form: normal block a on the diagonal, b off it; shear diagonal mu.
//   a = 2mu + (lam + 2mu/3) + lam / ((J_s + 1e-30) max(1-2nu, 0.1))
//   b = (lam + 2mu/3) - 2mu/3 - 2 lam lnJ / (3 (J_s + 1e-30))
// inv_cnu = 1 / max(1-2nu, 0.1).
__device__ __forceinline__ void tangent_ab(double mu, double lam, double J, double lnJ,
                                           double inv_cnu, double& a, double& b) {
    const double Js = J < kJSafe ? kJSafe : J;
    const double invJ = 1.0 / (Js + 1e-30);
    const double bulk = lam + 2.0 * mu / 3.0;
    a = 2.0 * mu + bulk + lam * invJ * inv_cnu;
    b = bulk - 2.0 * mu / 3.0 + (-2.0 * lam * lnJ * invJ / 3.0);
}

// 3x3 block (i,j) of the element tangent, scaled by vol, for owner node
// gradient dI, neighbour gradient dJ, fI = vol M dI (the element force at
// the owner node, which also carries the geometric term fI . dJ):
//   K_pq = va dI_p dJ_q (p==q) + vb dI_p dJ_q (p!=q)
//        + vm (p==q ? sum_{r!=p} dI_r dJ_r : dI_q dJ_p) + (p==q) fI.dJ
// This is vol (B_i^T C B_j + (dN_i . sigma . dN_j) I) of :599-692 written
// out for the tangent's sparsity.
template <typename T>
__device__ __forceinline__ void tangent_block_acc(const T dI[3], const T dJ[3], const T fI[3], T va,
                                                  T vb, T vm, T acc[9]) {
    const T t00 = dI[0] * dJ[0], t01 = dI[0] * dJ[1], t02 = dI[0] * dJ[2];
    const T t10 = dI[1] * dJ[0], t11 = dI[1] * dJ[1], t12 = dI[1] * dJ[2];
    const T t20 = dI[2] * dJ[0], t21 = dI[2] * dJ[1], t22 = dI[2] * dJ[2];
    const T g = fI[0] * dJ[0] + fI[1] * dJ[1] + fI[2] * dJ[2];
    acc[0] += va * t00 + vm * (t11 + t22) + g;
    acc[4] += va * t11 + vm * (t00 + t22) + g;
    acc[8] += va * t22 + vm * (t00 + t11) + g;
    acc[1] += vb * t01 + vm * t10;
    acc[2] += vb * t02 + vm * t20;
    acc[3] += vb * t10 + vm * t01;
    acc[5] += vb * t12 + vm * t21;
    acc[6] += vb * t20 + vm * t02;
    acc[7] += vb * t21 + vm * t12;
}

__device__ __forceinline__ void material_of(int mat_mode, const double* m0, const double* m1,
                                            uint32_t e, double mu_s, double lam_s, double c_mu,
                                            double c_lam, double& mu, double& lam) {
    if (mat_mode == 0) {
        mu = mu_s;
        lam = lam_s;
    } else if (mat_mode == 1) {
        const double E = __ldg(m0 + e);
        mu = E * c_mu;
        lam = E * c_lam;
    } else {
        mu = __ldg(m0 + e);
        lam = __ldg(m1 + e);
    }
}

}  // namespace fm
