// fm_adjoint.cu — exact Jacobian of the internal force and material
// gradients (no reference counterpart: the reference's tangent is a
// heuristic, not the derivative of its force).
//
// The element force is f_a = vol M g_a with M = mu (C - I) + lam lnJ I
// (C = F^T F, lnJ = ln max(J, 0.01), g_a = dN_a), so for a direction v with
// V = sum_b v_b (x) g_b:
//   dM = mu (V^T F + F^T V) + lam tr(F^-1 V) I          (lam term: J >= 0.01)
//   (K v)_a = vol dM g_a
// and for the transpose with L = sum_a w_a (x) g_a:
//   (K^T w)_b = vol [mu F (L + L^T) + lam tr(L) F^-T] g_b
// Parameter derivatives of f: df_a/dmu = vol (C - I) g_a, df_a/dlam =
// vol lnJ g_a, hence with an adjoint w (K^T w = dL/du on free DOFs):
//   dL/dmu_e = -vol (C - I) : L_e,   dL/dlam_e = -vol lnJ tr(L_e).
//
// Products are matrix-free: one warp per node gathers, over the node's
// incident tets (one lane each), the tets' contributions to its three
// entries, summed in ascending element order (deterministic).
#include "fm_adjoint.hpp"
#include "fm_kernels.hpp"

namespace fm {

constexpr int kAdjWarps = 8;

struct Inv3 {
    double m[9];
};

__device__ __forceinline__ Inv3 inverse3(const double F[9], double J) {
    Inv3 r;
    const double s = 1.0 / J;
    r.m[0] = (F[4] * F[8] - F[7] * F[5]) * s;
    r.m[1] = -(F[1] * F[8] - F[7] * F[2]) * s;
    r.m[2] = (F[1] * F[5] - F[4] * F[2]) * s;
    r.m[3] = -(F[3] * F[8] - F[6] * F[5]) * s;
    r.m[4] = (F[0] * F[8] - F[6] * F[2]) * s;
    r.m[5] = -(F[0] * F[5] - F[3] * F[2]) * s;
    r.m[6] = (F[3] * F[7] - F[6] * F[4]) * s;
    r.m[7] = -(F[0] * F[7] - F[6] * F[1]) * s;
    r.m[8] = (F[0] * F[4] - F[3] * F[1]) * s;
    return r;
}

// contribution of one tet to (K v) at local node a (transpose = 0) or to
// (K^T w) at local node a (transpose = 1); ve: the tet's 12 direction values
__device__ __forceinline__ void exact_contrib(const TetKin& k, double mu, double lam,
                                              const double ve[12], int a, int transpose,
                                              double out[3]) {
    double V[9];  // V_ik = sum_b v_b,i g_b,k
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int c = 0; c < 3; ++c)
            V[3 * i + c] = ve[i] * k.d[0][c] + ve[3 + i] * k.d[1][c] + ve[6 + i] * k.d[2][c] +
                           ve[9 + i] * k.d[3][c];
    const double* F = k.F;
    const bool vol_term = k.J >= kJSafe;
    Inv3 Fi;
    if (vol_term) Fi = inverse3(F, k.J);
    double g[3];
    grad_of(k, a, g);
    if (!transpose) {
        double dM[9];
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                double s = 0.0;
#pragma unroll
                for (int m = 0; m < 3; ++m) s += V[3 * m + i] * F[3 * m + c] + F[3 * m + i] * V[3 * m + c];
                dM[3 * i + c] = mu * s;
            }
        if (vol_term) {
            double tr = 0.0;
#pragma unroll
            for (int c = 0; c < 3; ++c)
#pragma unroll
                for (int m = 0; m < 3; ++m) tr += Fi.m[3 * c + m] * V[3 * m + c];
            const double add = lam * tr;
            dM[0] += add;
            dM[4] += add;
            dM[8] += add;
        }
#pragma unroll
        for (int i = 0; i < 3; ++i)
            out[i] = k.vol * (dM[3 * i] * g[0] + dM[3 * i + 1] * g[1] + dM[3 * i + 2] * g[2]);
    } else {
        // V holds L here (same construction from w)
        double Q[9];
#pragma unroll
        for (int j = 0; j < 3; ++j)
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                double s = 0.0;
#pragma unroll
                for (int m = 0; m < 3; ++m) s += F[3 * j + m] * (V[3 * m + c] + V[3 * c + m]);
                Q[3 * j + c] = mu * s;
            }
        if (vol_term) {
            const double tr = lam * (V[0] + V[4] + V[8]);
#pragma unroll
            for (int j = 0; j < 3; ++j)
#pragma unroll
                for (int c = 0; c < 3; ++c) Q[3 * j + c] += tr * Fi.m[3 * c + j];
        }
#pragma unroll
        for (int j = 0; j < 3; ++j)
            out[j] = k.vol * (Q[3 * j] * g[0] + Q[3 * j + 1] * g[1] + Q[3 * j + 2] * g[2]);
    }
}

__device__ __forceinline__ bool load_tet(const MeshDev& m, uint32_t e, const double* u,
                                         uint32_t cn[4], TetKin& k) {
    uint4 c = m.conn[e];
    if (c.x & 0x80000000u) return false;
    cn[0] = c.x;
    cn[1] = c.y;
    cn[2] = c.z;
    cn[3] = c.w;
    double x[12], ue[12];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            x[3 * a + d] = __ldg(m.xyz + 3 * (size_t)cn[a] + d);
            ue[3 * a + d] = __ldg(u + 3 * (size_t)cn[a] + d);
        }
    return tet_kinematics(x, ue, k);
}

__global__ void __launch_bounds__(kAdjWarps * 32)
    k_exact_apply(MeshDev m, const double* __restrict__ u, const double* __restrict__ v,
                  double* __restrict__ y, int transpose) {
    __shared__ double red[kAdjWarps][3][32];
    const int lane = threadIdx.x & 31, wi = threadIdx.x >> 5;
    const uint32_t n = blockIdx.x * kAdjWarps + wi;
    if (n >= m.n_nodes) return;
    const uint32_t e0 = m.inc_ptr[n];
    const int mi = (int)(m.inc_ptr[n + 1] - e0);
    double o[3] = {0.0, 0.0, 0.0};
    if (lane < mi) {
        const uint32_t e = __ldg(m.inc + e0 + lane);
        uint32_t cn[4];
        TetKin k;
        if (load_tet(m, e, u, cn, k)) {
            double mu, lam;
            material_of(m.mat_mode, m.m0, m.m1, e, m.mu_s, m.lam_s, m.c_mu, m.c_lam, mu, lam);
            double ve[12];
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int d = 0; d < 3; ++d) ve[3 * a + d] = __ldg(v + 3 * (size_t)cn[a] + d);
            const int a = (cn[0] == n) ? 0 : (cn[1] == n) ? 1 : (cn[2] == n) ? 2 : 3;
            exact_contrib(k, mu, lam, ve, a, transpose, o);
        }
    }
    red[wi][0][lane] = o[0];
    red[wi][1][lane] = o[1];
    red[wi][2][lane] = o[2];
    __syncwarp();
    if (lane < 3) {
        double s = 0.0;
        for (int l = 0; l < mi; ++l) s += red[wi][lane][l];
        y[3 * (size_t)n + lane] = s;
    }
}

// dL/dmu_e = -vol (C - I) : L_e, dL/dlam_e = -vol lnJ tr(L_e)
__global__ void k_param_grads(MeshDev m, const double* __restrict__ u,
                              const double* __restrict__ w, double* __restrict__ gmu,
                              double* __restrict__ glam) {
    const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= m.n_elems) return;
    uint32_t cn[4];
    TetKin k;
    double a = 0.0, b = 0.0;
    if (load_tet(m, e, u, cn, k)) {
        double L[9];
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                double s = 0.0;
#pragma unroll
                for (int q = 0; q < 4; ++q) s += __ldg(w + 3 * (size_t)cn[q] + i) * k.d[q][c];
                L[3 * i + c] = s;
            }
        const double* F = k.F;
        double cm = 0.0;
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const double Cic = F[i] * F[c] + F[3 + i] * F[3 + c] + F[6 + i] * F[6 + c];
                cm += (Cic - (i == c ? 1.0 : 0.0)) * L[3 * i + c];
            }
        const double Js = k.J < kJSafe ? kJSafe : k.J;
        a = -k.vol * cm;
        b = -k.vol * log(Js) * (L[0] + L[4] + L[8]);
    }
    gmu[e] = a;
    glam[e] = b;
}

// r = mask ? 0 : g - y; returns into out2 the squared norm (deterministic)
__global__ void k_adj_residual(uint32_t n, const uint8_t* __restrict__ mask,
                               const double* __restrict__ g, const double* __restrict__ y,
                               double* __restrict__ r, double* partials, unsigned* counter,
                               double* out2) {
    double s = 0.0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double v = (mask && mask[i]) ? 0.0 : g[i] - y[i];
        r[i] = v;
        s += v * v;
    }
    __shared__ double sbuf[32];
    const double bt = block_sum(s, sbuf);
    grid_reduce_finish<double>(bt, partials, counter, [&](double total) { *out2 = total; });
}

// w += mask ? 0 : dw
__global__ void k_adj_update(uint32_t n, const uint8_t* __restrict__ mask,
                             const double* __restrict__ dw, double* __restrict__ w) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        if (!(mask && mask[i])) w[i] += dw[i];
}

void launch_exact_apply(const MeshDev& m, const double* u, const double* v, double* y,
                        int transpose, cudaStream_t s) {
    if (!m.n_nodes) return;
    k_exact_apply<<<(m.n_nodes + kAdjWarps - 1) / kAdjWarps, kAdjWarps * 32, 0, s>>>(m, u, v, y,
                                                                                      transpose);
}
void launch_param_grads(const MeshDev& m, const double* u, const double* w, double* gmu,
                        double* glam, cudaStream_t s) {
    if (!m.n_elems) return;
    k_param_grads<<<(m.n_elems + 127) / 128, 128, 0, s>>>(m, u, w, gmu, glam);
}
void launch_adj_residual(uint32_t n, const uint8_t* mask, const double* g, const double* y,
                         double* r, double* partials, unsigned* counter, double* out2,
                         cudaStream_t s) {
    k_adj_residual<<<kRedBlocks, 256, 0, s>>>(n, mask, g, y, r, partials, counter, out2);
}
void launch_adj_update(uint32_t n, const uint8_t* mask, const double* dw, double* w,
                       cudaStream_t s) {
    k_adj_update<<<kRedBlocks * 2, 256, 0, s>>>(n, mask, dw, w);
}

}  // namespace fm
