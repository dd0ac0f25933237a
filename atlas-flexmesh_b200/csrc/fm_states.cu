// fm_states.cu — the element state update on the device.
//
// update_element_states_rigorous (FEM/adaptive_fem_engine.hpp:2716-2794)
// runs after every Newton iteration of the engine: per tetrahedron, the
// deformation gradient F = I + grad u from the reference-configuration
// shape gradients, its SL(3) retraction F_sl3 = exp(log F) / det^(1/3)
// (CORE/lie_operator.cpp:300, methods in fm_lie.cuh), the Neo-Hookean
// Mandel stress of F_sl3 (neo_hookean_response, :79-129), and the monitor's
// count of |det F_sl3 - 1| > 1e-8 (RuntimeInvariantMonitor::check_sl3_element,
// CORE/lie_operator.hpp:244-251).  The J2 return the engine calls next
// (:2109) is an empty stub in the reference and is not run.
//
// One thread per tet, FP64 throughout; the element is skipped (state left
// as it was) when the reference Jacobian's |det| < 1e-30, as the reference
// skips it.  Under node jitter the split's sliver tets have a tiny but
// nonzero reference Jacobian: the reference updates them, and their F can
// overflow; such states are counted (not flagged as a solver error).  The
// reference passes an uninitialized J to
// neo_hookean_response here (a local declared and never set, :2784-2785);
// this kernel passes det F_sl3 (1 up to rounding), the value the retraction
// defines.
#include "fm_kernels.hpp"
#include "fm_lie.cuh"

namespace fm {

namespace {

// matrix_3x3_inv of the engine (:52-71): |det| < 1e-30 gives the zero
// matrix with 1e30 on the diagonal
__device__ __forceinline__ void inv3_engine(const double A[9], double R[9]) {
    const double d = A[0] * (A[4] * A[8] - A[7] * A[5]) - A[3] * (A[1] * A[8] - A[7] * A[2]) +
                     A[6] * (A[1] * A[5] - A[4] * A[2]);
    if (fabs(d) < 1e-30) {
#pragma unroll
        for (int i = 0; i < 9; ++i) R[i] = (i % 4 == 0) ? 1e30 : 0.0;
        return;
    }
    const double id = 1.0 / d;
    R[0] = (A[4] * A[8] - A[7] * A[5]) * id;
    R[1] = -(A[1] * A[8] - A[7] * A[2]) * id;
    R[2] = (A[1] * A[5] - A[4] * A[2]) * id;
    R[3] = -(A[3] * A[8] - A[6] * A[5]) * id;
    R[4] = (A[0] * A[8] - A[6] * A[2]) * id;
    R[5] = -(A[0] * A[5] - A[3] * A[2]) * id;
    R[6] = (A[3] * A[7] - A[6] * A[4]) * id;
    R[7] = -(A[0] * A[7] - A[6] * A[1]) * id;
    R[8] = (A[0] * A[4] - A[3] * A[1]) * id;
}

// neo_hookean_response (:79-129) in the reference's operation order:
// C = F^T F, S = mu (I - C^-1) + lam ln(max(J, 0.01)) C^-1, M = C S, Voigt
// with sqrt2 = 1.41421356237 on the shear entries
__device__ __forceinline__ void nh_response(const double F[9], double mu, double lam, double J,
                                            double sig[6]) {
    double C[9];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            double s = 0.0;
#pragma unroll
            for (int k = 0; k < 3; ++k) s += F[k * 3 + i] * F[k * 3 + j];
            C[i * 3 + j] = s;
        }
    double Ci[9];
    inv3_engine(C, Ci);
    const double lnJ = log(J < 0.01 ? 0.01 : J);
    double S[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) S[i] = mu * ((i % 4 == 0 ? 1.0 : 0.0) - Ci[i]) + lam * lnJ * Ci[i];
    double M[9];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            double s = 0.0;
#pragma unroll
            for (int k = 0; k < 3; ++k) s += C[i * 3 + k] * S[k * 3 + j];
            M[i * 3 + j] = s;
        }
    const double r2 = 1.41421356237;
    sig[0] = M[0];
    sig[1] = M[4];
    sig[2] = M[8];
    sig[3] = M[1] * r2;
    sig[4] = M[2] * r2;
    sig[5] = M[5] * r2;
}

__global__ void __launch_bounds__(128)
    k_element_states(MeshDev m, const double* __restrict__ u, double nu, double* __restrict__ Fst,
                     double* __restrict__ stress, unsigned* __restrict__ counts) {
    unsigned bad = 0, nonfinite = 0;
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < m.n_elems;
         e += gridDim.x * blockDim.x) {
        const uint4 c = m.conn[e];
        const uint32_t cn[4] = {c.x & 0x7fffffffu, c.y, c.z, c.w};
        double x[4][3], ue[4][3];
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                x[a][d] = __ldg(m.xyz + 3 * (size_t)cn[a] + d);
                ue[a][d] = __ldg(u + 3 * (size_t)cn[a] + d);
            }
        double J[9];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            J[d * 3 + 0] = x[1][d] - x[0][d];
            J[d * 3 + 1] = x[2][d] - x[0][d];
            J[d * 3 + 2] = x[3][d] - x[0][d];
        }
        double Ji[9];
        inv3_engine(J, Ji);
        const double dJ = J[0] * (J[4] * J[8] - J[7] * J[5]) - J[3] * (J[1] * J[8] - J[7] * J[2]) +
                          J[6] * (J[1] * J[5] - J[4] * J[2]);
        if (fabs(dJ) < 1e-30) continue;
        // dN_a = Jinv^T dN_xi(a), dN_xi = (-1,-1,-1), e1, e2, e3
        const double xi[4][3] = {{-1, -1, -1}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
        double dN[4][3];
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                double s = 0.0;
#pragma unroll
                for (int j = 0; j < 3; ++j) s += Ji[j * 3 + i] * xi[a][j];
                dN[a][i] = s;
            }
        double g[9];
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                double s = 0.0;
#pragma unroll
                for (int a = 0; a < 4; ++a) s += ue[a][i] * dN[a][j];
                g[i * 3 + j] = s;
            }
        lie::M3 F;
#pragma unroll
        for (int i = 0; i < 9; ++i) F.a[i] = (i % 4 == 0) ? 1.0 + g[i] : g[i];
        const lie::M3 Fs = lie::sl3_retraction(F);
        double mu, lam;
        if (m.mat_mode == 2) {
            mu = __ldg(m.m0 + e);
            lam = __ldg(m.m1 + e);
        } else if (m.mat_mode == 1) {
            // mu, lambda from (E_e, nu) as neo_hookean_response forms them
            const double E = __ldg(m.m0 + e);
            mu = E / (2.0 * (1.0 + nu));
            lam = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
        } else {
            mu = m.mu_s;
            lam = m.lam_s;
        }
        const double dF = lie::det(Fs);
        double sig[6];
        nh_response(Fs.a, mu, lam, dF, sig);
        double chk = dF;
#pragma unroll
        for (int i = 0; i < 9; ++i) Fst[9 * (size_t)e + i] = Fs.a[i];
#pragma unroll
        for (int i = 0; i < 6; ++i) {
            stress[6 * (size_t)e + i] = sig[i];
            chk += sig[i];
        }
        if (!isfinite(chk)) ++nonfinite;
        if (fabs(dF - 1.0) > 1.0e-8) ++bad;
    }
    bad = __reduce_add_sync(kFull, bad);
    nonfinite = __reduce_add_sync(kFull, nonfinite);
    if ((threadIdx.x & 31) == 0) {
        if (bad) atomicAdd(counts, bad);
        if (nonfinite) atomicAdd(counts + 1, nonfinite);
    }
}

}  // namespace

void launch_element_states(const MeshDev& m, const double* u, double nu, double* F,
                           double* stress, unsigned* counts, cudaStream_t s) {
    if (!m.n_elems) return;
    unsigned grid = (m.n_elems + 127) / 128;
    if (grid > 148u * 16u) grid = 148u * 16u;
    k_element_states<<<grid, 128, 0, s>>>(m, u, nu, F, stress, counts);
}

}  // namespace fm
