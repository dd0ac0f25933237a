// fm_kernels.cu — sm_100a kernels of the FlexMesh hot path.
//
// Assembly: one warp owns one node and writes that node's three CSR rows
// exactly once (no atomics, deterministic).  Lanes first evaluate the
// node's incident tets (kinematics, Neo-Hookean stress, tangent scalars) in
// FP64, stage the per-tet data in shared memory, then each lane forms the
// 3x3 block of one neighbour node by summing over the tets that contain the
// edge (node, neighbour).  The diagonal block is minus the sum of the
// off-diagonal blocks (rows of every element tangent sum to zero because
// the shape gradients do).
//
// Solvers: SpMV over the node-block pattern, and sync-free ILU(0) and
// triangular solves: a persistent grid walks the rows in a topological
// order (dependency levels); each row waits on its dependencies' release
// flags with a bounded spin, so there is no per-level launch or barrier.
#include <algorithm>
#include <cstdio>

#include "fm_kernels.hpp"

namespace fm {

// ===========================================================================
// Assembly
// ===========================================================================
constexpr int kAsmWarps = 8;

template <typename KT>
struct AsmStage {
    KT d[32][12];     // shape gradients of the 4 nodes of incident tet l; after
                      // phase 2 reused as the [lane][9] gather of the row blocks
    KT fI[32][3];     // vol M dN_owner of tet l (force, and geometric term)
    KT vabm[32][3];   // vol*a, vol*b, vol*mu (tangent scalars)
    double f64[3][32];  // FP64 node-force contributions of the incident tets
    uint32_t pos[32]; // 4 x u8: position of each tet node in the owner's neighbour list
};

__device__ __forceinline__ int find_sorted(const uint32_t* a, int len, uint32_t key) {
    int lo = 0, hi = len - 1;
    while (lo <= hi) {
        const int mid = (lo + hi) >> 1;
        const uint32_t v = a[mid];
        if (v == key) return mid;
        if (v < key) lo = mid + 1;
        else hi = mid - 1;
    }
    return -1;
}

__device__ __forceinline__ int byte_index(uint32_t packed, uint32_t key) {
    // which of the 4 bytes equals key (0..3), -1 if none
    if ((packed & 0xffu) == key) return 0;
    if (((packed >> 8) & 0xffu) == key) return 1;
    if (((packed >> 16) & 0xffu) == key) return 2;
    if ((packed >> 24) == key) return 3;
    return -1;
}

// Element record (AoS, 16-byte multiple): vertex forces vol M dN_a (FP64,
// 4x3), shape gradients dN_a (4x3) and tangent scalars vol a, vol b, vol mu
// in the tangent's type, and an activity mark (0: skipped or degenerate).
template <typename KT>
struct ElemRec;
template <>
struct __align__(16) ElemRec<double> {
    double f[12];
    double d[12];
    double s[3];
    double active;
};
template <>
struct __align__(16) ElemRec<float> {
    double f[12];
    float d[12];
    float s[3];
    float active;
};
static_assert(sizeof(ElemRec<double>) <= kElemRecBytes && sizeof(ElemRec<double>) % 16 == 0, "");
static_assert(sizeof(ElemRec<float>) <= kElemRecBytes && sizeof(ElemRec<float>) % 16 == 0, "");

// 16-byte stores of a whole record from registers
__device__ __forceinline__ void store_rec(ElemRec<double>* dst, const ElemRec<double>& r) {
    double2* f = reinterpret_cast<double2*>(dst->f);
    double2* d = reinterpret_cast<double2*>(dst->d);
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        f[i] = make_double2(r.f[2 * i], r.f[2 * i + 1]);
        d[i] = make_double2(r.d[2 * i], r.d[2 * i + 1]);
    }
    double2* t = reinterpret_cast<double2*>(dst->s);
    t[0] = make_double2(r.s[0], r.s[1]);
    t[1] = make_double2(r.s[2], r.active);
}
__device__ __forceinline__ void store_rec(ElemRec<float>* dst, const ElemRec<float>& r) {
    double2* f = reinterpret_cast<double2*>(dst->f);
#pragma unroll
    for (int i = 0; i < 6; ++i) f[i] = make_double2(r.f[2 * i], r.f[2 * i + 1]);
    float4* d = reinterpret_cast<float4*>(dst->d);
#pragma unroll
    for (int i = 0; i < 3; ++i) d[i] = make_float4(r.d[4 * i], r.d[4 * i + 1], r.d[4 * i + 2], r.d[4 * i + 3]);
    *reinterpret_cast<float4*>(dst->s) = make_float4(r.s[0], r.s[1], r.s[2], r.active);
}

// One tet of the element pass: kinematics, Mandel stress, the four vertex
// forces (FP64) and, with_k, the tangent scalars and shape gradients in the
// tangent's type, stored as one 16-byte-aligned record.  Returns the flags.
template <typename KT>
__device__ __forceinline__ unsigned asm_element(const MeshDev& m, const double* __restrict__ u,
                                                uint32_t e, ElemRec<KT>* dst_rec, int with_k) {
    unsigned flags = 0;
    uint4 c = m.conn[e];
    const bool active = !(c.x & 0x80000000u);
    c.x &= 0x7fffffffu;
    const uint32_t cn[4] = {c.x, c.y, c.z, c.w};
    ElemRec<KT> r;
#pragma unroll
    for (int i = 0; i < 12; ++i) {
        r.f[i] = 0.0;
        r.d[i] = KT(0);
    }
    r.s[0] = r.s[1] = r.s[2] = KT(0);
    r.active = KT(0);
    if (active) {
        double x[12], ue[12];
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                x[3 * a + d] = __ldg(m.xyz + 3 * (size_t)cn[a] + d);
                ue[3 * a + d] = __ldg(u + 3 * (size_t)cn[a] + d);
            }
        TetKin k;
        if (tet_kinematics(x, ue, k)) {
            double mu, lam;
            material_of(m.mat_mode, m.m0, m.m1, e, m.mu_s, m.lam_s, m.c_mu, m.c_lam, mu, lam);
            const Mandel M = mandel_stress(k.F, k.J, mu, lam);
            double fs = 0.0;
#pragma unroll
            for (int a = 0; a < 4; ++a) {
                const double* dI = k.d[a];
                r.f[3 * a + 0] = k.vol * (M.m00 * dI[0] + M.m01 * dI[1] + M.m02 * dI[2]);
                r.f[3 * a + 1] = k.vol * (M.m01 * dI[0] + M.m11 * dI[1] + M.m12 * dI[2]);
                r.f[3 * a + 2] = k.vol * (M.m02 * dI[0] + M.m12 * dI[1] + M.m22 * dI[2]);
                fs += r.f[3 * a] + r.f[3 * a + 1] + r.f[3 * a + 2];
            }
            if (!(k.J > 0.0)) flags |= FM_FLAG_INVERTED;
            if (k.J < kJSafe) flags |= FM_FLAG_J_CLAMPED;
            if (!isfinite(fs)) flags |= FM_FLAG_NONFINITE;
            if (with_k) {
                double a, b;
                tangent_ab(mu, lam, k.J, M.lnJ, m.inv_cnu, a, b);
#pragma unroll
                for (int q = 0; q < 4; ++q)
#pragma unroll
                    for (int d = 0; d < 3; ++d) r.d[3 * q + d] = (KT)k.d[q][d];
                r.s[0] = (KT)(k.vol * a);
                r.s[1] = (KT)(k.vol * b);
                r.s[2] = (KT)(k.vol * mu);
                if (!isfinite(a + b)) flags |= FM_FLAG_NONFINITE;
            }
            r.active = KT(1);
        }
    }
    store_rec(dst_rec, r);
    return flags;
}

// Element pass: one thread per tet.  with_k = 0 (residual only) skips the
// tangent scalars and gradients.
template <typename KT>
__global__ void __launch_bounds__(128, 4)
    k_asm_elements(MeshDev m, const double* __restrict__ u, ElemRec<KT>* __restrict__ rec,
                   int with_k, unsigned* __restrict__ status) {
    unsigned flags = 0;
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < m.n_elems;
         e += gridDim.x * blockDim.x)
        flags |= asm_element<KT>(m, u, e, rec + e, with_k);
    if (flags) raise_flag(status, flags);
}

// Node pass for one node: one warp owns it.  Lane l < mi stages incident
// tet l's record (gradients, the owner's vertex force, tangent scalars) in
// shared memory; lane k then forms block (n, nbr[k]).
template <typename KT>
__device__ __forceinline__ void asm_node(const MeshDev& m, const ElemRec<KT>* __restrict__ rec,
                                         uint32_t n, KT* __restrict__ K,
                                         double* __restrict__ f, double* __restrict__ R,
                                         int apply_bc, AsmStage<KT>& S, int lane) {

    const uint32_t nb0 = m.nbr_ptr[n];
    const int deg = (int)(m.nbr_ptr[n + 1] - nb0);
    const uint32_t e0 = m.inc_ptr[n];
    const int mi = (int)(m.inc_ptr[n + 1] - e0);
    const uint32_t my_nbr = lane < deg ? __ldg(m.nbr + nb0 + lane) : 0xffffffffu;
    const int self_k = __ffs(__ballot_sync(kFull, my_nbr == n)) - 1;
    // edge lists of the tangent blocks: structural, built on the host
    const uint32_t my_members = (K != nullptr && lane < deg) ? __ldg(m.nbr_members + nb0 + lane) : 0u;

    double fi0 = 0.0, fi1 = 0.0, fi2 = 0.0;
    uint32_t packed = 0xffffffffu;
    if (lane < mi) {
        const uint32_t e = __ldg(m.inc + e0 + lane);
        packed = __ldg(m.inc_pos + e0 + lane);
        const ElemRec<KT>& r = rec[e];
        const bool act = r.active != KT(0);
        if (act) {
            const int il = byte_index(packed, (uint32_t)self_k);
            fi0 = r.f[3 * il];
            fi1 = r.f[3 * il + 1];
            fi2 = r.f[3 * il + 2];
        }
        if (K != nullptr) {
            // an inactive tet (degenerate at this state) stays in the edge
            // lists with zero data: it adds exact zeros
#pragma unroll
            for (int q = 0; q < 12; ++q) S.d[lane][q] = act ? r.d[q] : KT(0);
            S.fI[lane][0] = (KT)fi0;
            S.fI[lane][1] = (KT)fi1;
            S.fI[lane][2] = (KT)fi2;
            S.vabm[lane][0] = act ? r.s[0] : KT(0);
            S.vabm[lane][1] = act ? r.s[1] : KT(0);
            S.vabm[lane][2] = act ? r.s[2] : KT(0);
        }
    }
    S.pos[lane] = packed;
    S.f64[0][lane] = fi0;
    S.f64[1][lane] = fi1;
    S.f64[2][lane] = fi2;
    __syncwarp();

    // internal force of the node: lane p < 3 sums component p over the
    // incident tets in ascending element order (deterministic).  Shared
    // gathers replace FP64 shuffle trees, which are slow after divergence.
    if (lane < 3) {
        double fv = 0.0;
        for (int l = 0; l < mi; ++l) fv += S.f64[lane][l];
        const uint32_t row = 3 * n + lane;
        if (f) f[row] = fv;
        if (R) R[row] = (m.mask && m.mask[row]) ? 0.0 : -fv;
    }
    if (K == nullptr) return;
    __syncwarp();

    // phase 2: lane k forms block (n, nbr[k]) from the tets on that edge
    KT acc[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) acc[q] = KT(0);
    if (lane < deg && lane != self_k) {
        uint32_t members = my_members;
        while (members) {
            const int l = __ffs(members) - 1;
            members &= members - 1;
            const uint32_t pk = S.pos[l];
            const int j = byte_index(pk, (uint32_t)lane);
            const int il = byte_index(pk, (uint32_t)self_k);
            tangent_block_acc<KT>(&S.d[l][3 * il], &S.d[l][3 * j], S.fI[l], S.vabm[l][0],
                                  S.vabm[l][1], S.vabm[l][2], acc);
        }
    }
    // diagonal block = - sum of off-diagonal blocks of the row block: lane
    // q < 9 sums entry q over the neighbour lanes (fixed order)
    __syncwarp();
    KT* red = &S.d[0][0];
#pragma unroll
    for (int q = 0; q < 9; ++q) red[9 * lane + q] = acc[q];
    __syncwarp();
    if (lane < 9) {
        KT s = KT(0);
        for (int l = 0; l < deg; ++l) s += red[9 * l + lane];
        red[9 * self_k + lane] = -s;
    }
    __syncwarp();
    if (lane == self_k) {
#pragma unroll
        for (int q = 0; q < 9; ++q) acc[q] = red[9 * self_k + q];
    }
    if (lane < deg) {
        const uint32_t col0 = 3 * my_nbr;
#pragma unroll
        for (int p = 0; p < 3; ++p) {
            const uint32_t row = 3 * n + p;
            const size_t base = 9 * (size_t)nb0 + 3 * (size_t)p * deg + 3 * lane;
            const bool mrow = apply_bc && m.mask && m.mask[row];
#pragma unroll
            for (int q = 0; q < 3; ++q) {
                KT v = acc[3 * p + q];
                if (apply_bc && m.mask && (mrow || m.mask[col0 + q]))
                    v = (row == col0 + q) ? KT(1) : KT(0);
                K[base + q] = v;
            }
        }
    }
}

// CTAs per SM: the FP64 pass fits 64 registers for four without spilling
// (32 resident warps instead of 24: 0.784 -> 0.733 ms at 64^3), the FP32
// pass 40 for six (0.540 -> 0.531 ms).
template <typename KT>
__global__ void __launch_bounds__(kAsmWarps * 32, sizeof(KT) == 4 ? 6 : 4)
    k_assemble(MeshDev m, const ElemRec<KT>* __restrict__ rec, KT* __restrict__ K,
               double* __restrict__ f, double* __restrict__ R, int apply_bc,
               unsigned* __restrict__ status) {
    (void)status;
    __shared__ AsmStage<KT> stage[kAsmWarps];
    const int lane = threadIdx.x & 31;
    const int wi = threadIdx.x >> 5;
    const uint32_t n = blockIdx.x * kAsmWarps + wi;
    if (n >= m.n_nodes) return;  // uniform per warp
    asm_node<KT>(m, rec, n, K, f, R, apply_bc, stage[wi], lane);
}

template <typename KT>
static void launch_assemble_t(const MeshDev& m, const double* u, KT* K, double* f, double* R,
                              int apply_bc, unsigned* status, cudaStream_t s) {
    if (m.n_nodes == 0) return;
    ElemRec<KT>* rec = static_cast<ElemRec<KT>*>(m.elem_rec);
    if (m.n_elems) {
        unsigned ge = (m.n_elems + 127) / 128;
        if (ge > 148u * 32u) ge = 148u * 32u;
        k_asm_elements<KT><<<ge, 128, 0, s>>>(m, u, rec, K != nullptr, status);
    }
    const unsigned grid = (m.n_nodes + kAsmWarps - 1) / kAsmWarps;
    k_assemble<KT><<<grid, kAsmWarps * 32, 0, s>>>(m, rec, K, f, R, apply_bc, status);
}
void launch_assemble(const MeshDev& m, const double* u, double* K, double* f, double* R,
                     int apply_bc, unsigned* status, cudaStream_t s) {
    launch_assemble_t<double>(m, u, K, f, R, apply_bc, status, s);
}
void launch_assemble(const MeshDev& m, const double* u, float* K, double* f, double* R,
                     int apply_bc, unsigned* status, cudaStream_t s) {
    launch_assemble_t<float>(m, u, K, f, R, apply_bc, status, s);
}

// Full element tangent/force of one tet into Ke (row-major 12x12), fe.
// Returns false for a degenerate tet (outputs zero).
__device__ __forceinline__ bool element_full(const double x[12], const double ue[12], double mu,
                                             double lam, double inv_cnu, double* Ke, double* fe,
                                             size_t ks, unsigned& flags) {
    TetKin k;
    if (!tet_kinematics(x, ue, k)) {
        for (int q = 0; q < 144; ++q) Ke[q * ks] = 0.0;
        for (int q = 0; q < 12; ++q) fe[q] = 0.0;
        return false;
    }
    const Mandel M = mandel_stress(k.F, k.J, mu, lam);
    double a, b;
    tangent_ab(mu, lam, k.J, M.lnJ, inv_cnu, a, b);
    const double va = k.vol * a, vb = k.vol * b, vm = k.vol * mu;
    double fI[4][3];
    for (int i = 0; i < 4; ++i) {
        const double* d = k.d[i];
        fI[i][0] = k.vol * (M.m00 * d[0] + M.m01 * d[1] + M.m02 * d[2]);
        fI[i][1] = k.vol * (M.m01 * d[0] + M.m11 * d[1] + M.m12 * d[2]);
        fI[i][2] = k.vol * (M.m02 * d[0] + M.m12 * d[1] + M.m22 * d[2]);
        for (int p = 0; p < 3; ++p) fe[3 * i + p] = fI[i][p];
    }
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) {
            double acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
            tangent_block_acc<double>(k.d[i], k.d[j], fI[i], va, vb, vm, acc);
            for (int p = 0; p < 3; ++p)
                for (int q = 0; q < 3; ++q) Ke[((i * 3 + p) * 12 + j * 3 + q) * ks] = acc[3 * p + q];
        }
    if (!(k.J > 0.0)) flags |= FM_FLAG_INVERTED;
    if (k.J < kJSafe) flags |= FM_FLAG_J_CLAMPED;
    if (!isfinite(fe[0] + fe[4] + fe[8] + a + b)) flags |= FM_FLAG_NONFINITE;
    return true;
}

__global__ void k_elements(uint32_t n, const double* __restrict__ x, const double* __restrict__ u,
                           const double* __restrict__ E, double nu, double* __restrict__ K,
                           double* __restrict__ f, unsigned* status) {
    const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    double xe[12], ue[12];
    for (int q = 0; q < 12; ++q) {
        xe[q] = x[12 * (size_t)e + q];
        ue[q] = u[12 * (size_t)e + q];
    }
    const double Ee = E[e];
    const double mu = Ee / (2.0 * (1.0 + nu));
    const double lam = Ee * nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
    const double one_m = 1.0 - 2.0 * nu;
    const double inv_cnu = 1.0 / (one_m < 0.1 ? 0.1 : one_m);
    unsigned flags = 0;
    element_full(xe, ue, mu, lam, inv_cnu, K + 144 * (size_t)e, f + 12 * (size_t)e, 1, flags);
    if (flags) raise_flag(status, flags);
}

void launch_elements(uint32_t n, const double* x, const double* u, const double* E, double nu,
                     double* K, double* f, unsigned* status, cudaStream_t s) {
    if (!n) return;
    k_elements<<<(n + 127) / 128, 128, 0, s>>>(n, x, u, E, nu, K, f, status);
}

// Reference-pattern scatter: thread per tet, slot map with -1 for entries
// the reference's defective pattern lacks (last duplicate wins in the map).
__global__ void k_assemble_slotmap(MeshDev m, const double* __restrict__ u,
                                   const int32_t* __restrict__ slot, double* K, double* f,
                                   double* Ke_scratch, unsigned* status) {
    const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= m.n_elems) return;
    uint4 c = m.conn[e];
    if (c.x & 0x80000000u) return;
    const uint32_t cn[4] = {c.x, c.y, c.z, c.w};
    double x[12], ue[12];
    for (int a = 0; a < 4; ++a)
        for (int d = 0; d < 3; ++d) {
            x[3 * a + d] = m.xyz[3 * (size_t)cn[a] + d];
            ue[3 * a + d] = u[3 * (size_t)cn[a] + d];
        }
    double mu, lam;
    material_of(m.mat_mode, m.m0, m.m1, e, m.mu_s, m.lam_s, m.c_mu, m.c_lam, mu, lam);
    double fe[12];
    unsigned flags = 0;
    double* Ke = Ke_scratch + (size_t)e;  // strided by n_elems
    if (!element_full(x, ue, mu, lam, m.inv_cnu, Ke, fe, m.n_elems, flags)) return;
    if (flags) raise_flag(status, flags);
    for (int q = 0; q < 144; ++q) {
        const int32_t sl = slot[144 * (size_t)e + q];
        if (sl >= 0) atomicAdd(K + sl, Ke[(size_t)q * m.n_elems]);
    }
    for (int a = 0; a < 4; ++a)
        for (int d = 0; d < 3; ++d) atomicAdd(f + 3 * (size_t)cn[a] + d, fe[3 * a + d]);
}

void launch_assemble_slotmap(const MeshDev& m, const double* u, const int32_t* slot, double* K,
                             double* f, double* Ke_scratch, unsigned* status, cudaStream_t s) {
    if (!m.n_elems) return;
    k_assemble_slotmap<<<(m.n_elems + 127) / 128, 128, 0, s>>>(m, u, slot, K, f, Ke_scratch,
                                                               status);
}

// ===========================================================================
// SpMV
// ===========================================================================
constexpr int kSpmvBlocks = 148 * 8;

template <typename T>
__global__ void __launch_bounds__(256)
    k_spmv_nodes(uint32_t nn, const uint32_t* __restrict__ nbr_ptr,
                 const uint32_t* __restrict__ nbr, const T* __restrict__ val,
                 const T* __restrict__ x, T* __restrict__ y, T* partials, unsigned* counter,
                 double* dot) {
    const int lane = threadIdx.x & 31;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    T dsum = T(0);
    for (uint32_t n = warp; n < nn; n += nwarps) {
        const uint32_t nb0 = nbr_ptr[n];
        const int deg = (int)(nbr_ptr[n + 1] - nb0);
        const uint32_t my_nbr = lane < deg ? __ldg(nbr + nb0 + lane) : 0u;
        const T* v = val + 9 * (size_t)nb0;
        const int rl = 3 * deg;
        T s[3] = {T(0), T(0), T(0)};
        for (int i0 = 0; i0 < rl; i0 += 32) {
            const int idx = i0 + lane;
            const int k = idx < rl ? idx / 3 : 0;
            const uint32_t cn = __shfl_sync(kFull, my_nbr, k);
            if (idx < rl) {
                const T xv = __ldg(x + 3 * (size_t)cn + (idx - 3 * k));
#pragma unroll
                for (int p = 0; p < 3; ++p) s[p] += __ldg(v + (size_t)p * rl + idx) * xv;
            }
        }
#pragma unroll
        for (int p = 0; p < 3; ++p) s[p] = warp_sum(s[p]);
        if (lane < 3) {
            const T yv = lane == 0 ? s[0] : (lane == 1 ? s[1] : s[2]);
            y[3 * (size_t)n + lane] = yv;
            if (dot) dsum += yv * x[3 * (size_t)n + lane];
        }
    }
    if (dot) {
        __shared__ T sbuf[32];
        const T bt = block_sum(dsum, sbuf);
        grid_reduce_finish<T>(bt, partials, counter, [&](T total) { *dot = (double)total; });
    }
}

template <typename T>
void launch_spmv_nodes(uint32_t n_nodes, const uint32_t* nbr_ptr, const uint32_t* nbr,
                       const T* val, const T* x, T* y, T* partials, unsigned* counter,
                       double* dot, cudaStream_t s) {
    k_spmv_nodes<T><<<kSpmvBlocks, 256, 0, s>>>(n_nodes, nbr_ptr, nbr, val, x, y, partials,
                                                 counter, dot);
}

template <typename T>
__global__ void __launch_bounds__(256)
    k_spmv_csr(uint32_t n, const uint32_t* __restrict__ rp, const uint32_t* __restrict__ ci,
               const T* __restrict__ val, const T* __restrict__ x, T* __restrict__ y,
               T* partials, unsigned* counter, double* dot) {
    const int lane = threadIdx.x & 31;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    T dsum = T(0);
    for (uint32_t i = warp; i < n; i += nwarps) {
        T s = T(0);
        for (uint32_t k = rp[i] + lane; k < rp[i + 1]; k += 32) s += __ldg(val + k) * __ldg(x + ci[k]);
        s = warp_sum(s);
        if (lane == 0) {
            y[i] = s;
            if (dot) dsum += s * x[i];
        }
    }
    if (dot) {
        __shared__ T sbuf[32];
        const T bt = block_sum(dsum, sbuf);
        grid_reduce_finish<T>(bt, partials, counter, [&](T total) { *dot = (double)total; });
    }
}

template <typename T>
void launch_spmv_csr(uint32_t n, const uint32_t* rp, const uint32_t* ci, const T* val, const T* x,
                     T* y, T* partials, unsigned* counter, double* dot, cudaStream_t s) {
    k_spmv_csr<T><<<kSpmvBlocks, 256, 0, s>>>(n, rp, ci, val, x, y, partials, counter, dot);
}

// ===========================================================================
// Sync-free ILU(0) and triangular solves (scalar CSR rows, warp per row)
// ===========================================================================
constexpr int kSfWarps = 8;  // warps per block of the persistent kernels

// Row i of ILU(0), IKJ form in natural order, which performs the same
// subtractions in the same order as the reference's Doolittle loop
// (FEM/adaptive_fem_engine.hpp:327-466):
//   for each lower column c of row i, ascending:  l = w_c / d_c,
//     w_j -= l U(c,j) for every j > c of row c present in row i,
//     and u_ii -= l U(c,i);
//   u_ii perturbed by +-1e-8 when |u_ii| < 1e-12.
// The diagonal slot keeps a_ii (the reference's U_val does); pivots go to diag.
template <typename T>
__global__ void __launch_bounds__(kSfWarps * 32)
    k_ilu0_csr(CsrDev A, const T* __restrict__ a,
               T* __restrict__ lu, T* __restrict__ diag, unsigned* __restrict__ done,
               unsigned epoch, unsigned* __restrict__ status) {
    extern __shared__ unsigned char smem_raw[];
    const int lane = threadIdx.x & 31, wi = threadIdx.x >> 5;
    const uint32_t stride = (A.max_row + 1) & ~1u;
    uint32_t* cols = reinterpret_cast<uint32_t*>(smem_raw) + wi * stride;
    T* w = reinterpret_cast<T*>(reinterpret_cast<uint32_t*>(smem_raw) + kSfWarps * stride) +
           wi * stride;
    __shared__ T s_uii[kSfWarps];
    const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t W = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t t = gw; t < A.n; t += W) {
        const uint32_t i = A.fwd_order[t];
        const uint32_t b = A.rp[i];
        const int len = (int)(A.rp[i + 1] - b);
        const int dp = (int)(A.dpos[i] - b);
        for (int q = lane; q < len; q += 32) {
            cols[q] = A.ci[b + q];
            w[q] = a[b + q];
        }
        __syncwarp();
        const bool has_diag = dp < len && cols[dp] == i;
        bool ok = true;
        for (int q = lane; q < dp; q += 32) ok &= wait_flag(done + cols[q], epoch, status);
        ok = __all_sync(kFull, ok);
        if (lane == 0) s_uii[wi] = has_diag ? w[dp] : T(0);
        __syncwarp();
        if (ok) {
            for (int q = 0; q < dp; ++q) {
                const uint32_t c = cols[q];
                const T l = w[q] / ld_cg(diag + c);
                const uint32_t ue = A.rp[c + 1];
                for (uint32_t mm = A.upos[c] + lane; mm < ue; mm += 32) {
                    const uint32_t j = A.ci[mm];
                    const T uv = ld_cg(lu + mm);
                    if (j == i) {
                        s_uii[wi] -= l * uv;
                    } else {
                        const int p = find_sorted(cols + q + 1, len - q - 1, j);
                        if (p >= 0) w[q + 1 + p] -= l * uv;
                    }
                }
                __syncwarp();
                if (lane == 0) w[q] = l;
                __syncwarp();
            }
        }
        T uii = s_uii[wi];
        for (int q = lane; q < len; q += 32) lu[b + q] = w[q];
        if (lane == 0) {
            if (fabs((double)uii) < kPivotThreshold) {
                uii += (uii >= T(0) ? T(kPivotPerturb) : T(-kPivotPerturb));
                raise_flag(status, FM_FLAG_PIVOT);
            }
            if (!isfinite((double)uii)) raise_flag(status, FM_FLAG_NONFINITE);
            diag[i] = uii;
        }
        __threadfence();
        __syncwarp();
        if (lane == 0) st_release(done + i, epoch);
        __syncwarp();
    }
}

// z_i = r_i - sum_{c<i} L_ic z_c  (unit lower)
template <typename T>
__global__ void __launch_bounds__(kSfWarps * 32)
    k_trsv_lower_csr(CsrDev A, const T* __restrict__ lu, const T* __restrict__ r, T* z,
                     unsigned* __restrict__ done, unsigned epoch, unsigned* __restrict__ status) {
    const int lane = threadIdx.x & 31;
    const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t W = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t t = gw; t < A.n; t += W) {
        const uint32_t i = A.fwd_order[t];
        const uint32_t e = A.dpos[i];
        T s = T(0);
        for (uint32_t k = A.rp[i] + lane; k < e; k += 32) {
            const uint32_t c = A.ci[k];
            if (!wait_flag(done + c, epoch, status)) break;
            s += lu[k] * ld_cg(z + c);
        }
        s = warp_sum(s);
        if (lane == 0) {
            z[i] = r[i] - s;
            st_release(done + i, epoch);
        }
    }
}

// y_i = (z_i - sum_{c>i} U_ic y_c) / d_i
template <typename T>
__global__ void __launch_bounds__(kSfWarps * 32)
    k_trsv_upper_csr(CsrDev A, const T* __restrict__ lu,
                     const T* __restrict__ diag, const T* __restrict__ z, T* y,
                     unsigned* __restrict__ done, unsigned epoch, unsigned* __restrict__ status) {
    const int lane = threadIdx.x & 31;
    const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t W = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t t = gw; t < A.n; t += W) {
        const uint32_t i = A.bwd_order[t];
        const uint32_t e = A.rp[i + 1];
        T s = T(0);
        for (uint32_t k = A.upos[i] + lane; k < e; k += 32) {
            const uint32_t c = A.ci[k];
            if (!wait_flag(done + c, epoch, status)) break;
            s += lu[k] * ld_cg(y + c);
        }
        s = warp_sum(s);
        if (lane == 0) {
            y[i] = (z[i] - s) / diag[i];
            st_release(done + i, epoch);
        }
    }
}


static size_t ilu_smem_bytes(const CsrDev& A, size_t tsize) {
    const size_t stride = (A.max_row + 1) & ~1u;
    return kSfWarps * stride * (sizeof(uint32_t) + tsize);
}

template <typename T>
void launch_ilu0_csr(const CsrDev& A, const T* a_val, T* lu, T* diag, unsigned* done,
                     unsigned epoch, unsigned* status, int grid, cudaStream_t s) {
    if (!A.n) return;
    k_ilu0_csr<T><<<grid, kSfWarps * 32, ilu_smem_bytes(A, sizeof(T)), s>>>(A, a_val, lu, diag,
                                                                             done, epoch, status);
}
template <typename T>
void launch_trsv_lower_csr(const CsrDev& A, const T* lu, const T* r, T* z, unsigned* done,
                           unsigned epoch, unsigned* status, int grid, cudaStream_t s) {
    if (!A.n) return;
    k_trsv_lower_csr<T><<<grid, kSfWarps * 32, 0, s>>>(A, lu, r, z, done, epoch, status);
}
template <typename T>
void launch_trsv_upper_csr(const CsrDev& A, const T* lu, const T* diag, const T* z, T* y,
                           unsigned* done, unsigned epoch, unsigned* status, int grid,
                           cudaStream_t s) {
    if (!A.n) return;
    k_trsv_upper_csr<T><<<grid, kSfWarps * 32, 0, s>>>(A, lu, diag, z, y, done, epoch, status);
}

// All blocks of a sync-free kernel must be resident at once (rows wait on
// rows handled by other blocks), so the grid is the occupancy limit times
// the SM count.
template <typename K>
static int resident_grid(K kernel, int device, size_t smem) {
    int sms = 0, per_sm = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kSfWarps * 32, smem);
    if (per_sm < 1) per_sm = 1;
    return sms * per_sm;
}
int persistent_grid_ilu0_csr(int device, bool fp32, const CsrDev& A) {
    return fp32 ? resident_grid(k_ilu0_csr<float>, device, ilu_smem_bytes(A, 4))
                : resident_grid(k_ilu0_csr<double>, device, ilu_smem_bytes(A, 8));
}
int persistent_grid_trsv_csr(int device, bool fp32) {
    const int a = fp32 ? resident_grid(k_trsv_lower_csr<float>, device, 0)
                       : resident_grid(k_trsv_lower_csr<double>, device, 0);
    const int b = fp32 ? resident_grid(k_trsv_upper_csr<float>, device, 0)
                       : resident_grid(k_trsv_upper_csr<double>, device, 0);
    return a < b ? a : b;
}

// ===========================================================================
// Vector kernels (PCG and Newton)
// ===========================================================================
constexpr int kVecThreads = 256;

template <typename T>
__global__ void __launch_bounds__(kVecThreads)
    k_dot(uint32_t n, const T* __restrict__ x, const T* __restrict__ y, T* partials,
          unsigned* counter, double* out) {
    T s = T(0);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        s += x[i] * y[i];
    __shared__ T sbuf[32];
    const T bt = block_sum(s, sbuf);
    grid_reduce_finish<T>(bt, partials, counter, [&](T total) { *out = (double)total; });
}
template <typename T>
void launch_dot(uint32_t n, const T* x, const T* y, T* partials, unsigned* counter, double* out,
                cudaStream_t s) {
    k_dot<T><<<kRedBlocks, kVecThreads, 0, s>>>(n, x, y, partials, counter, out);
}

template <typename T>
__global__ void __launch_bounds__(kVecThreads)
    k_residual_init(uint32_t n, const T* __restrict__ b, T* __restrict__ r, T* partials,
                    unsigned* counter, double* rr) {
    T s = T(0);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += gridDim.x * blockDim.x) {
        const T v = b[i] - r[i];
        r[i] = v;
        s += v * v;
    }
    __shared__ T sbuf[32];
    const T bt = block_sum(s, sbuf);
    grid_reduce_finish<T>(bt, partials, counter, [&](T total) { *rr = (double)total; });
}
template <typename T>
void launch_residual_init(uint32_t n, const T* b, T* r, T* partials, unsigned* counter,
                          double* rr, cudaStream_t s) {
    k_residual_init<T><<<kRedBlocks, kVecThreads, 0, s>>>(n, b, r, partials, counter, rr);
}

// p = z; rz = r.z; bb = b.b.  Two sums share one pass (partials: 2 slots per block)
template <typename T>
__global__ void __launch_bounds__(kVecThreads)
    k_pcg_start(uint32_t n, const T* __restrict__ r, const T* __restrict__ z,
                const T* __restrict__ b, T* __restrict__ p, T* partials, unsigned* counter,
                DevScalars* sc) {
    T s1 = T(0), s2 = T(0);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += gridDim.x * blockDim.x) {
        const T zi = z[i];
        p[i] = zi;
        s1 += r[i] * zi;
        s2 += b[i] * b[i];
    }
    __shared__ T sbuf[32];
    const T b1 = block_sum(s1, sbuf);
    const T b2 = block_sum(s2, sbuf);
    grid_reduce_finish<T>(b1, partials, counter, [&](T total) {
        sc->rz_new = (double)total;
        sc->rz = (double)total;
    });
    grid_reduce_finish<T>(b2, partials + gridDim.x, counter + 1,
                          [&](T total) { sc->bb = (double)total; });
}
template <typename T>
void launch_pcg_start(uint32_t n, const T* r, const T* z, const T* b, T* p, T* partials,
                      unsigned* counter, DevScalars* sc, cudaStream_t s) {
    k_pcg_start<T><<<kRedBlocks, kVecThreads, 0, s>>>(n, r, z, b, p, partials, counter, sc);
}

// alpha = rz/pAp (current rz is rz_new); breakdown |pAp| < 1e-60 stops
// before touching x and r, as the reference breaks out (:1320).
template <typename T>
__global__ void __launch_bounds__(kVecThreads)
    k_pcg_update_xr(uint32_t n, const T* __restrict__ p, const T* __restrict__ Ap,
                    T* __restrict__ x, T* __restrict__ r, DevScalars* sc) {
    const double pAp = sc->pAp;
    if (fabs(pAp) < 1e-60) {
        if (blockIdx.x == 0 && threadIdx.x == 0) sc->stop = 1u;
        return;
    }
    const T alpha = (T)(sc->rz_new / pAp);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += gridDim.x * blockDim.x) {
        x[i] += alpha * p[i];
        r[i] -= alpha * Ap[i];
    }
}
template <typename T>
void launch_pcg_update_xr(uint32_t n, const T* p, const T* Ap, T* x, T* r, DevScalars* sc,
                          cudaStream_t s) {
    k_pcg_update_xr<T><<<kRedBlocks * 2, kVecThreads, 0, s>>>(n, p, Ap, x, r, sc);
}

// rz <- rz_new (old value kept for beta), rz_new <- r.z, relres
template <typename T>
__global__ void __launch_bounds__(kVecThreads)
    k_pcg_rz(uint32_t n, const T* __restrict__ r, const T* __restrict__ z, T* partials,
             unsigned* counter, DevScalars* sc) {
    T s = T(0);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += gridDim.x * blockDim.x)
        s += r[i] * z[i];
    __shared__ T sbuf[32];
    const T bt = block_sum(s, sbuf);
    grid_reduce_finish<T>(bt, partials, counter, [&](T total) {
        sc->rz = sc->rz_new;
        sc->rz_new = (double)total;
        const double bb = sc->bb > 1e-300 ? sc->bb : 1e-300;
        sc->relres = sqrt((double)total / bb);
    });
}
template <typename T>
void launch_pcg_rz(uint32_t n, const T* r, const T* z, T* partials, unsigned* counter,
                   DevScalars* sc, cudaStream_t s) {
    k_pcg_rz<T><<<kRedBlocks, kVecThreads, 0, s>>>(n, r, z, partials, counter, sc);
}

template <typename T>
__global__ void __launch_bounds__(kVecThreads)
    k_pcg_update_p(uint32_t n, const T* __restrict__ z, T* __restrict__ p, const DevScalars* sc) {
    const T beta = (T)(sc->rz_new / sc->rz);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += gridDim.x * blockDim.x)
        p[i] = z[i] + beta * p[i];
}
template <typename T>
void launch_pcg_update_p(uint32_t n, const T* z, T* p, DevScalars* sc, cudaStream_t s) {
    k_pcg_update_p<T><<<kRedBlocks * 2, kVecThreads, 0, s>>>(n, z, p, sc);
}

__global__ void k_set_bc_values(uint32_t n, const uint8_t* __restrict__ mask,
                                const double* __restrict__ val, double frac, double* u) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += gridDim.x * blockDim.x)
        if (mask[i]) u[i] = val ? frac * val[i] : 0.0;
}
void launch_set_bc_values(uint32_t n, const uint8_t* mask, const double* val, double frac,
                          double* u, cudaStream_t s) {
    k_set_bc_values<<<kRedBlocks, kVecThreads, 0, s>>>(n, mask, val, frac, u);
}

void launch_norm2(uint32_t n, const double* R, double* partials, unsigned* counter, double* out,
                  cudaStream_t s) {
    k_dot<double><<<kRedBlocks, kVecThreads, 0, s>>>(n, R, R, partials, counter, out);
}

__global__ void k_to_f32_scaled(uint32_t n, const double* __restrict__ R, double inv_scale,
                                float* __restrict__ b32, float* __restrict__ x32) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += gridDim.x * blockDim.x) {
        b32[i] = (float)(R[i] * inv_scale);
        if (x32) x32[i] = 0.0f;
    }
}

template <typename T>
__global__ void k_scale(uint32_t n, T* __restrict__ x, T g) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += gridDim.x * blockDim.x)
        x[i] *= g;
}
void launch_scale_f32(uint32_t n, float* x, float g, cudaStream_t s) {
    k_scale<float><<<kRedBlocks * 2, kVecThreads, 0, s>>>(n, x, g);
}
void launch_to_f32_scaled(uint32_t n, const double* R, double inv_scale, float* b32, float* x32,
                          cudaStream_t s) {
    k_to_f32_scaled<<<kRedBlocks * 2, kVecThreads, 0, s>>>(n, R, inv_scale, b32, x32);
}

__global__ void k_axpy_u(uint32_t n, const double* __restrict__ du, double* __restrict__ u) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += gridDim.x * blockDim.x)
        u[i] += du[i];
}
void launch_axpy_u(uint32_t n, const double* du, double* u, cudaStream_t s) {
    k_axpy_u<<<kRedBlocks * 2, kVecThreads, 0, s>>>(n, du, u);
}
__global__ void k_axpy_u_f32(uint32_t n, const float* __restrict__ du, double scale,
                             double* __restrict__ u) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += gridDim.x * blockDim.x)
        u[i] += scale * (double)du[i];
}
void launch_axpy_u_f32(uint32_t n, const float* du, double scale, double* u, cudaStream_t s) {
    k_axpy_u_f32<<<kRedBlocks * 2, kVecThreads, 0, s>>>(n, du, scale, u);
}

__global__ void k_f32_to_f64_scaled(uint32_t n, const float* __restrict__ x, double scale,
                                    double* __restrict__ y) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += gridDim.x * blockDim.x)
        y[i] = scale * (double)x[i];
}
void launch_f32_to_f64_scaled(uint32_t n, const float* x, double scale, double* y,
                              cudaStream_t s) {
    k_f32_to_f64_scaled<<<kRedBlocks * 2, kVecThreads, 0, s>>>(n, x, scale, y);
}
// y = u + alpha du
__global__ void k_axpby_trial(uint32_t n, const double* __restrict__ u, double alpha,
                              const double* __restrict__ du, double* __restrict__ y) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += gridDim.x * blockDim.x)
        y[i] = u[i] + alpha * du[i];
}
void launch_trial(uint32_t n, const double* u, double alpha, const double* du, double* y,
                  cudaStream_t s) {
    k_axpby_trial<<<kRedBlocks * 2, kVecThreads, 0, s>>>(n, u, alpha, du, y);
}

// One warp, one bounded wait on a flag that nothing sets: the wait gives up
// after the status word's wait limit and raises FM_FLAG_TIMEOUT.
__global__ void __launch_bounds__(32) k_wait_probe(const unsigned* flag, unsigned* status) {
    wait_flags_warp(flag, true, 1u, status, 0u);
}

void launch_wait_probe(const unsigned* flag, unsigned* status, cudaStream_t s) {
    k_wait_probe<<<1, 32, 0, s>>>(flag, status);
}

// Load-step predictor: v = frac*val - u on constrained DOFs (0 elsewhere),
// in FP64 and (optionally) FP32; ||v||^2 through the deterministic reduction.
__global__ void __launch_bounds__(kVecThreads)
    k_bc_increment(uint32_t n, const uint8_t* __restrict__ mask, const double* __restrict__ val,
                   double frac, const double* __restrict__ u, double* __restrict__ v,
                   float* __restrict__ v32, double* partials, unsigned* counter, double* out) {
    double s = 0.0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += gridDim.x * blockDim.x) {
        const double d = mask[i] ? (val ? frac * val[i] : 0.0) - u[i] : 0.0;
        v[i] = d;
        if (v32) v32[i] = (float)d;
        s += d * d;
    }
    __shared__ double sbuf[32];
    const double bt = block_sum(s, sbuf);
    grid_reduce_finish<double>(bt, partials, counter, [&](double total) { *out = total; });
}
void launch_bc_increment(uint32_t n, const uint8_t* mask, const double* val, double frac,
                         const double* u, double* v, float* v32, double* partials,
                         unsigned* counter, double* out, cudaStream_t s) {
    k_bc_increment<<<kRedBlocks, kVecThreads, 0, s>>>(n, mask, val, frac, u, v, v32, partials,
                                                     counter, out);
}

// R = -f - K v on free DOFs, 0 on constrained
template <typename T>
__global__ void k_predictor_rhs(uint32_t n, const uint8_t* __restrict__ mask,
                                const double* __restrict__ f, const T* __restrict__ Kv,
                                double* __restrict__ R) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += gridDim.x * blockDim.x)
        R[i] = mask[i] ? 0.0 : -f[i] - (double)Kv[i];
}
template <typename T>
void launch_predictor_rhs(uint32_t n, const uint8_t* mask, const double* f, const T* Kv,
                          double* R, cudaStream_t s) {
    k_predictor_rhs<T><<<kRedBlocks * 2, kVecThreads, 0, s>>>(n, mask, f, Kv, R);
}

// Dirichlet elimination on an assembled node-block K: entries in a
// constrained row or column become 0, constrained diagonals 1.
template <typename T>
__global__ void __launch_bounds__(256)
    k_apply_bc_nodes(uint32_t nn, const uint32_t* __restrict__ nbr_ptr,
                     const uint32_t* __restrict__ nbr, const uint8_t* __restrict__ mask,
                     T* __restrict__ K) {
    const int lane = threadIdx.x & 31;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t n = warp; n < nn; n += nwarps) {
        const uint32_t nb0 = nbr_ptr[n];
        const int deg = (int)(nbr_ptr[n + 1] - nb0);
        const int rl = 3 * deg;
        T* v = K + 9 * (size_t)nb0;
        for (int idx = lane; idx < 3 * rl; idx += 32) {
            const int p = idx / rl;
            const int rem = idx - p * rl;
            const int k = rem / 3;
            const uint32_t row = 3 * n + p;
            const uint32_t col = 3 * __ldg(nbr + nb0 + k) + (rem - 3 * k);
            if (mask[row] | mask[col]) v[idx] = (row == col) ? T(1) : T(0);
        }
    }
}
template <typename T>
void launch_apply_bc_nodes(uint32_t nn, const uint32_t* nbr_ptr, const uint32_t* nbr,
                           const uint8_t* mask, T* K, cudaStream_t s) {
    k_apply_bc_nodes<T><<<kSpmvBlocks, 256, 0, s>>>(nn, nbr_ptr, nbr, mask, K);
}

// ---- explicit instantiations ------------------------------------------------
template void launch_predictor_rhs<double>(uint32_t, const uint8_t*, const double*,
                                           const double*, double*, cudaStream_t);
template void launch_predictor_rhs<float>(uint32_t, const uint8_t*, const double*, const float*,
                                          double*, cudaStream_t);
template void launch_apply_bc_nodes<double>(uint32_t, const uint32_t*, const uint32_t*,
                                            const uint8_t*, double*, cudaStream_t);
template void launch_apply_bc_nodes<float>(uint32_t, const uint32_t*, const uint32_t*,
                                           const uint8_t*, float*, cudaStream_t);
#define FM_INST(T)                                                                              \
    template void launch_spmv_nodes<T>(uint32_t, const uint32_t*, const uint32_t*, const T*,    \
                                       const T*, T*, T*, unsigned*, double*, cudaStream_t);     \
    template void launch_spmv_csr<T>(uint32_t, const uint32_t*, const uint32_t*, const T*,      \
                                     const T*, T*, T*, unsigned*, double*, cudaStream_t);       \
    template void launch_ilu0_csr<T>(const CsrDev&, const T*, T*, T*, unsigned*, unsigned,      \
                                     unsigned*, int, cudaStream_t);                             \
    template void launch_trsv_lower_csr<T>(const CsrDev&, const T*, const T*, T*, unsigned*,    \
                                           unsigned, unsigned*, int, cudaStream_t);             \
    template void launch_trsv_upper_csr<T>(const CsrDev&, const T*, const T*, const T*, T*,     \
                                           unsigned*, unsigned, unsigned*, int, cudaStream_t);  \
    template void launch_dot<T>(uint32_t, const T*, const T*, T*, unsigned*, double*,           \
                                cudaStream_t);                                                  \
    template void launch_residual_init<T>(uint32_t, const T*, T*, T*, unsigned*, double*,       \
                                          cudaStream_t);                                        \
    template void launch_pcg_start<T>(uint32_t, const T*, const T*, const T*, T*, T*,           \
                                      unsigned*, DevScalars*, cudaStream_t);                    \
    template void launch_pcg_update_xr<T>(uint32_t, const T*, const T*, T*, T*, DevScalars*,    \
                                          cudaStream_t);                                        \
    template void launch_pcg_rz<T>(uint32_t, const T*, const T*, T*, unsigned*, DevScalars*,    \
                                   cudaStream_t);                                               \
    template void launch_pcg_update_p<T>(uint32_t, const T*, T*, DevScalars*, cudaStream_t);
FM_INST(double)
FM_INST(float)
#undef FM_INST

}  // namespace fm
