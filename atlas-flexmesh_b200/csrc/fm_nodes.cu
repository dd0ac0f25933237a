// fm_nodes.cu — node-block (3x3) ILU(0) factorization and triangular solves
// on the solve pattern of a tetrahedral mesh.
//
// The three rows of node n share one column structure (3 columns per
// neighbour node, neighbours ascending), so a warp handles a whole node:
// dependencies are tracked per node, the dependency depth drops by 3x
// against scalar rows (6N instead of 18N levels on the N^3 unit cube), and
// the intra-node coupling (the 3x3 diagonal block) is resolved in registers.
//
// Scheduling is sync-free: a persistent grid walks nodes in a topological
// order (dependency levels); every warp handles positions w, w+W, ... of
// that order, so the lowest unfinished node always has its inputs complete
// and all waits end.  Both the factorization and the triangular solves
// (fm_trsv.cu) wait on the dependencies' values themselves: the outputs are
// filled with a sentinel before the launch and a value is final once it
// differs from it.
#include <algorithm>
#include <cstdlib>

#include "fm_kernels.hpp"
#include "fm_nodes.hpp"
#include "fm_sync.cuh"

namespace fm {

constexpr int kNodeWarps = 4;

template <typename T>
__global__ void k_fill_sentinel(uint32_t n, T* __restrict__ x) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        x[i] = Sentinel<T>::value();
}

// ---------------------------------------------------------------------------
// ILU(0) factorization, one warp per node (its three rows), IKJ order.
// For each lower column c = 3m+q (m a lower neighbour, ascending; then the
// node's own columns), every row p of the node takes l_p = w_p[c] / d_c and
// subtracts l_p U(c, j) from each of its entries j > c present in its
// pattern; the pivot of row 3n+p is w_p[3n+p] after all its updates,
// perturbed by +-1e-8 when below 1e-12 in magnitude.  The subtraction order
// per entry is the reference's (ascending c).
//
// The node's three rows live in registers (lane owns columns lane,
// lane+32, lane+64).  The U parts of every lower neighbour's rows are
// loaded in one round of independent loads, re-read while any still holds
// the sentinel (at 64^3: 1.83 ms per FP32 factorization and 2.40 ms FP64,
// against 2.00 and 2.65 ms with a per-node release flag), and staged into
// shared memory, already scattered to the node's own column positions through a
// structural map built on the host (ilu_edge_maps): a dense row per
// (neighbour, row q), zero where the neighbour has no entry.  Each
// elimination step is then a broadcast of the pivot column (three
// shuffles) and three FMAs per owned column, with no shared-memory
// read-modify-write and no warp barrier.  Neighbours are staged in chunks
// of kStageNbrs (more only for meshes with more lower neighbours or nodes of
// more than 21 neighbours).
// ---------------------------------------------------------------------------
constexpr int kStageNbrs = 9;   // lower neighbours staged (and unrolled) at once
constexpr int kStageVals = kStageNbrs * 3 * 64;  // dense U rows of 64 columns each
constexpr int kPairRound = 3;   // (neighbour, node) pairs each lane loads per round

template <typename T>
struct IluStage {
    T u[kStageVals];           // [k - k0][q][column of n] U(3m+q, .) of staged neighbours
    T lm[3][96];               // multipliers L(3n+p, c) of the columns eliminated so far
    uint32_t poff[33];         // first pair of lower neighbour k (m, then its upper neighbours)
    uint32_t mb0[32];          // lower neighbour k: first neighbour entry
    uint8_t mdeg[32], msk[32];
};

template <typename T>
__device__ __forceinline__ T pick3(const T v[3], int s) {
    return s == 0 ? v[0] : s == 1 ? v[1] : v[2];
}

// Elimination against lower neighbour k (the node's columns 3k .. 3k+2):
// multipliers by forward substitution through the neighbour's own U block,
// then l_0 U_0j, l_1 U_1j, l_2 U_2j subtracted from every owned column in
// that order (the reference's column order).  Entries outside the
// neighbour's pattern are staged as zeros: x - l 0 = x.  The multipliers go
// to G.lm; the pivot columns in w are not read again (write-back takes G.lm
// for every column left of the diagonal), so the updates need no selects.
template <typename T>
__device__ __forceinline__ void ilu_step(IluStage<T>& G, T (&w)[3][3], int k, int k0, int rs,
                                         int nsl, int lane, T dv0, T dv1, T dv2) {
    const T d0 = __shfl_sync(kFull, dv0, k), d1 = __shfl_sync(kFull, dv1, k),
            d2 = __shfl_sync(kFull, dv2, k);
    const T* ur0 = G.u + ((k - k0) * 3 + 0) * rs;
    const T* ur1 = ur0 + rs;
    const T* ur2 = ur1 + rs;
    const int c0 = 3 * k;
    const T u01 = ur0[c0 + 1], u02 = ur0[c0 + 2], u12 = ur1[c0 + 2];
    T l[3][3];  // l[p][q]
#pragma unroll
    for (int p = 0; p < 3; ++p) {
        T wq[3];
#pragma unroll
        for (int q = 0; q < 3; ++q)
            wq[q] = __shfl_sync(kFull, pick3(w[p], (c0 + q) >> 5), (c0 + q) & 31);
        l[p][0] = wq[0] * d0;
        l[p][1] = (wq[1] - l[p][0] * u01) * d1;
        l[p][2] = ((wq[2] - l[p][0] * u02) - l[p][1] * u12) * d2;
    }
    if (lane == 0)
#pragma unroll
        for (int p = 0; p < 3; ++p)
#pragma unroll
            for (int q = 0; q < 3; ++q) G.lm[p][c0 + q] = l[p][q];
#pragma unroll
    for (int s = 0; s < 3; ++s) {
        if (s < nsl) {
            const int j = lane + 32 * s;
            const T a0 = ur0[j], a1 = ur1[j], a2 = ur2[j];
#pragma unroll
            for (int p = 0; p < 3; ++p)
                w[p][s] = ((w[p][s] - l[p][0] * a0) - l[p][1] * a1) - l[p][2] * a2;
        }
    }
}

// A value another warp writes over the sentinel: read until it differs
// (bounded; on a timeout FM_FLAG_TIMEOUT is set and ok cleared).
template <typename T>
__device__ __forceinline__ T ld_final(const T* p, unsigned* status, bool& ok) {
    T v = ld_relaxed(p);
    if (!Sentinel<T>::is(v)) return v;
    const long long t0 = clock64(), limit = wait_limit(status);
    for (unsigned it = 1; ok; ++it) {
        v = ld_relaxed(p);
        if (!Sentinel<T>::is(v)) break;
        if ((it & 31u) == 0 &&
            ((ld_volatile_u32(status) & FM_FLAG_TIMEOUT) || clock64() - t0 > limit)) {
            raise_flag(status, FM_FLAG_TIMEOUT);
            ok = false;
        }
    }
    return v;
}

template <typename T>
__global__ void __launch_bounds__(kNodeWarps * 32, sizeof(T) == 4 ? 3 : 2)
    k_ilu0_nodes(NodeSched S, const T* __restrict__ a, T* __restrict__ lu, T* __restrict__ dg,
                 T* __restrict__ dinv, unsigned* __restrict__ status) {
    extern __shared__ __align__(16) unsigned char ilu_smem[];
    IluStage<T>* stage = reinterpret_cast<IluStage<T>*>(ilu_smem);
    constexpr int UCAP = kStageVals;
    const int lane = threadIdx.x & 31, wi = threadIdx.x >> 5;
    IluStage<T>& G = stage[wi];
    const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t W = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t t = gw; t < S.n_nodes; t += W) {
        const uint32_t n = __ldg(S.fwd_order + t);
        const uint32_t nb0 = __ldg(S.nbr_ptr + n);
        const int deg = (int)(__ldg(S.nbr_ptr + n + 1) - nb0);
        const int sk = (int)__ldg(S.self_pos + n);
        const int rl = 3 * deg, ds = 3 * sk;
        const T* arow = a + 9 * (size_t)nb0;
        T w[3][3];
#pragma unroll
        for (int p = 0; p < 3; ++p)
#pragma unroll
            for (int s = 0; s < 3; ++s) {
                const int j = lane + 32 * s;
                w[p][s] = j < rl ? arow[(size_t)p * rl + j] : T(0);
            }
        const T adiag = lane < 3 ? arow[(size_t)lane * rl + ds + lane] : T(0);
        const uint32_t my_nbr = lane < deg ? __ldg(S.nbr + nb0 + lane) : 0xffffffffu;
        uint32_t mb0 = 0, mdeg = 0, msk = 0;
        if (lane < sk) {
            mb0 = __ldg(S.nbr_ptr + my_nbr);
            mdeg = __ldg(S.nbr_ptr + my_nbr + 1) - mb0;
            msk = __ldg(S.self_pos + my_nbr);
        }
        const uint32_t np = mdeg - msk;  // pairs of lower neighbour `lane` (0 beyond sk)
        uint32_t incl = np;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t v = __shfl_up_sync(kFull, incl, o);
            if (lane >= o) incl += v;
        }
        const uint32_t eb = __ldg(S.emap_ptr + n);
        const uint32_t tot = __shfl_sync(kFull, incl, 31);  // pairs of all lower neighbours
        __syncwarp();  // the previous node's reads of G are done
        G.poff[lane] = incl - np;
        if (lane == 31) G.poff[32] = incl;
        G.mb0[lane] = mb0;
        G.mdeg[lane] = (uint8_t)mdeg;
        G.msk[lane] = (uint8_t)msk;
        // staged rows are padded to whole 32-column slots (zeros beyond rl), so
        // the updates need no column mask
        const int nsl = (rl + 31) >> 5;
        const int rs = 32 * nsl;
        const int cap_k = UCAP / (3 * rs) > 0 ? UCAP / (3 * rs) : 1;
        // Usual case (all lower neighbours in one stage, one round of pairs per
        // lane): everything structural about the staging — the zeroed stage,
        // each pair's neighbour, source row and destination column — is done
        // before the wait, so after it only the U values are loaded.
        const bool fast = sk > 0 && sk <= cap_k && sk <= kStageNbrs &&
                          tot <= (uint32_t)(32 * kPairRound);
        const T* fsrc[kPairRound];
        int fmrl[kPairRound], fjb[kPairRound], flim[kPairRound], fdst[kPairRound];
        uint32_t fpos[kPairRound];
        if (fast) {
            for (int i = lane; i < sk * 3 * rs; i += 32) G.u[i] = T(0);
            __syncwarp();
#pragma unroll
            for (int r = 0; r < kPairRound; ++r) {
                const uint32_t pr = lane + 32 * r;
                fpos[r] = 0xffu;
                fdst[r] = 0;
                fsrc[r] = nullptr;
                fmrl[r] = fjb[r] = flim[r] = 0;
                if (pr < tot) {
                    int k = 0;
                    for (int kk = 1; kk < sk; ++kk) k += (int)(G.poff[kk] <= pr);
                    fpos[r] = __ldg(S.emap + eb + pr);
                    const int ms = G.msk[k];
                    const int kk = ms + (int)(pr - G.poff[k]);
                    fmrl[r] = 3 * (int)G.mdeg[k];
                    fjb[r] = 3 * kk;
                    flim[r] = 3 * ms;
                    fsrc[r] = lu + 9 * (size_t)G.mb0[k] + 3 * kk;
                    fdst[r] = (k * 3) * rs;
                }
            }
        }
        // The lower neighbours' U rows and reciprocal pivots are final once
        // they differ from the sentinel the launch filled LU and dinv with:
        // every load is issued at once and what still reads the sentinel is
        // read again (bounded).  No per-node flag: releasing one cost the
        // producer a fence that waits for its row stores, and the reader a
        // second L2 round trip after the flag.
        const bool nb_lane = lane < sk;
        const T* dsrc = dinv + 3 * (size_t)(nb_lane ? my_nbr : 0u);
        T dv0 = T(0), dv1 = T(0), dv2 = T(0);
        if (nb_lane) {
            dv0 = ld_relaxed(dsrc);
            dv1 = ld_relaxed(dsrc + 1);
            dv2 = ld_relaxed(dsrc + 2);
        }
        T val[kPairRound][9];
#pragma unroll
        for (int r = 0; r < kPairRound; ++r)
#pragma unroll
            for (int q = 0; q < 3; ++q)
#pragma unroll
                for (int c = 0; c < 3; ++c)
                    val[r][3 * q + c] = fast && fpos[r] != 0xffu && fjb[r] + c > flim[r] + q
                                            ? ld_relaxed(fsrc[r] + (size_t)q * fmrl[r] + c)
                                            : T(0);
        auto pending = [&]() {
            bool p = Sentinel<T>::is(dv0) | Sentinel<T>::is(dv1) | Sentinel<T>::is(dv2);
#pragma unroll
            for (int r = 0; r < kPairRound; ++r)
#pragma unroll
                for (int k = 0; k < 9; ++k) p |= Sentinel<T>::is(val[r][k]);
            return p;
        };
        bool ok = true;
        bool need = pending();
        if (__any_sync(kFull, need)) {
            const long long t0 = clock64(), limit = wait_limit(status);
            for (unsigned it = 1;; ++it) {
                if (need) {
                    if (Sentinel<T>::is(dv0)) dv0 = ld_relaxed(dsrc);
                    if (Sentinel<T>::is(dv1)) dv1 = ld_relaxed(dsrc + 1);
                    if (Sentinel<T>::is(dv2)) dv2 = ld_relaxed(dsrc + 2);
#pragma unroll
                    for (int r = 0; r < kPairRound; ++r)
#pragma unroll
                        for (int q = 0; q < 3; ++q)
#pragma unroll
                            for (int c = 0; c < 3; ++c)
                                if (Sentinel<T>::is(val[r][3 * q + c]))
                                    val[r][3 * q + c] = ld_relaxed(fsrc[r] + (size_t)q * fmrl[r] + c);
                    need = pending();
                }
                if (!__any_sync(kFull, need)) break;
                if ((it & 31u) == 0 &&
                    __any_sync(kFull, (ld_volatile_u32(status) & FM_FLAG_TIMEOUT) ||
                                          clock64() - t0 > limit)) {
                    if (lane == 0) raise_flag(status, FM_FLAG_TIMEOUT);
                    ok = false;
                    break;
                }
            }
        }
        __syncwarp();
        if (ok && fast) {
#pragma unroll
            for (int r = 0; r < kPairRound; ++r)
                if (fpos[r] != 0xffu) {
                    const int d = fdst[r] + 3 * (int)fpos[r];
#pragma unroll
                    for (int q = 0; q < 3; ++q)
#pragma unroll
                        for (int c = 0; c < 3; ++c) G.u[d + q * rs + c] = val[r][3 * q + c];
                }
            __syncwarp();
#pragma unroll
            for (int k = 0; k < kStageNbrs; ++k)
                if (k < sk) ilu_step(G, w, k, 0, rs, nsl, lane, dv0, dv1, dv2);
            __syncwarp();
        }
        for (int k0 = 0; ok && !fast && k0 < sk; k0 += cap_k) {
            const int k1 = k0 + cap_k < sk ? k0 + cap_k : sk;
            const int nu = (k1 - k0) * 3 * rs;
            for (int i = lane; i < nu; i += 32) G.u[i] = T(0);
            __syncwarp();
            const uint32_t p0 = G.poff[k0], p1 = G.poff[k1];
            for (uint32_t base = p0; base < p1; base += 32 * kPairRound) {
                T val[kPairRound][9];
                int dst[kPairRound];
                // loads of a round in flight together
#pragma unroll
                for (int r = 0; r < kPairRound; ++r) {
                    dst[r] = -1;
                    const uint32_t pr = base + lane + 32 * r;
                    if (pr < p1) {
                        // neighbour of this pair: independent compares, not a chain
                        int k = k0;
                        for (int kk = k0 + 1; kk < k1; ++kk) k += (int)(G.poff[kk] <= pr);
                        const uint32_t pos = __ldg(S.emap + eb + pr);
                        if (pos != 0xffu) {
                            const int ms = G.msk[k], mrl = 3 * (int)G.mdeg[k];
                            const int kk = ms + (int)(pr - G.poff[k]);
                            const T* urow = lu + 9 * (size_t)G.mb0[k];
                            dst[r] = ((k - k0) * 3) * rs + 3 * (int)pos;
#pragma unroll
                            for (int q = 0; q < 3; ++q)
#pragma unroll
                                for (int c = 0; c < 3; ++c) {
                                    const int j = 3 * kk + c;
                                    val[r][3 * q + c] =
                                        j > 3 * ms + q
                                            ? ld_final(urow + (size_t)q * mrl + j, status, ok)
                                            : T(0);
                                }
                        }
                    }
                }
#pragma unroll
                for (int r = 0; r < kPairRound; ++r)
                    if (dst[r] >= 0)
#pragma unroll
                        for (int q = 0; q < 3; ++q)
#pragma unroll
                            for (int c = 0; c < 3; ++c) G.u[dst[r] + q * rs + c] = val[r][3 * q + c];
            }
            ok = __all_sync(kFull, ok);  // uniform before the loop tests it
            // one chunk starting at neighbour 0 (the usual case) runs fully
            // unrolled: pivot columns, shuffle lanes and stage offsets become
            // constants and the loads of later steps are hoisted (1.8x per step)
            if (k0 == 0 && k1 <= kStageNbrs) {
#pragma unroll
                for (int k = 0; k < kStageNbrs; ++k)
                    if (k < k1) ilu_step(G, w, k, 0, rs, nsl, lane, dv0, dv1, dv2);
            } else {
                for (int k = k0; k < k1; ++k) ilu_step(G, w, k, k0, rs, nsl, lane, dv0, dv1, dv2);
            }
            __syncwarp();  // before the next chunk overwrites G.u
        }
        // the node's own 3x3 block: columns 3n and 3n+1 eliminate rows below
        T piv[3];
#pragma unroll
        for (int p = 0; p < 3; ++p) {
            const int c = ds + p, owner = c & 31, sl = c >> 5;
            T u = __shfl_sync(kFull, pick3(w[p], sl), owner);
            if (fabs((double)u) < kPivotThreshold) {
                u += (u >= T(0) ? T(kPivotPerturb) : T(-kPivotPerturb));
                if (lane == 0) raise_flag(status, FM_FLAG_PIVOT);
            }
            piv[p] = u;
#pragma unroll
            for (int r2 = p + 1; r2 < 3; ++r2) {
                const T l = __shfl_sync(kFull, pick3(w[r2], sl), owner) / u;
                if (lane == 0) G.lm[r2][c] = l;
                // columns left of c only hold values write-back replaces
#pragma unroll
                for (int s = 0; s < 3; ++s) w[r2][s] = w[r2][s] - l * w[p][s];
            }
        }
        // write back: multipliers left of the diagonal, a_ii on the diagonal
        // slot (the pivots go to dg), U right of it
        __syncwarp();
        T* out = lu + 9 * (size_t)nb0;
#pragma unroll
        for (int p = 0; p < 3; ++p) {
            const T ap = __shfl_sync(kFull, adiag, p);
#pragma unroll
            for (int s = 0; s < 3; ++s) {
                const int j = lane + 32 * s;
                if (j < rl)
                    out[(size_t)p * rl + j] = j < ds + p ? G.lm[p][j] : j == ds + p ? ap : w[p][s];
            }
        }
        if (lane < 3) {
            const T pv = pick3(piv, lane);
            dg[3 * (size_t)n + lane] = pv;
            dinv[3 * (size_t)n + lane] = T(1) / pv;
            if (!isfinite((double)pv)) raise_flag(status, FM_FLAG_NONFINITE);
        }
    }
}

// ---------------------------------------------------------------------------
template <typename K>
static int resident_grid_nodes(K kernel, int device, size_t smem) {
    int sms = 0, per_sm = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kNodeWarps * 32, smem);
    if (per_sm < 1) per_sm = 1;
    return sms * per_sm;
}

// warps: about twice the widest dependency level, never more than resident
static int grid_for(int resident, uint32_t max_width) {
    long want = (2l * max_width + kNodeWarps - 1) / kNodeWarps;
    if (want < 1) want = 1;
    return (int)(want < resident ? want : resident);
}

template <typename T>
void launch_fill_sentinel(uint32_t n, T* x, cudaStream_t s) {
    k_fill_sentinel<T><<<592, 256, 0, s>>>(n, x);
}

template <typename T>
void launch_ilu0_nodes(const NodeSched& S, const T* a, T* lu, uint64_t nnz, T* d, T* dinv,
                       unsigned* status, int device, cudaStream_t s) {
    if (!S.n_nodes) return;
    // every LU entry and reciprocal pivot holds the sentinel until its node
    // writes it: the readers wait on the values themselves
    for (uint64_t o = 0; o < nnz; o += 1u << 30)
        launch_fill_sentinel<T>((uint32_t)std::min<uint64_t>(nnz - o, 1u << 30), lu + o, s);
    launch_fill_sentinel<T>(3 * S.n_nodes, dinv, s);
    static int res[2] = {0, 0};
    const int f = sizeof(T) == 4;
    const size_t smem = kNodeWarps * sizeof(IluStage<T>);
    if (!res[f]) {
        cudaFuncSetAttribute(k_ilu0_nodes<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem);
        res[f] = resident_grid_nodes(k_ilu0_nodes<T>, device, smem);
    }
    k_ilu0_nodes<T><<<grid_for(res[f], S.max_width_fwd), kNodeWarps * 32, smem, s>>>(
        S, a, lu, d, dinv, status);
}

template void launch_ilu0_nodes<double>(const NodeSched&, const double*, double*, uint64_t,
                                        double*, double*, unsigned*, int, cudaStream_t);
template void launch_ilu0_nodes<float>(const NodeSched&, const float*, float*, uint64_t, float*,
                                       float*, unsigned*, int, cudaStream_t);
template void launch_fill_sentinel<double>(uint32_t, double*, cudaStream_t);
template void launch_fill_sentinel<float>(uint32_t, float*, cudaStream_t);

}  // namespace fm
