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
// and all waits end.  The factorization, whose outputs are whole rows,
// releases a per-node flag; the triangular solves (fm_trsv.cu) wait on the
// dependencies' values directly.
#include "fm_kernels.hpp"
#include "fm_nodes.hpp"
#include "fm_sync.cuh"

namespace fm {

constexpr int kNodeWarps = 8;

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
// Shared memory per warp: the node's 3 rows (3*3*deg values), its
// neighbour list, and the position map of neighbour m's upper neighbours.
// ---------------------------------------------------------------------------
template <typename T>
struct IluStage {
    T w[3][3 * 32];       // rows p of node n, entries [k][q] flattened, deg <= 32
    uint32_t nbr[32];     // neighbours of n
};

// U part of the three rows of lower neighbour m, held in registers: lane
// owns column j = 3*msk + 1 + lane (+32) of m's rows, with its destination
// in n's rows (-1 when n's pattern lacks that column).
template <typename T>
struct URows {
    T u[2][3];
    int dst[2];
    int jj[2];
    T dinv[3];
};

template <typename T>
__device__ __forceinline__ void load_urows(const NodeSched& S, const T* lu, const T* dinv,
                                           const uint32_t* nbr_n, int deg, uint32_t m, int lane,
                                           URows<T>& U) {
    const uint32_t mb0 = __ldg(S.nbr_ptr + m);
    const int mdeg = (int)(__ldg(S.nbr_ptr + m + 1) - mb0);
    const int msk = (int)__ldg(S.self_pos + m);
    const int mrl = 3 * mdeg;
    const T* urow = lu + 9 * (size_t)mb0;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        const int j = 3 * msk + 1 + lane + 32 * h;
        U.jj[h] = j;
        U.dst[h] = -1;
        U.u[h][0] = U.u[h][1] = U.u[h][2] = T(0);
        if (j < mrl) {
            const int kk = j / 3;
            const uint32_t mm = __ldg(S.nbr + mb0 + kk);
            int lo = 0, hi = deg - 1, pos = -1;
            while (lo <= hi) {
                const int mid = (lo + hi) >> 1;
                const uint32_t v = nbr_n[mid];
                if (v == mm) { pos = mid; break; }
                if (v < mm) lo = mid + 1; else hi = mid - 1;
            }
            if (pos >= 0) {
                U.dst[h] = 3 * pos + (j - 3 * kk);
                // row q of m owns j when j > 3*msk + q (strictly upper)
#pragma unroll
                for (int q = 0; q < 3; ++q)
                    if (j > 3 * msk + q) U.u[h][q] = ld_cg(urow + (size_t)q * mrl + j);
            }
        }
    }
#pragma unroll
    for (int q = 0; q < 3; ++q) U.dinv[q] = ld_cg(dinv + 3 * (size_t)m + q);
    (void)U.jj;
}

template <typename T>
__global__ void __launch_bounds__(kNodeWarps * 32)
    k_ilu0_nodes(NodeSched S, const T* __restrict__ a, T* __restrict__ lu, T* __restrict__ dg,
                 T* __restrict__ dinv, unsigned* __restrict__ done, unsigned epoch,
                 unsigned* __restrict__ status) {
    __shared__ IluStage<T> stage[kNodeWarps];
    const int lane = threadIdx.x & 31, wi = threadIdx.x >> 5;
    IluStage<T>& G = stage[wi];
    const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t W = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t t = gw; t < S.n_nodes; t += W) {
        const uint32_t n = __ldg(S.fwd_order + t);
        const uint32_t nb0 = __ldg(S.nbr_ptr + n);
        const int deg = (int)(__ldg(S.nbr_ptr + n + 1) - nb0);
        const int sk = (int)__ldg(S.self_pos + n);
        const int rl = 3 * deg;
        const T* arow = a + 9 * (size_t)nb0;
        __syncwarp();
        for (int i = lane; i < rl; i += 32) {
            G.w[0][i] = arow[i];
            G.w[1][i] = arow[rl + i];
            G.w[2][i] = arow[2 * rl + i];
        }
        const uint32_t my_nbr = lane < deg ? __ldg(S.nbr + nb0 + lane) : 0xffffffffu;
        G.nbr[lane] = my_nbr;
        // wait for every lower neighbour node's rows
        bool ok = true;
        if (lane < sk) ok = wait_flag(done + my_nbr, epoch, status);
        ok = __all_sync(kFull, ok);
        __syncwarp();
        if (ok && sk > 0) {
            URows<T> cur, nxt;
            load_urows(S, lu, dinv, G.nbr, deg, G.nbr[0], lane, cur);
            for (int k = 0; k < sk; ++k) {
                if (k + 1 < sk) load_urows(S, lu, dinv, G.nbr, deg, G.nbr[k + 1], lane, nxt);
#pragma unroll
                for (int q = 0; q < 3; ++q) {
                    // multipliers of column c = 3m+q in the node's three rows
                    const T l0 = G.w[0][3 * k + q] * cur.dinv[q];
                    const T l1 = G.w[1][3 * k + q] * cur.dinv[q];
                    const T l2 = G.w[2][3 * k + q] * cur.dinv[q];
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        const int d = cur.dst[h];
                        if (d >= 0 && cur.u[h][q] != T(0)) {
                            const T uv = cur.u[h][q];
                            G.w[0][d] -= l0 * uv;
                            G.w[1][d] -= l1 * uv;
                            G.w[2][d] -= l2 * uv;
                        }
                    }
                    __syncwarp();
                    if (lane == 0) {
                        G.w[0][3 * k + q] = l0;
                        G.w[1][3 * k + q] = l1;
                        G.w[2][3 * k + q] = l2;
                    }
                    __syncwarp();
                }
                if (k + 1 < sk) cur = nxt;
            }
        }
        // the node's own 3x3 block: columns 3n and 3n+1 eliminate rows below
        const int ds = 3 * sk;
        T piv[3];
        for (int p = 0; p < 3; ++p) {
            T u = G.w[p][ds + p];
            if (fabs((double)u) < kPivotThreshold) {
                u += (u >= T(0) ? T(kPivotPerturb) : T(-kPivotPerturb));
                if (lane == 0) raise_flag(status, FM_FLAG_PIVOT);
            }
            piv[p] = u;
            __syncwarp();
            for (int r2 = p + 1; r2 < 3; ++r2) {
                const T l = G.w[r2][ds + p] / u;
                for (int j = ds + p + 1 + lane; j < rl; j += 32) G.w[r2][j] -= l * G.w[p][j];
                __syncwarp();
                if (lane == 0) G.w[r2][ds + p] = l;
                __syncwarp();
            }
        }
        // write back: diagonal slots keep a_ii (the pivots go to dg)
        T* out = lu + 9 * (size_t)nb0;
        for (int i = lane; i < rl; i += 32) {
            out[i] = (i == ds) ? arow[i] : G.w[0][i];
            out[rl + i] = (i == ds + 1) ? arow[rl + i] : G.w[1][i];
            out[2 * rl + i] = (i == ds + 2) ? arow[2 * rl + i] : G.w[2][i];
        }
        if (lane < 3) {
            dg[3 * (size_t)n + lane] = piv[lane];
            dinv[3 * (size_t)n + lane] = T(1) / piv[lane];
            if (!isfinite((double)piv[lane])) raise_flag(status, FM_FLAG_NONFINITE);
        }
        __threadfence();
        __syncwarp();
        if (lane == 0) st_release(done + n, epoch);
    }
}

// ---------------------------------------------------------------------------
template <typename K>
static int resident_grid_nodes(K kernel, int device) {
    int sms = 0, per_sm = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kNodeWarps * 32, 0);
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
void launch_ilu0_nodes(const NodeSched& S, const T* a, T* lu, T* d, T* dinv, unsigned* done,
                       unsigned epoch, unsigned* status, int device, cudaStream_t s) {
    if (!S.n_nodes) return;
    static int res[2] = {0, 0};
    const int f = sizeof(T) == 4;
    if (!res[f]) res[f] = resident_grid_nodes(k_ilu0_nodes<T>, device);
    k_ilu0_nodes<T><<<grid_for(res[f], S.max_width_fwd), kNodeWarps * 32, 0, s>>>(
        S, a, lu, d, dinv, done, epoch, status);
}

template void launch_ilu0_nodes<double>(const NodeSched&, const double*, double*, double*,
                                        double*, unsigned*, unsigned, unsigned*, int,
                                        cudaStream_t);
template void launch_ilu0_nodes<float>(const NodeSched&, const float*, float*, float*, float*,
                                       unsigned*, unsigned, unsigned*, int, cudaStream_t);
template void launch_fill_sentinel<double>(uint32_t, double*, cudaStream_t);
template void launch_fill_sentinel<float>(uint32_t, float*, cudaStream_t);

}  // namespace fm
