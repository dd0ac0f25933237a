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
// and all waits end.  Triangular solves wait on the dependency's VALUES: the
// output vector is pre-filled with a NaN sentinel that arithmetic cannot
// produce, and a consumer spins (bounded) until the three values of a
// neighbour are no longer the sentinel - one L2 round trip per dependency.
// The factorization, whose outputs are whole rows, releases a per-node flag.
#include "fm_kernels.hpp"
#include "fm_nodes.hpp"

namespace fm {

constexpr int kNodeWarps = 8;

template <typename T>
struct Sentinel;
template <>
struct Sentinel<double> {
    static __device__ __forceinline__ double value() {
        return __longlong_as_double(0x7ff4dead0000beefll);
    }
    static __device__ __forceinline__ bool is(double v) {
        return __double_as_longlong(v) == 0x7ff4dead0000beefll;
    }
};
template <>
struct Sentinel<float> {
    static __device__ __forceinline__ float value() { return __int_as_float(0x7fa0beef); }
    static __device__ __forceinline__ bool is(float v) { return __float_as_int(v) == 0x7fa0beef; }
};

__device__ __forceinline__ double ld_relaxed(const double* p) {
    double v;
    asm volatile("ld.relaxed.gpu.global.f64 %0, [%1];" : "=d"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ float ld_relaxed(const float* p) {
    float v;
    asm volatile("ld.relaxed.gpu.global.f32 %0, [%1];" : "=f"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_relaxed(double* p, double v) {
    asm volatile("st.relaxed.gpu.global.f64 [%0], %1;" ::"l"(p), "d"(v) : "memory");
}
__device__ __forceinline__ void st_relaxed(float* p, float v) {
    asm volatile("st.relaxed.gpu.global.f32 [%0], %1;" ::"l"(p), "f"(v) : "memory");
}

// Spin (bounded) until *p is not the sentinel; returns the value, or the
// sentinel when the wait gave up (FM_FLAG_TIMEOUT then set).
template <typename T>
__device__ __forceinline__ T wait_value(const T* p, unsigned* status) {
    T v = ld_relaxed(p);
    if (!Sentinel<T>::is(v)) return v;
    const long long t0 = clock64();
    for (unsigned it = 1;; ++it) {
        v = ld_relaxed(p);
        if (!Sentinel<T>::is(v)) return v;
        if ((it & 63u) == 0) {
            if (ld_volatile_u32(status) & FM_FLAG_TIMEOUT) return v;
            if (clock64() - t0 > kWaitCycles) {
                raise_flag(status, FM_FLAG_TIMEOUT);
                return v;
            }
        }
    }
}

template <typename T>
__global__ void k_fill_sentinel(uint32_t n, T* __restrict__ x) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        x[i] = Sentinel<T>::value();
}

// ---------------------------------------------------------------------------
// Forward solve L z = r (L unit lower), one warp per node, value-sentinel waits.
// Every lane owns up to 3 (neighbour, column) items; everything that does not
// depend on the neighbours' values (indices, LU entries, r, the node's own
// block) is loaded before the first wait, so a dependency costs one poll.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(kNodeWarps * 32)
    k_trsv_lower_nodes(NodeSched S, const T* __restrict__ lu, const T* __restrict__ r,
                       T* __restrict__ z, unsigned* __restrict__ status) {
    const int lane = threadIdx.x & 31;
    const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t W = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t t = gw; t < S.n_nodes; t += W) {
        const uint32_t n = __ldg(S.fwd_order + t);
        const uint32_t nb0 = __ldg(S.nbr_ptr + n);
        const int deg = (int)(__ldg(S.nbr_ptr + n + 1) - nb0);
        const int sk = (int)__ldg(S.self_pos + n);  // lower neighbours are k < sk
        const T* row = lu + 9 * (size_t)nb0;
        const int rl = 3 * deg, ni = 3 * sk;
        T a0[3], a1[3], a2[3];
        const T* zp[3];
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const int idx = lane + 32 * j;
            zp[j] = nullptr;
            a0[j] = a1[j] = a2[j] = T(0);
            if (idx < ni) {
                const int k = idx / 3;
                zp[j] = z + 3 * (size_t)__ldg(S.nbr + nb0 + k) + (idx - 3 * k);
                a0[j] = __ldg(row + idx);
                a1[j] = __ldg(row + rl + idx);
                a2[j] = __ldg(row + 2 * rl + idx);
            }
        }
        T r0 = T(0), r1 = T(0), r2 = T(0), l10 = T(0), l20 = T(0), l21 = T(0);
        if (lane == 0) {
            r0 = __ldg(r + 3 * (size_t)n);
            r1 = __ldg(r + 3 * (size_t)n + 1);
            r2 = __ldg(r + 3 * (size_t)n + 2);
            l10 = __ldg(row + rl + ni);
            l20 = __ldg(row + 2 * rl + ni);
            l21 = __ldg(row + 2 * rl + ni + 1);
        }
        T s0 = T(0), s1 = T(0), s2 = T(0);
#pragma unroll
        for (int j = 0; j < 3; ++j)
            if (zp[j]) {
                const T zv = wait_value(zp[j], status);
                s0 += a0[j] * zv;
                s1 += a1[j] * zv;
                s2 += a2[j] * zv;
            }
        s0 = warp_sum(s0);
        s1 = warp_sum(s1);
        s2 = warp_sum(s2);
        if (lane == 0) {
            const T z0 = r0 - s0;
            const T z1 = r1 - s1 - l10 * z0;
            const T z2 = r2 - s2 - l20 * z0 - l21 * z1;
            st_relaxed(z + 3 * (size_t)n, z0);
            st_relaxed(z + 3 * (size_t)n + 1, z1);
            st_relaxed(z + 3 * (size_t)n + 2, z2);
        }
    }
}

// ---------------------------------------------------------------------------
// Backward solve U y = z with reciprocal pivots dinv, reverse topological order
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(kNodeWarps * 32)
    k_trsv_upper_nodes(NodeSched S, const T* __restrict__ lu, const T* __restrict__ dinv,
                       const T* __restrict__ z, T* __restrict__ y, unsigned* __restrict__ status) {
    const int lane = threadIdx.x & 31;
    const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t W = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t t = gw; t < S.n_nodes; t += W) {
        const uint32_t n = __ldg(S.bwd_order + t);
        const uint32_t nb0 = __ldg(S.nbr_ptr + n);
        const int deg = (int)(__ldg(S.nbr_ptr + n + 1) - nb0);
        const int sk = (int)__ldg(S.self_pos + n);  // upper neighbours are k > sk
        const T* row = lu + 9 * (size_t)nb0;
        const int rl = 3 * deg, lo = 3 * (sk + 1), ds = 3 * sk;
        T a0[3], a1[3], a2[3];
        const T* yp[3];
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const int idx = lo + lane + 32 * j;
            yp[j] = nullptr;
            a0[j] = a1[j] = a2[j] = T(0);
            if (idx < rl) {
                const int k = idx / 3;
                yp[j] = y + 3 * (size_t)__ldg(S.nbr + nb0 + k) + (idx - 3 * k);
                a0[j] = __ldg(row + idx);
                a1[j] = __ldg(row + rl + idx);
                a2[j] = __ldg(row + 2 * rl + idx);
            }
        }
        const size_t b = 3 * (size_t)n;
        T z0 = T(0), z1 = T(0), z2 = T(0), u01 = T(0), u02 = T(0), u12 = T(0);
        T i0 = T(0), i1 = T(0), i2 = T(0);
        if (lane == 0) {
            z0 = z[b];
            z1 = z[b + 1];
            z2 = z[b + 2];
            u01 = __ldg(row + ds + 1);
            u02 = __ldg(row + ds + 2);
            u12 = __ldg(row + rl + ds + 2);
            i0 = __ldg(dinv + b);
            i1 = __ldg(dinv + b + 1);
            i2 = __ldg(dinv + b + 2);
        }
        T s0 = T(0), s1 = T(0), s2 = T(0);
#pragma unroll
        for (int j = 0; j < 3; ++j)
            if (yp[j]) {
                const T yv = wait_value(yp[j], status);
                s0 += a0[j] * yv;
                s1 += a1[j] * yv;
                s2 += a2[j] * yv;
            }
        s0 = warp_sum(s0);
        s1 = warp_sum(s1);
        s2 = warp_sum(s2);
        if (lane == 0) {
            const T y2 = (z2 - s2) * i2;
            const T y1 = (z1 - s1 - u12 * y2) * i1;
            const T y0 = (z0 - s0 - u01 * y1 - u02 * y2) * i0;
            st_relaxed(y + b, y0);
            st_relaxed(y + b + 1, y1);
            st_relaxed(y + b + 2, y2);
        }
    }
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
void launch_trsv_nodes(const NodeSched& S, const T* lu, const T* dinv, const T* r, T* tmp, T* y,
                       unsigned* status, int device, cudaStream_t s) {
    if (!S.n_nodes) return;
    static int res_lo[2] = {0, 0}, res_up[2] = {0, 0};
    const int f = sizeof(T) == 4;
    if (!res_lo[f]) res_lo[f] = resident_grid_nodes(k_trsv_lower_nodes<T>, device);
    if (!res_up[f]) res_up[f] = resident_grid_nodes(k_trsv_upper_nodes<T>, device);
    const uint32_t n = 3 * S.n_nodes;
    k_fill_sentinel<T><<<592, 256, 0, s>>>(n, tmp);
    k_trsv_lower_nodes<T><<<grid_for(res_lo[f], S.max_width_fwd), kNodeWarps * 32, 0, s>>>(
        S, lu, r, tmp, status);
    k_fill_sentinel<T><<<592, 256, 0, s>>>(n, y);
    k_trsv_upper_nodes<T><<<grid_for(res_up[f], S.max_width_bwd), kNodeWarps * 32, 0, s>>>(
        S, lu, dinv, tmp, y, status);
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

template void launch_trsv_nodes<double>(const NodeSched&, const double*, const double*,
                                        const double*, double*, double*, unsigned*, int,
                                        cudaStream_t);
template void launch_trsv_nodes<float>(const NodeSched&, const float*, const float*, const float*,
                                       float*, float*, unsigned*, int, cudaStream_t);
template void launch_ilu0_nodes<double>(const NodeSched&, const double*, double*, double*,
                                        double*, unsigned*, unsigned, unsigned*, int,
                                        cudaStream_t);
template void launch_ilu0_nodes<float>(const NodeSched&, const float*, float*, float*, float*,
                                       unsigned*, unsigned, unsigned*, int, cudaStream_t);
template void launch_fill_sentinel<double>(uint32_t, double*, cudaStream_t);
template void launch_fill_sentinel<float>(uint32_t, float*, cudaStream_t);

}  // namespace fm
