// fm_trsv.cu — sync-free node-block triangular solves of the ILU(0)
// preconditioner, software-pipelined.
//
// A persistent grid walks the nodes in dependency-level order; warp w takes
// positions w, w+W, w+2W, ...  Each position has a 16-byte schedule record
// {node, first neighbour slot, degree, own slot} so the setup of a node is
// one load.  While a warp waits on the neighbour values of its current node
// it already has the next node's record, LU entries and neighbour indices in
// flight, so what is left on the critical path of a dependency level is
// the dependency itself (one L2 round trip to observe the neighbour's value;
// outputs are pre-filled with a NaN sentinel, polls are relaxed gpu-scope
// loads) plus the node's own finish.
//
// Lane k of the warp owns neighbour node k of the solve's side (lower
// neighbours for L, upper ones for U): it waits for that node's three
// values and forms the 3x3 block product; a butterfly sums the partials.
// The waits run in lock step (the loop's exit is a warp vote): lanes that
// spin separately split the warp, and on B200 its reconvergence before the
// reduction cost more than the dependency hop itself (traced per node with
// %globaltimer: 1.23 -> 0.73 ms per FP32 forward+backward pair at 64^3).
#include <cstdlib>

#include "fm_kernels.hpp"
#include "fm_nodes.hpp"
#include "fm_sync.cuh"

namespace fm {

constexpr int kTrsvWarps = 8;

// Everything of one node that does not depend on other nodes' outputs.
template <typename T>
struct TrsvPre {
    const T* vp;  // the lane's neighbour's 3 values (nullptr: no neighbour)
    T a[9];       // 3x3 block of the node's rows against that neighbour
    T c[6];       // lane 0: rhs (3) and the node's own-block couplings (3)
    T s[3];       // lane 0 (upper): reciprocal pivots
    uint32_t n;
    int cnt;      // neighbours on this side
};

template <typename T>
__device__ __forceinline__ void load_block(const T* row, int rl, int k, T a[9]) {
#pragma unroll
    for (int p = 0; p < 3; ++p)
#pragma unroll
        for (int q = 0; q < 3; ++q) a[3 * p + q] = __ldg(row + (size_t)p * rl + 3 * k + q);
}

// forward: lane k < sk owns lower neighbour k
template <typename T>
__device__ __forceinline__ void pre_lower(const NodeSched& S, uint4 rec, const T* lu, const T* r,
                                          const T* z, int lane, TrsvPre<T>& P) {
    const uint32_t n = rec.x, nb0 = rec.y;
    const int deg = (int)rec.z, sk = (int)rec.w;
    const T* row = lu + 9 * (size_t)nb0;
    const int rl = 3 * deg, ds = 3 * sk;
    P.n = n;
    P.cnt = sk;
    P.vp = nullptr;
    if (lane < sk) {
        P.vp = z + 3 * (size_t)__ldg(S.nbr + nb0 + lane);
        load_block(row, rl, lane, P.a);
    }
    if (lane == 0) {
        P.c[0] = __ldg(r + 3 * (size_t)n);
        P.c[1] = __ldg(r + 3 * (size_t)n + 1);
        P.c[2] = __ldg(r + 3 * (size_t)n + 2);
        P.c[3] = __ldg(row + rl + ds);          // L(3n+1, 3n)
        P.c[4] = __ldg(row + 2 * rl + ds);      // L(3n+2, 3n)
        P.c[5] = __ldg(row + 2 * rl + ds + 1);  // L(3n+2, 3n+1)
    }
}

// backward: lane j < deg-sk-1 owns upper neighbour sk+1+j
template <typename T>
__device__ __forceinline__ void pre_upper(const NodeSched& S, uint4 rec, const T* lu,
                                          const T* dinv, const T* zin, const T* y, int lane,
                                          TrsvPre<T>& P) {
    const uint32_t n = rec.x, nb0 = rec.y;
    const int deg = (int)rec.z, sk = (int)rec.w;
    const T* row = lu + 9 * (size_t)nb0;
    const int rl = 3 * deg, ds = 3 * sk;
    P.n = n;
    P.cnt = deg - sk - 1;
    P.vp = nullptr;
    if (lane < P.cnt) {
        const int k = sk + 1 + lane;
        P.vp = y + 3 * (size_t)__ldg(S.nbr + nb0 + k);
        load_block(row, rl, k, P.a);
    }
    if (lane == 0) {
        const size_t b = 3 * (size_t)n;
        P.c[0] = zin[b];
        P.c[1] = zin[b + 1];
        P.c[2] = zin[b + 2];
        P.c[3] = __ldg(row + ds + 1);       // U(3n, 3n+1)
        P.c[4] = __ldg(row + ds + 2);       // U(3n, 3n+2)
        P.c[5] = __ldg(row + rl + ds + 2);  // U(3n+1, 3n+2)
        P.s[0] = __ldg(dinv + b);
        P.s[1] = __ldg(dinv + b + 1);
        P.s[2] = __ldg(dinv + b + 2);
    }
}

// Row sums sum_k A_k v_k of the node (valid in every lane).  The waits run
// in lock step (warp-uniform exit), so the butterfly that follows starts on
// a converged warp.
template <typename T>
__device__ __forceinline__ void block_sums(const TrsvPre<T>& P, unsigned* status,
                                           unsigned sleep_ns, int lane, T& s0, T& s1, T& s2) {
    (void)lane;
    T v0, v1, v2;
    wait_values3_warp(P.vp, status, sleep_ns, v0, v1, v2);
    s0 = s1 = s2 = T(0);
    if (P.vp) {
        s0 = P.a[0] * v0 + P.a[1] * v1 + P.a[2] * v2;
        s1 = P.a[3] * v0 + P.a[4] * v1 + P.a[5] * v2;
        s2 = P.a[6] * v0 + P.a[7] * v1 + P.a[8] * v2;
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        s0 += __shfl_xor_sync(kFull, s0, o);
        s1 += __shfl_xor_sync(kFull, s1, o);
        s2 += __shfl_xor_sync(kFull, s2, o);
    }
}

// z = L^-1 r, L unit lower (per node: z0, then z1 and z2 with the own block)
template <typename T>
__global__ void __launch_bounds__(kTrsvWarps * 32)
    k_trsv_lower_pipe(NodeSched S, const T* __restrict__ lu, const T* __restrict__ r,
                      T* __restrict__ z, unsigned* __restrict__ status, unsigned backoff) {
    const int lane = threadIdx.x & 31;
    const uint32_t W = (gridDim.x * blockDim.x) >> 5;
    uint32_t t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (t >= S.n_nodes) return;
    TrsvPre<T> cur, nxt;
    pre_lower(S, __ldg(S.fwd_rec + t), lu, r, z, lane, cur);
    uint4 rec_n = t + W < S.n_nodes ? __ldg(S.fwd_rec + t + W) : make_uint4(0, 0, 0, 0);
    for (;;) {
        const bool more = t + W < S.n_nodes;
        if (more) pre_lower(S, rec_n, lu, r, z, lane, nxt);
        if (t + 2 * W < S.n_nodes) rec_n = __ldg(S.fwd_rec + t + 2 * W);
        T s0, s1, s2;
        block_sums(cur, status, backoff, lane, s0, s1, s2);
        if (lane == 0) {
            const T z0 = cur.c[0] - s0;
            const T z1 = cur.c[1] - s1 - cur.c[3] * z0;
            const T z2 = cur.c[2] - s2 - cur.c[4] * z0 - cur.c[5] * z1;
            T* o = z + 3 * (size_t)cur.n;
            st_relaxed(o, z0);
            st_relaxed(o + 1, z1);
            st_relaxed(o + 2, z2);
        }
        if (!more) break;
        t += W;
        cur = nxt;
    }
}

// y = U^-1 z with reciprocal pivots (per node: y2, then y1 and y0)
template <typename T>
__global__ void __launch_bounds__(kTrsvWarps * 32)
    k_trsv_upper_pipe(NodeSched S, const T* __restrict__ lu, const T* __restrict__ dinv,
                      const T* __restrict__ zin, T* __restrict__ y, unsigned* __restrict__ status,
                      unsigned backoff) {
    const int lane = threadIdx.x & 31;
    const uint32_t W = (gridDim.x * blockDim.x) >> 5;
    uint32_t t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (t >= S.n_nodes) return;
    TrsvPre<T> cur, nxt;
    pre_upper(S, __ldg(S.bwd_rec + t), lu, dinv, zin, y, lane, cur);
    uint4 rec_n = t + W < S.n_nodes ? __ldg(S.bwd_rec + t + W) : make_uint4(0, 0, 0, 0);
    for (;;) {
        const bool more = t + W < S.n_nodes;
        if (more) pre_upper(S, rec_n, lu, dinv, zin, y, lane, nxt);
        if (t + 2 * W < S.n_nodes) rec_n = __ldg(S.bwd_rec + t + 2 * W);
        T s0, s1, s2;
        block_sums(cur, status, backoff, lane, s0, s1, s2);
        if (lane == 0) {
            const T y2 = (cur.c[2] - s2) * cur.s[2];
            const T y1 = (cur.c[1] - s1 - cur.c[5] * y2) * cur.s[1];
            const T y0 = (cur.c[0] - s0 - cur.c[3] * y1 - cur.c[4] * y2) * cur.s[0];
            T* o = y + 3 * (size_t)cur.n;
            st_relaxed(o, y0);
            st_relaxed(o + 1, y1);
            st_relaxed(o + 2, y2);
        }
        if (!more) break;
        t += W;
        cur = nxt;
    }
}

template <typename K>
static int resident_grid_trsv(K kernel, int device) {
    int sms = 0, per_sm = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kTrsvWarps * 32, 0);
    if (per_sm < 1) per_sm = 1;
    return sms * per_sm;
}

// Tuning (environment, read once): FM_TRSV_WARPS_PER_WIDTH = warps per 16
// nodes of the widest dependency level (default 24, i.e. 1.5x);
// FM_TRSV_BACKOFF_NS = longest sleep between a waiting warp's polls
// (default 0: plain spinning).  The grid never exceeds what can be resident at once:
// every warp must run for the waits to end.
static unsigned env_u(const char* name, unsigned dflt) {
    const char* v = getenv(name);
    return v ? (unsigned)strtoul(v, nullptr, 10) : dflt;
}
static int trsv_grid(int resident, uint32_t max_width) {
    static const unsigned per16 = env_u("FM_TRSV_WARPS_PER_WIDTH", 24);
    long want = ((long)per16 * max_width / 16 + kTrsvWarps - 1) / kTrsvWarps;
    if (want < 1) want = 1;
    return (int)(want < resident ? want : resident);
}

template <typename T>
void launch_trsv_nodes(const NodeSched& S, const T* lu, const T* dinv, const T* r, T* tmp, T* y,
                       unsigned* status, int device, cudaStream_t s) {
    if (!S.n_nodes) return;
    static int res_lo[2] = {0, 0}, res_up[2] = {0, 0};
    const int f = sizeof(T) == 4;
    if (!res_lo[f]) res_lo[f] = resident_grid_trsv(k_trsv_lower_pipe<T>, device);
    if (!res_up[f]) res_up[f] = resident_grid_trsv(k_trsv_upper_pipe<T>, device);
    static const unsigned backoff = env_u("FM_TRSV_BACKOFF_NS", 0);
    const uint32_t n = 3 * S.n_nodes;
    launch_fill_sentinel<T>(n, tmp, s);
    k_trsv_lower_pipe<T><<<trsv_grid(res_lo[f], S.max_width_fwd), kTrsvWarps * 32, 0, s>>>(
        S, lu, r, tmp, status, backoff);
    launch_fill_sentinel<T>(n, y, s);
    k_trsv_upper_pipe<T><<<trsv_grid(res_up[f], S.max_width_bwd), kTrsvWarps * 32, 0, s>>>(
        S, lu, dinv, tmp, y, status, backoff);
}

template void launch_trsv_nodes<double>(const NodeSched&, const double*, const double*,
                                        const double*, double*, double*, unsigned*, int,
                                        cudaStream_t);
template void launch_trsv_nodes<float>(const NodeSched&, const float*, const float*, const float*,
                                       float*, float*, unsigned*, int, cudaStream_t);

}  // namespace fm
