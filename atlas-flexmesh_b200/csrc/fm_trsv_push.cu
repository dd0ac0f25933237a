// fm_trsv_push.cu — node-block ILU(0) triangular solves on a slab partition
// of the nodes, with the dependency values pushed into the readers' shared
// memory inside each thread-block cluster.
//
// Both solves are chains of dependency levels (6N node levels each on the
// N^3 block); in the grid-wide solves (fm_trsv.cu) every hop of the chain
// is a value stored to L2 and polled back by another SM, ~0.43 us of the
// ~0.92 us a level costs.  Here the node range is cut into one contiguous
// slab per cluster (9 CTAs on B200, one per SM), whose blocks of consecutive nodes
// are dealt round-robin to the cluster's CTAs (so that each CTA holds a
// share of every level).  The forward solve only waits on lower-numbered
// nodes and the backward on higher-numbered ones, so any dependency chain
// leaves a slab at most (clusters - 1) times; every other hop stays inside
// a cluster:
//
//   * the producing warp stores the node's three values, with one relaxed
//     cluster-scope vector store per reading CTA, into a slot of that CTA's
//     shared memory (one slot per producer and reading CTA, planned on the
//     host, never reused), and its reader polls its own shared memory;
//   * values that cross slabs, and every output, go to global memory as in
//     the grid-wide solves (outputs pre-filled with the wait sentinel);
//   * slots are filled with the sentinel before a cluster barrier that
//     precedes every push, and a second barrier keeps every CTA resident
//     until no store into its shared memory can still be in flight.
//
// Each CTA walks its nodes in level order; a warp resolves two nodes at a
// time, one per half-warp, and lane k of a half owns the node's k-th
// neighbour on the solve's side (at most 16; meshes with more keep the
// grid-wide solves).  The host pads every CTA's level runs with holes so
// that the two nodes of a warp never belong to different levels: neither
// then waits on the other, and the waits of both halves run in lock step
// (one warp vote), ending in butterflies inside each half.  The next pair's
// records (batched 16 per half-warp, a batch ahead, handed out by
// shuffles), LU blocks, slots and destinations are in flight while the
// warp waits.  The per-node arithmetic is that of fm_trsv.cu term for term
// (lanes without a neighbour add zeros), so both paths give the same values.
//
// Measured on B200 at 64^3 x 6 tets, FP32 (per forward+backward pair):
// 0.716 ms grid-wide, 0.444 ms here with 32 warps per CTA (FP64: 0.806 ->
// 0.691 ms with 16).  A per-node %globaltimer trace of the critical path
// (384 nodes per direction) splits a level into the hop (last dependency
// pushed -> the reader's wait ends, ~300 ns, set by the poll round: ~150 ns
// per round when the warp polls shared memory only, ~500 ns when a lane
// polls L2) and the node's own work (wait end -> push, ~260 ns: products,
// four butterfly rounds, finish, stores).  Two nodes per warp halved the
// per-node work of a one-node-per-warp build.
//
// The backward solve runs its slabs in reverse block order (the top slab on
// the first clusters), so in both directions clusters only wait on clusters
// launched before them.
#include <algorithm>

#include "fm_cluster.cuh"
#include "fm_kernels.hpp"
#include "fm_nodes.hpp"
#include "fm_setup.hpp"
#include "fm_sync.cuh"

namespace fm {

namespace {

using namespace clu;

template <typename T>
constexpr uint32_t kSlotBytes = sizeof(T) == 4 ? 16u : 32u;

// Everything of one node that does not depend on other nodes' outputs, as
// held by the lanes of the half-warp that takes it.  Loaded values are kept
// raw (slot, neighbour, push entry) and resolved when used, so issuing a
// node's loads never waits for any of them.
template <typename T>
struct PushPre {
    T a[9];        // 3x3 block of the node's rows against the lane's neighbour
    T c[6];        // rhs (3) and the node's own-block couplings (3)
    T s[3];        // backward: reciprocal pivots
    uint32_t sv;   // hl < cnt: the neighbour's slot in this CTA, ~0u: in global memory
    uint32_t nb;   // hl < cnt: the neighbour
    uint32_t pe;   // hl < kPushMax: rank << 20 | slot of a reading CTA, ~0u: none
    uint32_t n;    // the node, ~0u: the half-warp has no node at this step
    int cnt;       // neighbours on the solve's side
};

// hl: lane within the half-warp
template <typename T, bool Lower>
__device__ __forceinline__ void push_pre(const PushSolve& P, const NodeSched& S, bool valid,
                                         uint4 rec, const T* lu, const T* dinv, const T* rhs,
                                         int hl, PushPre<T>& Q) {
    Q.n = ~0u;
    Q.cnt = 0;
    Q.sv = ~0u;
    Q.nb = 0;
    Q.pe = ~0u;
    if (!valid || rec.x == ~0u) return;  // no position, or a hole
    const uint32_t n = rec.x, nb0 = rec.y;
    const int deg = (int)rec.z, sk = (int)rec.w;
    const T* row = lu + 9 * (size_t)nb0;
    const int rl = 3 * deg, ds = 3 * sk;
    const int cnt = Lower ? sk : deg - sk - 1;
    Q.n = n;
    Q.cnt = cnt;
    if (hl < cnt) {
        const int k = Lower ? hl : sk + 1 + hl;
        const uint32_t e = nb0 + (uint32_t)k;
        Q.sv = __ldg(P.src + e);
        Q.nb = __ldg(S.nbr + e);
#pragma unroll
        for (int p = 0; p < 3; ++p)
#pragma unroll
            for (int q = 0; q < 3; ++q) Q.a[3 * p + q] = __ldg(row + (size_t)p * rl + 3 * k + q);
    }
    const size_t b = 3 * (size_t)n;
    Q.c[0] = __ldg(rhs + b);
    Q.c[1] = __ldg(rhs + b + 1);
    Q.c[2] = __ldg(rhs + b + 2);
    if (Lower) {
        Q.c[3] = __ldg(row + rl + ds);          // L(3n+1, 3n)
        Q.c[4] = __ldg(row + 2 * rl + ds);      // L(3n+2, 3n)
        Q.c[5] = __ldg(row + 2 * rl + ds + 1);  // L(3n+2, 3n+1)
    } else {
        Q.c[3] = __ldg(row + ds + 1);       // U(3n, 3n+1)
        Q.c[4] = __ldg(row + ds + 2);       // U(3n, 3n+2)
        Q.c[5] = __ldg(row + rl + ds + 2);  // U(3n+1, 3n+2)
        Q.s[0] = __ldg(dinv + b);
        Q.s[1] = __ldg(dinv + b + 1);
        Q.s[2] = __ldg(dinv + b + 2);
    }
    if (hl < (int)kPushMax)
        Q.pe = __ldg((Lower ? P.push_f : P.push_b) + (size_t)n * kPushMax + hl);
}

// Bounded lock-step wait for the lane's neighbour's three values, from this
// CTA's shared memory (sl) or from global memory (gp; neither: no
// neighbour).  On a timeout FM_FLAG_TIMEOUT is set and the values may
// still be sentinels.  When no lane of the warp reads global memory (three
// warp steps in four at 64^3), every lane runs the same branch-free loop of
// shared-memory polls, lanes without a neighbour on zero, a slot that
// always holds zeros: the per-lane branches of the general loop doubled the
// time of a poll round (about 150 against 320 ns in a %globaltimer trace).
template <typename T>
__device__ __forceinline__ void wait_push(uint32_t sl, const T* gp, uint32_t zero,
                                          unsigned* status, unsigned m, T& v0, T& v1, T& v2) {
    if (!__any_sync(m, gp != nullptr)) {
        const uint32_t a = sl != ~0u ? sl : zero;
        ld_slot_cta(a, v0, v1, v2);
        bool need = Sentinel<T>::is(v0) | Sentinel<T>::is(v1) | Sentinel<T>::is(v2);
        if (!__any_sync(m, need)) return;
        const long long t0 = clock64(), limit = wait_limit(status);
        for (unsigned it = 1;; ++it) {
            ld_slot_cta(a, v0, v1, v2);
            need = Sentinel<T>::is(v0) | Sentinel<T>::is(v1) | Sentinel<T>::is(v2);
            if (!__any_sync(m, need)) return;
            if ((it & 255u) == 0 &&
                __any_sync(m, (ld_volatile_u32(status) & FM_FLAG_TIMEOUT) ||
                                  clock64() - t0 > limit)) {
                if ((threadIdx.x & 15) == 0) raise_flag(status, FM_FLAG_TIMEOUT);
                return;
            }
        }
    }
    v0 = v1 = v2 = T(0);
    auto poll = [&]() {
        if (sl != ~0u) {
            ld_slot_cta(sl, v0, v1, v2);
        } else {
            if (Sentinel<T>::is(v0)) v0 = ld_relaxed(gp);
            if (Sentinel<T>::is(v1)) v1 = ld_relaxed(gp + 1);
            if (Sentinel<T>::is(v2)) v2 = ld_relaxed(gp + 2);
        }
        return Sentinel<T>::is(v0) | Sentinel<T>::is(v1) | Sentinel<T>::is(v2);
    };
    bool need = sl != ~0u || gp != nullptr;
    if (need) {
        v0 = v1 = v2 = Sentinel<T>::value();
        need = poll();
    }
    if (!__any_sync(m, need)) return;
    const long long t0 = clock64(), limit = wait_limit(status);
    for (unsigned it = 1;; ++it) {
        if (need) need = poll();
        if (!__any_sync(m, need)) return;
        // shared-memory polls are short: look at the clock and the grid's
        // timeout flag every 256 rounds
        if ((it & 255u) == 0 &&
            __any_sync(m, (ld_volatile_u32(status) & FM_FLAG_TIMEOUT) ||
                              clock64() - t0 > limit)) {
            if ((threadIdx.x & 15) == 0) raise_flag(status, FM_FLAG_TIMEOUT);
            return;
        }
    }
}

// The half-warps' two nodes once their loads are in Q: wait (both halves in
// lock step), sum, finish, push.  The butterfly stays inside each half and
// runs only over the lanes that can hold neighbours (8 or 16, the same for
// the whole warp); the other lanes hold zeros, so the sums are those of a
// full butterfly.  Lanes hl < kPushMax of each half hold its results.
// zero: a slot of this CTA that always holds zeros.
template <typename T, bool Lower>
__device__ __forceinline__ void push_node(const PushPre<T>& Q, uint32_t base, uint32_t zero,
                                          T* out, unsigned* status, int hl, unsigned m) {
    const bool has = hl < Q.cnt;
    const bool local = has && Q.sv != ~0u;
    // resolved before the wait, off the chain: the reading CTA's slot address
    // and the butterfly's width
    const uint32_t pa =
        Q.pe != ~0u ? mapa(base + (Q.pe & 0xfffffu) * kSlotBytes<T>, Q.pe >> 20) : 0u;
    const bool wide = __any_sync(m, Q.cnt > 8);
    T v0, v1, v2;
    wait_push<T>(local ? base + Q.sv * kSlotBytes<T> : ~0u,
                 has && !local ? out + 3 * (size_t)Q.nb : nullptr, zero, status, m, v0, v1,
                 v2);
    T s0 = T(0), s1 = T(0), s2 = T(0);
    if (has) {
        s0 = Q.a[0] * v0 + Q.a[1] * v1 + Q.a[2] * v2;
        s1 = Q.a[3] * v0 + Q.a[4] * v1 + Q.a[5] * v2;
        s2 = Q.a[6] * v0 + Q.a[7] * v1 + Q.a[8] * v2;
    }
    if (wide) {
        s0 += __shfl_xor_sync(m, s0, 8);
        s1 += __shfl_xor_sync(m, s1, 8);
        s2 += __shfl_xor_sync(m, s2, 8);
    }
#pragma unroll
    for (int o = 4; o; o >>= 1) {
        s0 += __shfl_xor_sync(m, s0, o);
        s1 += __shfl_xor_sync(m, s1, o);
        s2 += __shfl_xor_sync(m, s2, o);
    }
    if (Q.n == ~0u) return;
    T x0, x1, x2;
    if (Lower) {
        x0 = Q.c[0] - s0;
        x1 = Q.c[1] - s1 - Q.c[3] * x0;
        x2 = Q.c[2] - s2 - Q.c[4] * x0 - Q.c[5] * x1;
    } else {
        x2 = (Q.c[2] - s2) * Q.s[2];
        x1 = (Q.c[1] - s1 - Q.c[5] * x2) * Q.s[1];
        x0 = (Q.c[0] - s0 - Q.c[3] * x1 - Q.c[4] * x2) * Q.s[0];
    }
    if (Q.pe != ~0u) st_slot_cluster(pa, x0, x1, x2);
    if (hl == 0) {
        T* o = out + 3 * (size_t)Q.n;
        st_relaxed(o, x0);
        st_relaxed(o + 1, x1);
        st_relaxed(o + 2, x2);
    }
}

__device__ __forceinline__ uint4 shfl4(uint4 v, int src, unsigned m) {
    return make_uint4(__shfl_sync(m, v.x, src), __shfl_sync(m, v.y, src),
                      __shfl_sync(m, v.z, src), __shfl_sync(m, v.w, src));
}

// One direction.  fill/n_fill: a vector the kernel sets to the wait
// sentinel once its CTA is done (the forward solve prepares the backward's
// output this way).
template <typename T, bool Lower>
__global__ void __launch_bounds__(push_max_warps(sizeof(T)) * 32, 1)
    k_trsv_push(PushSolve P, NodeSched S, const T* __restrict__ lu, const T* __restrict__ dinv,
                const T* __restrict__ rhs, T* __restrict__ out, T* __restrict__ fill,
                uint32_t n_fill, unsigned* __restrict__ status) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ __align__(16) T zero_slot[4];
    T* slots = reinterpret_cast<T*>(smem_raw);
    if (threadIdx.x < 4) zero_slot[threadIdx.x] = T(0);
    const uint32_t cs = P.cluster, n_cl = P.n_ctas / cs;
    const uint32_t cl = blockIdx.x / cs, rank = blockIdx.x % cs;
    const uint32_t g = (Lower ? cl : n_cl - 1 - cl) * cs + rank;
    const uint32_t ns = Lower ? P.nslot_f[g] : P.nslot_b[g];
    for (uint32_t i = threadIdx.x; i < 4 * ns; i += blockDim.x) slots[i] = Sentinel<T>::value();
    cluster_barrier();  // every slot of the cluster holds the sentinel before any push

    const uint32_t base = smem_u32(slots);
    const int lane = threadIdx.x & 31, hl = lane & 15;
    // half-warp v = 2 * warp + half takes positions beg + v, beg + v + H, ...
    const uint32_t H = blockDim.x >> 4;
    const uint32_t* pos = Lower ? P.pos_f : P.pos_b;
    const uint32_t beg = pos[g], end = pos[g + 1];
    const uint32_t v0 = 2 * (threadIdx.x >> 5), v = v0 + (uint32_t)(lane >> 4);
    const uint4* rec = Lower ? P.rec_f : P.rec_b;
    const unsigned m = kFull;  // both halves vote and shuffle over the whole warp
    if (beg + v0 < end) {
        // steps of the warp: the first half's count (it starts first)
        const uint32_t nq = (end - beg - v0 + H - 1) / H;
        const uint32_t mine = beg + v < end ? (end - beg - v + H - 1) / H : 0;
        // records come 16 per half-warp, one per lane, a batch ahead of use,
        // and are handed out by shuffles: no record load is ever waited on
        const uint4 zero = make_uint4(0, 0, 0, 0);
        auto batch = [&](uint32_t b) {
            const uint32_t q = 16 * b + (uint32_t)hl;
            return q < mine ? __ldg(rec + beg + v + q * H) : zero;
        };
        uint4 ba = batch(0), bb = batch(1);
        // record q of this half's batch cb or cb + 1
        auto rec_of = [&](uint32_t q, uint32_t cb) {
            return shfl4((q >> 4) == cb ? ba : bb, (lane & 16) | (int)(q & 15), m);
        };
        if constexpr (sizeof(T) == 4) {
            // FP32: one node's loads at a time, issued when the warp reaches
            // the node (a warp's consecutive nodes are mostly several levels
            // apart); the registers this frees give 32 warps per CTA instead
            // of 24 (0.444 against 0.467 ms per pair at 64^3)
            for (uint32_t q = 0; q < nq; ++q) {
                PushPre<T> qa;
                push_pre<T, Lower>(P, S, q < mine, rec_of(q, q >> 4), lu, dinv, rhs, hl, qa);
                push_node<T, Lower>(qa, base, smem_u32(zero_slot), out, status, hl, m);
                if (((q + 1) & 15) == 0 && q + 1 < nq) {
                    ba = bb;
                    bb = batch(((q + 1) >> 4) + 1);
                }
            }
        } else {
            // FP64: the next node's loads in flight while the warp waits on
            // the current one (single-buffered at 20 or 24 warps it was
            // slower than this at 16)
            PushPre<T> qa, qb;
            push_pre<T, Lower>(P, S, 0 < mine, rec_of(0, 0), lu, dinv, rhs, hl, qa);
            uint32_t q = 0;
            // cur is processed while nxt's loads are in flight; the two swap
            // roles every step (no register copies that would wait on them)
            auto step = [&](const PushPre<T>& cur, PushPre<T>& nxt) {
                const uint32_t cb = q >> 4;
                const bool more = q + 1 < nq;
                if (more)
                    push_pre<T, Lower>(P, S, q + 1 < mine, rec_of(q + 1, cb), lu, dinv, rhs, hl,
                                       nxt);
                push_node<T, Lower>(cur, base, smem_u32(zero_slot), out, status, hl, m);
                ++q;
                if ((q & 15) == 0 && more) {
                    ba = bb;
                    bb = batch((q >> 4) + 1);
                }
                return more;
            };
            for (;;) {
                if (!step(qa, qb)) break;
                if (!step(qb, qa)) break;
            }
        }
    }
    if (n_fill) {
        const T sv = Sentinel<T>::value();
        for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n_fill;
             i += gridDim.x * blockDim.x)
            fill[i] = sv;
    }
    cluster_barrier();  // no CTA leaves while a store into its slots may be in flight
}

template <typename K>
static void allow_smem(K kernel, size_t smem) {
    if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
        cudaSuccess)
        cudaGetLastError();
    // clusters of 9 CTAs are above the portable size of 8
    if (cudaFuncSetAttribute(kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) !=
        cudaSuccess)
        cudaGetLastError();
}

template <typename K>
static int max_clusters(K kernel, int cluster, int warps, size_t smem) {
    allow_smem(kernel, smem);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(cluster);
    cfg.blockDim = dim3(32 * warps);
    cfg.dynamicSmemBytes = smem;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = cluster;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    int n = 0;
    if (cudaOccupancyMaxActiveClusters(&n, kernel, &cfg) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

template <typename T, bool Lower>
static cudaError_t launch_dir(const PushSolve& P, const NodeSched& S, const T* lu, const T* dinv,
                              const T* rhs, T* out, T* fill, uint32_t n_fill, unsigned* status,
                              cudaStream_t s) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(P.n_ctas);
    cfg.blockDim = dim3(32 * (sizeof(T) == 4 ? P.warps32 : P.warps64));
    cfg.dynamicSmemBytes = push_smem_bytes(Lower ? P.max_slot_f : P.max_slot_b, sizeof(T));
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = P.cluster;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, k_trsv_push<T, Lower>, P, S, lu, dinv, rhs, out, fill, n_fill,
                              status);
}

}  // namespace

size_t push_smem_bytes(uint32_t max_slot, size_t value_bytes) {
    return (size_t)std::max(max_slot, 1u) * (value_bytes == 4 ? 16 : 32);
}

int push_max_clusters(size_t value_bytes, int cluster, int warps, size_t smem) {
    if (warps < 1 || warps > push_max_warps(value_bytes) || cluster < 1 ||
        cluster > (int)kPushMax)
        return 0;
    // raises each kernel's dynamic shared memory limit to smem, so every later
    // launch up to that size is accepted
    if (value_bytes == 4)
        return std::min(max_clusters(k_trsv_push<float, true>, cluster, warps, smem),
                        max_clusters(k_trsv_push<float, false>, cluster, warps, smem));
    return std::min(max_clusters(k_trsv_push<double, true>, cluster, warps, smem),
                    max_clusters(k_trsv_push<double, false>, cluster, warps, smem));
}

template <typename T>
cudaError_t launch_trsv_push(const PushSolve& P, const NodeSched& S, const T* lu, const T* dinv,
                             const T* r, T* tmp, T* y, unsigned* status, cudaStream_t s) {
    if (!S.n_nodes) return cudaSuccess;
    const uint32_t n = 3 * S.n_nodes;
    launch_fill_sentinel<T>(n, tmp, s);
    // in place (y == r) the forward solve still reads r: fill y after it
    const bool fuse = y != r;
    cudaError_t e =
        launch_dir<T, true>(P, S, lu, dinv, r, tmp, fuse ? y : nullptr, fuse ? n : 0, status, s);
    if (e != cudaSuccess) return e;
    if (!fuse) launch_fill_sentinel<T>(n, y, s);
    return launch_dir<T, false>(P, S, lu, dinv, tmp, y, nullptr, 0, status, s);
}

template cudaError_t launch_trsv_push<double>(const PushSolve&, const NodeSched&, const double*,
                                              const double*, const double*, double*, double*,
                                              unsigned*, cudaStream_t);
template cudaError_t launch_trsv_push<float>(const PushSolve&, const NodeSched&, const float*,
                                             const float*, const float*, float*, float*,
                                             unsigned*, cudaStream_t);

}  // namespace fm
