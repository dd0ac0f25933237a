// fm_trsv_cluster.cu — node-block ILU(0) triangular solves on one thread-
// block cluster, with the dependency values exchanged through distributed
// shared memory.
//
// The solves are latency-bound: 6N node levels (384 on the 64^3 block) run
// back to back, and through L2 every dependency hop costs ~0.4 us plus the
// node's own work.  Here the CTAs of one cluster (16 SMs where the device
// allows it, else 8) walk the levels:
//
//   * a node's three values go to a slot in its writer CTA's shared memory
//     (interval-allocated on the host); readers poll them with relaxed
//     ld.shared::cluster until no component is the wait sentinel (one
//     DSMEM round trip, ~0.1 us);
//   * every `window` levels a hardware cluster barrier closes the window;
//     after it each CTA resets the slots whose last reads fell in that
//     window to the sentinel, and the plan hands them out again from the
//     second window on, so a slot is never rewritten under a late reader;
//   * everything of a node that does not change between solves (schedule
//     record, its LU blocks on the solve's side, the neighbours' slots) is
//     packed after each factorization into 16-byte-aligned cards, ordered
//     by (level, warp), so that a warp's cards of one level are one
//     contiguous chunk: one bulk copy (cp.async.bulk, completion on an
//     mbarrier) per warp and level, issued D-1 levels ahead.  Only the
//     right-hand side (three values per node) is gathered per solve, with
//     cp.async.
//
// Warp gw = cta * warps_per_cta + w takes positions gw, gw + W, ... of each
// level (the plan of fm_setup.cpp cluster_plan); lane k owns the node's
// k-th neighbour on the solve's side.  Results equal the pipelined solves'
// up to the order of the per-node neighbour sum (a butterfly here).
#include <cooperative_groups.h>

#include "fm_kernels.hpp"
#include "fm_nodes.hpp"
#include "fm_setup.hpp"
#include "fm_cluster.cuh"
#include "fm_sync.cuh"

namespace fm {

namespace {

using namespace clu;

constexpr int kChunk = 3;  // nodes of one level a warp resolves together

// Packed card of one node (byte offsets; 16-byte multiple):
//   [0,16)    schedule record {node, first entry, deg | sk<<8 | cnt<<16, own slot}
//   h[6]      forward: L(1,0) L(2,0) L(2,1), unused(3)
//             backward: U(0,1) U(0,2) U(1,2), reciprocal pivots(3)
//   a[9*maxc] lane-major 3x3 blocks against the side's neighbours
//   slot[maxc] neighbour slots (cta << 16 | index)
template <typename T>
struct Card {
    static __host__ __device__ constexpr uint32_t h_off() { return 16; }
    static __host__ __device__ constexpr uint32_t a_off() { return 16 + 6 * sizeof(T); }
    static __host__ __device__ uint32_t s_off(uint32_t maxc) {
        return a_off() + 9 * maxc * sizeof(T);
    }
    static __host__ __device__ uint32_t bytes(uint32_t maxc) {
        return (s_off(maxc) + 4 * maxc + 15) & ~15u;
    }
};

// Bytes of the right-hand sides in one stage (3 values per card, 16-byte padded).
template <typename T>
__host__ __device__ inline uint32_t rhs_bytes(uint32_t mpw) {
    return (3 * mpw * (uint32_t)sizeof(T) + 15) & ~15u;
}

template <typename T, bool Lower>
__global__ void k_pack_cards(ClusterSolve P, const uint32_t* __restrict__ card_of_pos,
                             uint32_t n_pos, const T* __restrict__ lu,
                             const T* __restrict__ dinv, unsigned char* __restrict__ packed) {
    const int lane = threadIdx.x & 31;
    const uint32_t card = Card<T>::bytes(P.maxc);
    for (uint32_t p = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; p < n_pos;
         p += (gridDim.x * blockDim.x) >> 5) {
        const uint4 rec = __ldg(P.rec + p);
        unsigned char* cd = packed + (size_t)__ldg(card_of_pos + p) * card;
        const uint32_t n = rec.x, nb0 = rec.y;
        const uint32_t deg = rec.z & 0xff, sk = (rec.z >> 8) & 0xff, cnt = rec.z >> 16;
        const uint32_t rl = 3 * deg, ds = 3 * sk;
        const T* row = lu + 9 * (size_t)nb0;
        if (lane == 0) *reinterpret_cast<uint4*>(cd) = rec;
        T* h = reinterpret_cast<T*>(cd + Card<T>::h_off());
        if (lane < 3) {
            const uint32_t off = Lower ? (lane == 0 ? rl + ds : lane == 1 ? 2 * rl + ds : 2 * rl + ds + 1)
                                       : (lane == 0 ? ds + 1 : lane == 1 ? ds + 2 : rl + ds + 2);
            h[lane] = row[off];
        } else if (lane < 6) {
            h[lane] = Lower ? T(0) : dinv[3 * (size_t)n + lane - 3];
        }
        const uint32_t kb = Lower ? 0 : sk + 1;
        T* a = reinterpret_cast<T*>(cd + Card<T>::a_off());
        for (uint32_t v = lane; v < 9 * P.maxc; v += 32) {
            const uint32_t k = v / 9, pq = v - 9 * k, pr = pq / 3, q = pq - 3 * pr;
            a[v] = k < cnt ? row[pr * rl + 3 * (kb + k) + q] : T(0);
        }
        uint32_t* sl = reinterpret_cast<uint32_t*>(cd + Card<T>::s_off(P.maxc));
        if ((uint32_t)lane < P.maxc) sl[lane] = (uint32_t)lane < cnt ? __ldg(P.nslot + nb0 + kb + lane) : 0u;
    }
}

template <typename T, bool Lower, int D>
__global__ void __launch_bounds__(1024, 1)
    k_trsv_cluster(ClusterSolve P, const unsigned char* __restrict__ packed,
                   const T* __restrict__ rhs, T* __restrict__ out, unsigned* __restrict__ status) {
    extern __shared__ __align__(16) unsigned char smem[];
    namespace cg = cooperative_groups;
    cg::cluster_group cluster = cg::this_cluster();
    const uint32_t cta = cluster.block_rank();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const uint32_t W = P.n_ctas * P.warps_per_cta;
    const uint32_t gw = cta * P.warps_per_cta + w;
    constexpr uint32_t VS = sizeof(T) == 4 ? 16 : 32;  // slot bytes
    constexpr uint32_t VT = VS / sizeof(T);            // values per slot
    T* pool = reinterpret_cast<T*>(smem);
    const uint32_t pool_sa = smem_u32(smem);
    const uint32_t card = Card<T>::bytes(P.maxc);
    const uint32_t cards_bytes = card * P.max_per_warp;
    const uint32_t stage_bytes = cards_bytes + rhs_bytes<T>(P.max_per_warp);
    unsigned char* bars = smem + (size_t)P.pool_slots * VS;  // D mbarriers per warp
    unsigned char* stages = bars + 8 * D * P.warps_per_cta;
    unsigned char* my = stages + (size_t)w * D * stage_bytes;
    const uint32_t my_sa = smem_u32(my);
    const uint32_t bar_sa = smem_u32(bars) + 8 * D * w;

    for (uint32_t i = threadIdx.x; i < P.pool_slots * VT; i += blockDim.x)
        pool[i] = Sentinel<T>::value();
    if (lane == 0)
        for (int s = 0; s < D; ++s) mbar_init(bar_sa + 8 * s, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    cluster.sync();

    // this warp's nodes at a level: count m and first card c0
    auto level_info = [&](uint32_t l, uint32_t& m, uint32_t& c0) -> uint32_t {
        const uint32_t a = __ldg(P.lvl_ptr + l), b = __ldg(P.lvl_ptr + l + 1);
        m = b - a > gw ? (b - a - gw + W - 1) / W : 0;
        c0 = first_card(a, b - a, W, gw);
        return a;
    };
    // node id of this warp's j-th node of level l in lane j < m
    auto load_nodes = [&](uint32_t l, uint32_t& m) -> uint32_t {
        uint32_t node = 0, c0;
        m = 0;
        if (l < P.n_levels) {
            const uint32_t a = level_info(l, m, c0);
            if ((uint32_t)lane < m) node = __ldg(&P.rec[a + gw + lane * W].x);
        }
        return node;
    };
    // stage of level l: one bulk copy of the cards, cp.async of the rhs
    auto issue = [&](uint32_t l, uint32_t node, uint32_t m) {
        if (l < P.n_levels && m > 0) {
            uint32_t mm, c0;
            level_info(l, mm, c0);
            const uint32_t st = my_sa + (l % D) * stage_bytes;
            if (lane == 0) {
                const uint32_t bar = bar_sa + 8 * (l % D);
                // the stage's previous cards were read through the generic proxy
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                mbar_expect_tx(bar, m * card);
                bulk_g2s(st, packed + (size_t)c0 * card, m * card, bar);
            }
            if ((uint32_t)lane < m)
#pragma unroll
                for (int i = 0; i < 3; ++i)
                    cp_async_val(st + cards_bytes + (3 * lane + i) * sizeof(T),
                                 rhs + 3 * (size_t)node + i);
        }
        cp_async_commit();
    };

    // prologue: stages of levels 0 .. D-2, node ids of level D-1
    for (uint32_t l = 0; l + 1 < D; ++l) {
        uint32_t m;
        const uint32_t nd = load_nodes(l, m);
        issue(l, nd, m);
    }
    uint32_t m_next;
    uint32_t node_next = load_nodes(D - 1, m_next);
    uint32_t phase = 0;  // bit s: parity of stage s's next phase

    for (uint32_t l = 0; l < P.n_levels; ++l) {
        issue(l + D - 1, node_next, m_next);
        node_next = load_nodes(l + D, m_next);
        uint32_t m, c0;
        level_info(l, m, c0);
        const uint32_t s = l % D;
        if (m > 0) {
            mbar_wait(bar_sa + 8 * s, (phase >> s) & 1u, status);
            phase ^= 1u << s;
        }
        cp_async_wait<D - 1>();
        __syncwarp();
        const unsigned char* st = my + s * stage_bytes;
        const T* rh = reinterpret_cast<const T*>(st + cards_bytes);
        for (uint32_t j0 = 0; j0 < m; j0 += kChunk) {
            // the chunk's dependency values: lane k polls neighbour k of each
            // node; the loop runs in lock step (its exit is warp-uniform), so
            // the warp never splits into separately spinning lanes, whose
            // reconvergence before the shuffles costs microseconds
            T v[kChunk][3];
            uint32_t addr[kChunk];
            bool need[kChunk];
#pragma unroll
            for (int c = 0; c < kChunk; ++c) {
                const uint32_t j = j0 + c;
                need[c] = false;
                addr[c] = 0;
                if (j < m) {
                    const unsigned char* cd = st + j * card;
                    const uint32_t cnt = reinterpret_cast<const uint4*>(cd)->z >> 16;
                    if ((uint32_t)lane < cnt) {
                        const uint32_t sl =
                            reinterpret_cast<const uint32_t*>(cd + Card<T>::s_off(P.maxc))[lane];
                        addr[c] = mapa(pool_sa + (sl & 0xffffu) * VS, sl >> 16);
                        need[c] = true;
                    }
                }
                v[c][0] = v[c][1] = v[c][2] = T(0);
            }
            const long long t0 = clock64();
            for (unsigned it = 0;; ++it) {
                bool ready = true;
#pragma unroll
                for (int c = 0; c < kChunk; ++c)
                    if (need[c]) {
                        ld_slot<T>(addr[c], v[c][0], v[c][1], v[c][2]);
                        need[c] = Sentinel<T>::is(v[c][0]) | Sentinel<T>::is(v[c][1]) |
                                  Sentinel<T>::is(v[c][2]);
                        ready &= !need[c];
                    }
                if (__all_sync(0xffffffffu, ready)) break;
                if ((it & 63u) == 63u &&
                    __any_sync(0xffffffffu, (ld_volatile_u32(status) & FM_FLAG_TIMEOUT) ||
                                                clock64() - t0 > kWaitCycles)) {
                    if (lane == 0) raise_flag(status, FM_FLAG_TIMEOUT);
                    break;
                }
            }
            T part[kChunk][3];
#pragma unroll
            for (int c = 0; c < kChunk; ++c) {
                const uint32_t j = j0 + c;
                part[c][0] = part[c][1] = part[c][2] = T(0);
                const unsigned char* cd = st + (j < m ? j : 0) * card;
                const uint32_t cnt = j < m ? reinterpret_cast<const uint4*>(cd)->z >> 16 : 0;
                if ((uint32_t)lane < cnt) {
                    const T* a = reinterpret_cast<const T*>(cd + Card<T>::a_off()) + 9 * lane;
                    part[c][0] = a[0] * v[c][0] + a[1] * v[c][1] + a[2] * v[c][2];
                    part[c][1] = a[3] * v[c][0] + a[4] * v[c][1] + a[5] * v[c][2];
                    part[c][2] = a[6] * v[c][0] + a[7] * v[c][1] + a[8] * v[c][2];
                }
            }
#pragma unroll
            for (int o = 16; o; o >>= 1)
#pragma unroll
                for (int c = 0; c < kChunk; ++c)
#pragma unroll
                    for (int q = 0; q < 3; ++q)
                        part[c][q] += __shfl_xor_sync(0xffffffffu, part[c][q], o);
#pragma unroll
            for (int c = 0; c < kChunk; ++c) {
                const uint32_t j = j0 + c;
                if (lane == c && j < m) {
                    const unsigned char* cd = st + j * card;
                    const uint4 rec = *reinterpret_cast<const uint4*>(cd);
                    const T* h = reinterpret_cast<const T*>(cd + Card<T>::h_off());
                    const T* r = rh + 3 * j;
                    T x0, x1, x2;
                    if constexpr (Lower) {
                        x0 = r[0] - part[c][0];
                        x1 = r[1] - part[c][1] - h[0] * x0;
                        x2 = r[2] - part[c][2] - h[1] * x0 - h[2] * x1;
                    } else {
                        x2 = (r[2] - part[c][2]) * h[5];
                        x1 = (r[1] - part[c][1] - h[2] * x2) * h[4];
                        x0 = (r[0] - part[c][0] - h[0] * x1 - h[1] * x2) * h[3];
                    }
                    st_slot<T>(pool_sa + rec.w * VS, x0, x1, x2);
                    T* o = out + 3 * (size_t)rec.x;
                    o[0] = x0;
                    o[1] = x1;
                    o[2] = x2;
                }
            }
        }
        __syncwarp();
        if ((l + 1) % P.window == 0 || l + 1 == P.n_levels) {
            // close the window; then reset the slots whose last reads were in it
            // (handed out again two windows later, after the next barrier)
            cluster_barrier();
            const uint32_t t = l / P.window;
            const uint32_t r0 = __ldg(P.reset_ptr + t * P.n_ctas + cta);
            const uint32_t r1 = __ldg(P.reset_ptr + t * P.n_ctas + cta + 1);
            for (uint32_t i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
                const uint32_t a = pool_sa + __ldg(P.reset + i) * VS;
                st_slot<T>(a, Sentinel<T>::value(), Sentinel<T>::value(), Sentinel<T>::value());
            }
        }
    }
    cp_async_wait<0>();
}

template <typename K>
static int max_clusters(K kernel, int cs, size_t smem) {
    if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
            cudaSuccess ||
        (cs > 8 &&
         cudaFuncSetAttribute(kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) !=
             cudaSuccess)) {
        cudaGetLastError();
        return 0;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(cs);
    cfg.blockDim = dim3(1024);
    cfg.dynamicSmemBytes = smem;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = cs;
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

template <typename T, bool Lower, int D>
static cudaError_t launch_one(const ClusterSolve& P, const unsigned char* packed, const T* rhs,
                              T* out, unsigned* status, cudaStream_t s) {
    auto kern = k_trsv_cluster<T, Lower, D>;
    const size_t smem = cluster_smem_bytes(P, sizeof(T), D);
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    if (P.n_ctas > 8) {
        e = cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
        if (e != cudaSuccess) return e;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(P.n_ctas);
    cfg.blockDim = dim3(32 * P.warps_per_cta);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = P.n_ctas;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kern, P, packed, rhs, out, status);
}

}  // namespace

size_t cluster_card_bytes(const ClusterSolve& P, size_t value_bytes) {
    return value_bytes == 4 ? Card<float>::bytes(P.maxc) : Card<double>::bytes(P.maxc);
}

size_t cluster_smem_bytes(const ClusterSolve& P, size_t value_bytes, int stages) {
    const size_t card = cluster_card_bytes(P, value_bytes);
    const size_t slot = value_bytes == 4 ? 16 : 32;
    const size_t rhs = value_bytes == 4 ? rhs_bytes<float>(P.max_per_warp)
                                        : rhs_bytes<double>(P.max_per_warp);
    return P.pool_slots * slot + 8 * (size_t)stages * P.warps_per_cta +
           (size_t)P.warps_per_cta * stages * (P.max_per_warp * card + rhs);
}

int cluster_stages(size_t value_bytes) { return value_bytes == 4 ? 3 : 2; }

int cluster_max_active(size_t value_bytes, int cs, size_t smem) {
    // the forward and backward kernels of one width share their resources
    if (value_bytes == 4) return max_clusters(k_trsv_cluster<float, true, 3>, cs, smem);
    return max_clusters(k_trsv_cluster<double, true, 2>, cs, smem);
}

template <typename T>
void launch_pack_cards(const ClusterSolve& F, const ClusterSolve& B, const uint32_t* card_f,
                       const uint32_t* card_b, uint32_t n_pos, const T* lu, const T* dinv,
                       unsigned char* packed_f, unsigned char* packed_b, cudaStream_t s) {
    if (!n_pos) return;
    unsigned grid = (n_pos + 7) / 8;
    if (grid > 4736) grid = 4736;
    k_pack_cards<T, true><<<grid, 256, 0, s>>>(F, card_f, n_pos, lu, dinv, packed_f);
    k_pack_cards<T, false><<<grid, 256, 0, s>>>(B, card_b, n_pos, lu, dinv, packed_b);
}

template <typename T>
cudaError_t launch_trsv_cluster(const ClusterSolve& F, const ClusterSolve& B,
                                const unsigned char* packed_f, const unsigned char* packed_b,
                                const T* r, T* tmp, T* y, unsigned* status, cudaStream_t s) {
    constexpr int D = sizeof(T) == 4 ? 3 : 2;
    cudaError_t e = launch_one<T, true, D>(F, packed_f, r, tmp, status, s);
    if (e != cudaSuccess) return e;
    return launch_one<T, false, D>(B, packed_b, tmp, y, status, s);
}

template void launch_pack_cards<float>(const ClusterSolve&, const ClusterSolve&, const uint32_t*,
                                       const uint32_t*, uint32_t, const float*, const float*,
                                       unsigned char*, unsigned char*, cudaStream_t);
template void launch_pack_cards<double>(const ClusterSolve&, const ClusterSolve&,
                                        const uint32_t*, const uint32_t*, uint32_t,
                                        const double*, const double*, unsigned char*,
                                        unsigned char*, cudaStream_t);
template cudaError_t launch_trsv_cluster<float>(const ClusterSolve&, const ClusterSolve&,
                                                const unsigned char*, const unsigned char*,
                                                const float*, float*, float*, unsigned*,
                                                cudaStream_t);
template cudaError_t launch_trsv_cluster<double>(const ClusterSolve&, const ClusterSolve&,
                                                 const unsigned char*, const unsigned char*,
                                                 const double*, double*, double*, unsigned*,
                                                 cudaStream_t);

}  // namespace fm
