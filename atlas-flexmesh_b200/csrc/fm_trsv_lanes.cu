// fm_trsv_lanes.cu — node-block ILU(0) triangular solves on one thread-block
// cluster, one lane per node.
//
// The solves are a chain of 6N dependency levels (384 on the 64^3 block).
// The grid-wide solves (fm_trsv.cu) pay one L2 round trip per level (~0.4
// us); the warp-per-node cluster solves (fm_trsv_cluster.cu) cut the hop to
// a DSMEM load but leave each warp 1-3 nodes of work per level.  Here a
// level's nodes are cut into groups of 32 and a warp resolves a whole group
// at once, one node per lane: the lane polls its (at most MAXC) dependency
// slots in distributed shared memory, forms the 3x3 block products against
// them (81 FMAs for 9 neighbours) and substitutes through its own 3x3
// block, with no cross-lane reduction.  Groups go round-robin to the
// cluster's warps, so a level needs ~width/32 warps and a warp meets its
// next group several levels later: its card for that group (the node ids,
// neighbour slots, the L or U blocks, lane-major so every shared-memory read
// of the group is conflict-free) is packed after each factorization and
// fetched by one bulk copy long before it is needed; the right-hand side
// comes with it by cp.async.
//
// Value slots, windows, cluster barriers and slot resets are those of
// fm_trsv_cluster.cu (plan: fm_setup.cpp cluster_plan in lane-group mode).
#include <cooperative_groups.h>

#include "fm_cluster.cuh"
#include "fm_kernels.hpp"
#include "fm_nodes.hpp"
#include "fm_setup.hpp"
#include "fm_sync.cuh"

namespace fm {

namespace {

using namespace clu;

constexpr int kLaneMaxC = 12;  // neighbours per side a lane resolves

// Group card (lane-major; every block a multiple of 128 bytes):
//   node[32] | own slot[32] | cnt[32] | slot[maxc][32] | h[6][32] | a[9 maxc][32]
// h: forward L(1,0) L(2,0) L(2,1), 0, 0, 0; backward U(0,1) U(0,2) U(1,2),
// reciprocal pivots.  a[9k + 3p + q]: block row p, column q of neighbour k.
template <typename T>
struct GCard {
    static __host__ __device__ uint32_t slot_off() { return 3 * 128; }
    static __host__ __device__ uint32_t h_off(uint32_t maxc) { return slot_off() + 128 * maxc; }
    static __host__ __device__ uint32_t a_off(uint32_t maxc) {
        return h_off(maxc) + 6 * 32 * (uint32_t)sizeof(T);
    }
    static __host__ __device__ uint32_t bytes(uint32_t maxc) {
        return a_off(maxc) + 9 * maxc * 32 * (uint32_t)sizeof(T);
    }
};

// One warp per card lane (group g, lane l): empty lanes get node 0xffffffff.
template <typename T, bool Lower>
__global__ void k_pack_groups(ClusterSolve P, const uint32_t* __restrict__ grp_first,
                              const T* __restrict__ lu, const T* __restrict__ dinv,
                              unsigned char* __restrict__ cards) {
    const int lane = threadIdx.x & 31;
    const uint32_t card = GCard<T>::bytes(P.maxc);
    const uint32_t n_lanes = 32 * P.n_groups;
    for (uint32_t cl = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; cl < n_lanes;
         cl += (gridDim.x * blockDim.x) >> 5) {
        const uint32_t g = cl >> 5, l = cl & 31;
        const uint32_t first = __ldg(grp_first + g), last = __ldg(grp_first + g + 1);
        unsigned char* cd = cards + (size_t)g * card;
        uint32_t* ci = reinterpret_cast<uint32_t*>(cd);
        T* h = reinterpret_cast<T*>(cd + GCard<T>::h_off(P.maxc));
        T* a = reinterpret_cast<T*>(cd + GCard<T>::a_off(P.maxc));
        uint32_t* sl = reinterpret_cast<uint32_t*>(cd + GCard<T>::slot_off());
        if (first + l >= last) {
            if (lane == 0) {
                ci[l] = 0xffffffffu;
                ci[32 + l] = 0;
                ci[64 + l] = 0;
            }
            if ((uint32_t)lane < 6) h[32 * lane + l] = T(0);
            for (uint32_t v = lane; v < 9 * P.maxc; v += 32) a[32 * v + l] = T(0);
            if ((uint32_t)lane < P.maxc) sl[32 * lane + l] = 0;
            continue;
        }
        const uint4 rec = __ldg(P.rec + first + l);
        const uint32_t n = rec.x, nb0 = rec.y;
        const uint32_t deg = rec.z & 0xff, sk = (rec.z >> 8) & 0xff, cnt = rec.z >> 16;
        const uint32_t rl = 3 * deg, ds = 3 * sk;
        const T* row = lu + 9 * (size_t)nb0;
        if (lane == 0) {
            ci[l] = n;
            ci[32 + l] = rec.w;
            ci[64 + l] = cnt;
        }
        if (lane < 3) {
            const uint32_t off = Lower ? (lane == 0 ? rl + ds : lane == 1 ? 2 * rl + ds : 2 * rl + ds + 1)
                                       : (lane == 0 ? ds + 1 : lane == 1 ? ds + 2 : rl + ds + 2);
            h[32 * lane + l] = row[off];
        } else if (lane < 6) {
            h[32 * lane + l] = Lower ? T(0) : dinv[3 * (size_t)n + lane - 3];
        }
        const uint32_t kb = Lower ? 0 : sk + 1;
        for (uint32_t v = lane; v < 9 * P.maxc; v += 32) {
            const uint32_t k = v / 9, pq = v - 9 * k, pr = pq / 3, q = pq - 3 * pr;
            a[32 * v + l] = k < cnt ? row[pr * rl + 3 * (kb + k) + q] : T(0);
        }
        if ((uint32_t)lane < P.maxc)
            sl[32 * lane + l] = (uint32_t)lane < cnt ? __ldg(P.nslot + nb0 + kb + lane) : 0u;
    }
}

template <typename T, bool Lower, int NB>
__global__ void __launch_bounds__(256, 1)
    k_trsv_lanes(ClusterSolve P, const uint32_t* __restrict__ grp_first,
                 const unsigned char* __restrict__ cards, const T* __restrict__ rhs,
                 T* __restrict__ out, unsigned* __restrict__ status) {
    extern __shared__ __align__(128) unsigned char smem[];
    namespace cg = cooperative_groups;
    cg::cluster_group cluster = cg::this_cluster();
    const uint32_t cta = cluster.block_rank();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const uint32_t W = P.n_ctas * P.warps_per_cta;
    const uint32_t gw = cta * P.warps_per_cta + w;
    constexpr uint32_t VS = sizeof(T) == 4 ? 16 : 32;
    constexpr uint32_t VT = VS / sizeof(T);
    const uint32_t maxc = P.maxc;
    const uint32_t card = GCard<T>::bytes(maxc);
    const uint32_t rhs_b = 3 * 32 * sizeof(T);
    const uint32_t buf_b = card + rhs_b;
    T* pool = reinterpret_cast<T*>(smem);
    const uint32_t pool_sa = smem_u32(smem);
    const uint32_t pool_bytes = (P.pool_slots * VS + 127) & ~127u;
    unsigned char* bufs = smem + pool_bytes + (size_t)w * NB * buf_b;
    const uint32_t bufs_sa = smem_u32(bufs);
    const uint32_t bar_sa =
        smem_u32(smem + pool_bytes + (size_t)P.warps_per_cta * NB * buf_b) + 8 * NB * w;

    for (uint32_t i = threadIdx.x; i < P.pool_slots * VT; i += blockDim.x)
        pool[i] = Sentinel<T>::value();
    if (lane == 0)
        for (int b = 0; b < NB; ++b) mbar_init(bar_sa + 8 * b, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    cluster.sync();

    // the warp's groups are gw, gw + W, ...; group ordinal j lives in buffer j % NB
    const uint32_t n_mine = P.n_groups > gw ? (P.n_groups - gw + W - 1) / W : 0;
    auto issue = [&](uint32_t j) {
        if (j < n_mine) {
            const uint32_t g = gw + j * W, b = j % NB;
            const uint32_t st = bufs_sa + b * buf_b;
            if (lane == 0) {
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                mbar_expect_tx(bar_sa + 8 * b, card);
                bulk_g2s(st, cards + (size_t)g * card, card, bar_sa + 8 * b);
            }
            const uint32_t first = __ldg(grp_first + g), last = __ldg(grp_first + g + 1);
            if (first + lane < last) {
                const uint32_t n = __ldg(&P.rec[first + lane].x);
#pragma unroll
                for (int i = 0; i < 3; ++i)
                    cp_async_val(st + card + (3 * lane + i) * sizeof(T), rhs + 3 * (size_t)n + i);
            }
        }
        cp_async_commit();
    };
    for (uint32_t j = 0; j < (uint32_t)NB; ++j) issue(j);
    uint32_t done_j = 0;  // groups of this warp resolved so far

    for (uint32_t l = 0; l < P.n_levels; ++l) {
        // lvl_ptr holds each level's group range in lane-group plans
        const uint32_t g0 = __ldg(P.lvl_ptr + l), g1 = __ldg(P.lvl_ptr + l + 1);
        // this warp's group of the level, if any (groups per level <= W)
        const uint32_t off = (gw + W - g0 % W) % W;
        if (g0 + off < g1) {
            const uint32_t j = done_j, b = j % NB;
            mbar_wait(bar_sa + 8 * b, (j / NB) & 1u, status);
            cp_async_wait<NB - 1>();
            __syncwarp();
            const unsigned char* cd = bufs + b * buf_b;
            const uint32_t* ci = reinterpret_cast<const uint32_t*>(cd);
            const uint32_t node = ci[lane];
            const uint32_t cnt = node != 0xffffffffu ? ci[64 + lane] : 0u;
            const uint32_t* csl = reinterpret_cast<const uint32_t*>(cd + GCard<T>::slot_off());
            const T* h = reinterpret_cast<const T*>(cd + GCard<T>::h_off(maxc));
            const T* a = reinterpret_cast<const T*>(cd + GCard<T>::a_off(maxc));
            const T* r = reinterpret_cast<const T*>(cd + card);
            // poll the lane's dependency slots in lock step
            T v[kLaneMaxC][3];
            uint32_t need = 0;
#pragma unroll
            for (int k = 0; k < kLaneMaxC; ++k) {
                v[k][0] = v[k][1] = v[k][2] = T(0);
                if ((uint32_t)k < cnt) need |= 1u << k;
            }
            const long long t0 = clock64();
            unsigned ns = 32;
            for (unsigned it = 0;; ++it) {
                if (P.sleep_ns && it > 2) {
                    __nanosleep(ns);
                    if (ns < P.sleep_ns) ns <<= 1;
                }
#pragma unroll
                for (int k = 0; k < kLaneMaxC; ++k)
                    if (need & (1u << k)) {
                        const uint32_t s = csl[32 * k + lane];
                        ld_slot<T>(mapa(pool_sa + (s & 0xffffu) * VS, s >> 16), v[k][0], v[k][1],
                                   v[k][2]);
                        if (!(Sentinel<T>::is(v[k][0]) | Sentinel<T>::is(v[k][1]) |
                              Sentinel<T>::is(v[k][2])))
                            need &= ~(1u << k);
                    }
                if (__all_sync(0xffffffffu, need == 0)) break;
                if ((it & 63u) == 63u &&
                    __any_sync(0xffffffffu, (ld_volatile_u32(status) & FM_FLAG_TIMEOUT) ||
                                                clock64() - t0 > kWaitCycles)) {
                    if (lane == 0) raise_flag(status, FM_FLAG_TIMEOUT);
                    break;
                }
            }
            T s0 = T(0), s1 = T(0), s2 = T(0);
#pragma unroll
            for (int k = 0; k < kLaneMaxC; ++k) {
                if ((uint32_t)k < cnt) {
                    const T* ak = a + 32 * 9 * k + lane;
                    s0 += ak[0] * v[k][0] + ak[32] * v[k][1] + ak[64] * v[k][2];
                    s1 += ak[96] * v[k][0] + ak[128] * v[k][1] + ak[160] * v[k][2];
                    s2 += ak[192] * v[k][0] + ak[224] * v[k][1] + ak[256] * v[k][2];
                }
            }
            if (node != 0xffffffffu) {
                const T h0 = h[lane], h1 = h[32 + lane], h2 = h[64 + lane];
                T x0, x1, x2;
                if constexpr (Lower) {
                    x0 = r[3 * lane] - s0;
                    x1 = r[3 * lane + 1] - s1 - h0 * x0;
                    x2 = r[3 * lane + 2] - s2 - h1 * x0 - h2 * x1;
                } else {
                    x2 = (r[3 * lane + 2] - s2) * h[160 + lane];
                    x1 = (r[3 * lane + 1] - s1 - h2 * x2) * h[128 + lane];
                    x0 = (r[3 * lane] - s0 - h0 * x1 - h1 * x2) * h[96 + lane];
                }
                st_slot<T>(pool_sa + ci[32 + lane] * VS, x0, x1, x2);
                T* o = out + 3 * (size_t)node;
                o[0] = x0;
                o[1] = x1;
                o[2] = x2;
            }
            __syncwarp();
            ++done_j;
            issue(done_j + NB - 1);
        }
        if ((l + 1) % P.window == 0 || l + 1 == P.n_levels) {
            cluster_barrier();
            const uint32_t t = l / P.window;
            const uint32_t r0 = __ldg(P.reset_ptr + t * P.n_ctas + cta);
            const uint32_t r1 = __ldg(P.reset_ptr + t * P.n_ctas + cta + 1);
            for (uint32_t i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
                const uint32_t sa = pool_sa + __ldg(P.reset + i) * VS;
                st_slot<T>(sa, Sentinel<T>::value(), Sentinel<T>::value(), Sentinel<T>::value());
            }
        }
    }
    cp_async_wait<0>();
}

template <typename K>
static int max_clusters_lanes(K kernel, int cs, int threads, size_t smem) {
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
    cfg.blockDim = dim3(threads);
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

template <typename T, bool Lower, int NB>
static cudaError_t launch_lanes_one(const ClusterSolve& P, const uint32_t* grp_first,
                                    const unsigned char* cards, const T* rhs, T* out,
                                    unsigned* status, cudaStream_t s) {
    auto kern = k_trsv_lanes<T, Lower, NB>;
    const size_t smem = lanes_smem_bytes(P, sizeof(T));
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
    return cudaLaunchKernelEx(&cfg, kern, P, grp_first, cards, rhs, out, status);
}

}  // namespace

int lanes_buffers(size_t value_bytes) { return value_bytes == 4 ? 2 : 1; }

size_t lanes_card_bytes(const ClusterSolve& P, size_t value_bytes) {
    return value_bytes == 4 ? GCard<float>::bytes(P.maxc) : GCard<double>::bytes(P.maxc);
}

size_t lanes_smem_bytes(const ClusterSolve& P, size_t value_bytes) {
    const size_t slot = value_bytes == 4 ? 16 : 32;
    const size_t pool = (P.pool_slots * slot + 127) & ~(size_t)127;
    const size_t nb = lanes_buffers(value_bytes);
    const size_t buf = lanes_card_bytes(P, value_bytes) + 3 * 32 * value_bytes;
    return pool + P.warps_per_cta * nb * (buf + 8);
}

int lanes_max_active(size_t value_bytes, const ClusterSolve& P) {
    const size_t smem = lanes_smem_bytes(P, value_bytes);
    const int threads = 32 * (int)P.warps_per_cta;
    if (value_bytes == 4) return max_clusters_lanes(k_trsv_lanes<float, true, 2>, (int)P.n_ctas, threads, smem);
    return max_clusters_lanes(k_trsv_lanes<double, true, 1>, (int)P.n_ctas, threads, smem);
}

int lanes_max_neighbours() { return kLaneMaxC; }

template <typename T>
void launch_pack_groups(const ClusterSolve& F, const ClusterSolve& B, const uint32_t* grp_f,
                        const uint32_t* grp_b, const T* lu, const T* dinv, unsigned char* cards_f,
                        unsigned char* cards_b, cudaStream_t s) {
    auto grid = [](uint32_t n_groups) {
        unsigned g = (32 * n_groups + 7) / 8;
        return g > 4736 ? 4736u : (g ? g : 1u);
    };
    if (F.n_groups) k_pack_groups<T, true><<<grid(F.n_groups), 256, 0, s>>>(F, grp_f, lu, dinv, cards_f);
    if (B.n_groups) k_pack_groups<T, false><<<grid(B.n_groups), 256, 0, s>>>(B, grp_b, lu, dinv, cards_b);
}

template <typename T>
cudaError_t launch_trsv_lanes(const ClusterSolve& F, const ClusterSolve& B, const uint32_t* grp_f,
                              const uint32_t* grp_b, const unsigned char* cards_f,
                              const unsigned char* cards_b, const T* r, T* tmp, T* y,
                              unsigned* status, cudaStream_t s) {
    constexpr int NB = sizeof(T) == 4 ? 2 : 1;
    cudaError_t e = launch_lanes_one<T, true, NB>(F, grp_f, cards_f, r, tmp, status, s);
    if (e != cudaSuccess) return e;
    return launch_lanes_one<T, false, NB>(B, grp_b, cards_b, tmp, y, status, s);
}

template void launch_pack_groups<float>(const ClusterSolve&, const ClusterSolve&, const uint32_t*,
                                        const uint32_t*, const float*, const float*,
                                        unsigned char*, unsigned char*, cudaStream_t);
template void launch_pack_groups<double>(const ClusterSolve&, const ClusterSolve&,
                                         const uint32_t*, const uint32_t*, const double*,
                                         const double*, unsigned char*, unsigned char*,
                                         cudaStream_t);
template cudaError_t launch_trsv_lanes<float>(const ClusterSolve&, const ClusterSolve&,
                                              const uint32_t*, const uint32_t*,
                                              const unsigned char*, const unsigned char*,
                                              const float*, float*, float*, unsigned*,
                                              cudaStream_t);
template cudaError_t launch_trsv_lanes<double>(const ClusterSolve&, const ClusterSolve&,
                                               const uint32_t*, const uint32_t*,
                                               const unsigned char*, const unsigned char*,
                                               const double*, double*, double*, unsigned*,
                                               cudaStream_t);

}  // namespace fm
