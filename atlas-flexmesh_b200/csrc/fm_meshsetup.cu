// fm_meshsetup.cu — the per-mesh structures built on the device (see
// fm_meshsetup.hpp), and the linear-time form of the reference's element
// colouring.
#include <algorithm>
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>
#include <vector>

#include "fm_device.cuh"
#include "fm_meshsetup.hpp"

namespace fm {

namespace {

constexpr int kSetupWarps = 8;  // warps per block of the per-node kernels
constexpr uint32_t kNone = 0xffffffffu;

__device__ __forceinline__ uint32_t vtx(const uint4& c, int q) {
    return q == 0 ? (c.x & 0x7fffffffu) : q == 1 ? c.y : q == 2 ? c.z : c.w;
}

__global__ void k_inc_count(uint32_t ne, const uint4* __restrict__ conn, uint32_t* cnt) {
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < ne; e += gridDim.x * blockDim.x) {
        const uint4 c = conn[e];
#pragma unroll
        for (int q = 0; q < 4; ++q) atomicAdd(cnt + vtx(c, q), 1u);
    }
}

__global__ void k_inc_fill(uint32_t ne, const uint4* __restrict__ conn,
                           const uint32_t* __restrict__ ptr, uint32_t* fill, uint32_t* inc_e) {
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < ne; e += gridDim.x * blockDim.x) {
        const uint4 c = conn[e];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const uint32_t n = vtx(c, q);
            inc_e[ptr[n] + atomicAdd(fill + n, 1u)] = e;
        }
    }
}

// ascending sort of the 32 lanes' values (bitonic network over shuffles)
__device__ __forceinline__ uint32_t warp_sort_asc(uint32_t v, int lane) {
#pragma unroll
    for (int k = 2; k <= 32; k <<= 1)
#pragma unroll
        for (int j = k >> 1; j > 0; j >>= 1) {
            const uint32_t o = __shfl_xor_sync(kFull, v, j);
            const bool asc = (lane & k) == 0, low = (lane & j) == 0;
            v = (low == asc) ? min(v, o) : max(v, o);
        }
    return v;
}

// each node's incident tets ascending (the fill order above is arbitrary)
__global__ void k_inc_sort(uint32_t nn, const uint32_t* __restrict__ ptr, uint32_t* inc_e,
                           unsigned* max_inc) {
    const int lane = threadIdx.x & 31;
    for (uint32_t n = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; n < nn;
         n += (gridDim.x * blockDim.x) >> 5) {
        const uint32_t b = ptr[n], m = ptr[n + 1] - b;
        if (lane == 0) atomicMax(max_inc, m);
        if (m > 32) continue;  // beyond the kernels' limit: reported, not sorted
        uint32_t v = lane < (int)m ? inc_e[b + lane] : kNone;
        v = warp_sort_asc(v, lane);
        if (lane < (int)m) inc_e[b + lane] = v;
    }
}

// The union of the incident tets' vertices of node n (at most 32 tets, 128
// candidates) in shared memory; first[i]: candidate i is the first copy of
// its value.  Returns the number of distinct values.
__device__ __forceinline__ int node_candidates(uint32_t n, const uint4* __restrict__ conn,
                                               const uint32_t* __restrict__ inc_ptr,
                                               const uint32_t* __restrict__ inc_e, uint32_t* cand,
                                               uint8_t* first, int lane) {
    const uint32_t b = inc_ptr[n], m = inc_ptr[n + 1] - b;
    uint4 c = make_uint4(kNone, kNone, kNone, kNone);
    if (lane < (int)m) {
        c = conn[inc_e[b + lane]];
        c.x &= 0x7fffffffu;
    }
    cand[4 * lane + 0] = c.x;
    cand[4 * lane + 1] = c.y;
    cand[4 * lane + 2] = c.z;
    cand[4 * lane + 3] = c.w;
    __syncwarp();
    int mine = 0;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int i = 4 * lane + q;
        const uint32_t v = cand[i];
        bool f = v != kNone;
        for (int j = 0; j < i && f; ++j) f = cand[j] != v;
        first[i] = f;
        mine += f;
    }
    __syncwarp();
    return (int)warp_sum((unsigned)mine);
}

__global__ void __launch_bounds__(kSetupWarps * 32)
    k_graph_degree(uint32_t nn, const uint4* __restrict__ conn, const uint32_t* __restrict__ inc_ptr,
                   const uint32_t* __restrict__ inc_e, uint32_t* deg, unsigned* max_deg) {
    __shared__ uint32_t cand_s[kSetupWarps][128];
    __shared__ uint8_t first_s[kSetupWarps][128];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (uint32_t n = blockIdx.x * kSetupWarps + w; n < nn; n += gridDim.x * kSetupWarps) {
        const int d = node_candidates(n, conn, inc_ptr, inc_e, cand_s[w], first_s[w], lane);
        if (lane == 0) {
            deg[n] = (uint32_t)d;
            atomicMax(max_deg, (unsigned)d);
        }
        __syncwarp();
    }
}

__global__ void __launch_bounds__(kSetupWarps * 32)
    k_graph_fill(uint32_t nn, const uint4* __restrict__ conn, const uint32_t* __restrict__ inc_ptr,
                 const uint32_t* __restrict__ inc_e, const uint32_t* __restrict__ nbr_ptr,
                 uint32_t* nbr, uint32_t* self_pos) {
    __shared__ uint32_t cand_s[kSetupWarps][128];
    __shared__ uint8_t first_s[kSetupWarps][128];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (uint32_t n = blockIdx.x * kSetupWarps + w; n < nn; n += gridDim.x * kSetupWarps) {
        node_candidates(n, conn, inc_ptr, inc_e, cand_s[w], first_s[w], lane);
        const uint32_t b = nbr_ptr[n];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int i = 4 * lane + q;
            if (!first_s[w][i]) continue;
            const uint32_t v = cand_s[w][i];
            uint32_t r = 0;
            for (int j = 0; j < 128; ++j) r += first_s[w][j] && cand_s[w][j] < v;
            nbr[b + r] = v;
            if (v == n) self_pos[n] = r;
        }
        __syncwarp();
    }
}

// Node dependency depth: depth(n) = 1 + max depth(m) over the neighbours m
// before n (lower) / after n (upper), 0 when there are none.  Warps take
// nodes by ticket in dependency order, so every node a warp waits on holds
// an earlier ticket of a warp that is running; waits are bounded.
__global__ void __launch_bounds__(256)
    k_node_depth(uint32_t nn, int lower, const uint32_t* __restrict__ nbr_ptr,
                 const uint32_t* __restrict__ nbr, uint32_t* depth, unsigned* flag,
                 unsigned* ticket, unsigned* status) {
    const int lane = threadIdx.x & 31;
    for (;;) {
        uint32_t t = 0;
        if (lane == 0) t = atomicAdd(ticket, 1u);
        t = __shfl_sync(kFull, t, 0);
        if (t >= nn) break;
        const uint32_t n = lower ? t : nn - 1 - t;
        const uint32_t b = nbr_ptr[n], deg = nbr_ptr[n + 1] - b;
        const uint32_t m = lane < (int)deg ? nbr[b + lane] : n;
        const bool need = lower ? m < n : m > n;
        wait_flags_warp(flag + m, need, 1u, status, 0u);
        __syncwarp();
        uint32_t d = need ? ld_volatile_u32(depth + m) + 1u : 0u;
        d = __reduce_max_sync(kFull, d);
        if (lane == 0) {
            depth[n] = d;
            st_release(flag + n, 1u);
        }
    }
}

__global__ void k_depth_keys(uint32_t nn, const uint32_t* __restrict__ depth,
                             unsigned long long* keys, uint32_t* hist) {
    for (uint32_t n = blockIdx.x * blockDim.x + threadIdx.x; n < nn; n += gridDim.x * blockDim.x) {
        const uint32_t d = depth[n];
        keys[n] = ((unsigned long long)d << 32) | n;
        atomicAdd(hist + d, 1u);
    }
}

__global__ void k_node_records(uint32_t nn, const unsigned long long* __restrict__ keys,
                               const uint32_t* __restrict__ nbr_ptr,
                               const uint32_t* __restrict__ self_pos, uint32_t* order,
                               uint4* rec) {
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < nn; t += gridDim.x * blockDim.x) {
        const uint32_t nd = (uint32_t)(keys[t] & 0xffffffffull);
        order[t] = nd;
        rec[t] = make_uint4(nd, nbr_ptr[nd], nbr_ptr[nd + 1] - nbr_ptr[nd], self_pos[nd]);
    }
}

// entries of node n's ILU update map: sum over its lower neighbours m of
// deg(m) - self(m)
__global__ void k_emap_count(uint32_t nn, const uint32_t* __restrict__ nbr_ptr,
                             const uint32_t* __restrict__ nbr, const uint32_t* __restrict__ self_pos,
                             uint32_t* cnt) {
    for (uint32_t n = blockIdx.x * blockDim.x + threadIdx.x; n < nn; n += gridDim.x * blockDim.x) {
        uint32_t c = 0;
        for (uint32_t k = nbr_ptr[n]; k < nbr_ptr[n] + self_pos[n]; ++k) {
            const uint32_t m = nbr[k];
            c += (nbr_ptr[m + 1] - nbr_ptr[m]) - self_pos[m];
        }
        cnt[n] = c;
    }
}

// position of v in the sorted list s[0..len) or 0xff
__device__ __forceinline__ uint32_t pos_in(const uint32_t* s, uint32_t len, uint32_t v) {
    uint32_t lo = 0, hi = len;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (s[mid] < v) lo = mid + 1;
        else hi = mid;
    }
    return (lo < len && s[lo] == v) ? lo : 0xffu;
}

__global__ void __launch_bounds__(kSetupWarps * 32)
    k_emap_fill(uint32_t nn, const uint32_t* __restrict__ nbr_ptr, const uint32_t* __restrict__ nbr,
                const uint32_t* __restrict__ self_pos, const uint32_t* __restrict__ emap_ptr,
                uint8_t* emap) {
    __shared__ uint32_t list_s[kSetupWarps][32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (uint32_t n = blockIdx.x * kSetupWarps + w; n < nn; n += gridDim.x * kSetupWarps) {
        const uint32_t b = nbr_ptr[n], deg = nbr_ptr[n + 1] - b, sk = self_pos[n];
        if (lane < (int)deg) list_s[w][lane] = nbr[b + lane];
        __syncwarp();
        uint32_t o = emap_ptr[n];
        for (uint32_t k = 0; k < sk; ++k) {
            const uint32_t m = list_s[w][k];
            const uint32_t mb = nbr_ptr[m] + self_pos[m], mu = nbr_ptr[m + 1] - mb;
            if (lane < (int)mu) emap[o + lane] = (uint8_t)pos_in(list_s[w], deg, nbr[mb + lane]);
            o += mu;
        }
        __syncwarp();
    }
}

// node-pass scatter structure of the assembly: per incidence the 4 vertex
// positions in the owner's list, per neighbour entry the owner's incident
// (not skipped) tets holding that edge
__global__ void __launch_bounds__(kSetupWarps * 32)
    k_scatter_struct(uint32_t nn, const uint4* __restrict__ conn,
                     const uint32_t* __restrict__ inc_ptr, const uint32_t* __restrict__ inc_e,
                     const uint32_t* __restrict__ nbr_ptr, const uint32_t* __restrict__ nbr,
                     uint32_t* inc_pos, uint32_t* members) {
    __shared__ uint32_t list_s[kSetupWarps][32];
    __shared__ unsigned memb_s[kSetupWarps][32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (uint32_t n = blockIdx.x * kSetupWarps + w; n < nn; n += gridDim.x * kSetupWarps) {
        const uint32_t b = nbr_ptr[n], deg = nbr_ptr[n + 1] - b;
        const uint32_t ib = inc_ptr[n], mi = inc_ptr[n + 1] - ib;
        if (lane < (int)deg) list_s[w][lane] = nbr[b + lane];
        memb_s[w][lane] = 0u;
        __syncwarp();
        if (lane < (int)mi) {
            const uint32_t e = inc_e[ib + lane];
            const uint4 c = conn[e];
            const bool skip = (c.x & 0x80000000u) != 0;
            uint32_t pk = 0;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const uint32_t v = vtx(c, q);
                const uint32_t p = pos_in(list_s[w], deg, v);
                pk |= p << (8 * q);
                if (p != 0xffu && v != n && !skip) atomicOr(&memb_s[w][p], 1u << lane);
            }
            inc_pos[ib + lane] = pk;
        }
        __syncwarp();
        if (lane < (int)deg) members[b + lane] = memb_s[w][lane];
        __syncwarp();
    }
}

unsigned blocks_for(size_t items, unsigned per_block) {
    const size_t b = (items + per_block - 1) / per_block;
    return (unsigned)std::max<size_t>(1, std::min<size_t>(b, 148u * 32u));
}

template <typename T>
cudaError_t down(std::vector<T>& h, const T* d, size_t n, cudaStream_t s) {
    h.resize(n);
    return n ? cudaMemcpyAsync(h.data(), d, n * sizeof(T), cudaMemcpyDeviceToHost, s)
             : cudaSuccess;
}

#define SCK(call)                            \
    do {                                     \
        const cudaError_t e_ = (call);       \
        if (e_ != cudaSuccess) return e_;    \
    } while (0)

// exclusive prefix sum of in[0..n) into out[0..n] (out[n] = total)
cudaError_t exclusive_scan(const uint32_t* in, uint32_t* out, uint32_t n, DevBuf<unsigned char>& tmp,
                           cudaStream_t s) {
    size_t bytes = 0;
    SCK(cub::DeviceScan::ExclusiveSum(nullptr, bytes, in, out, n + 1, s));
    SCK(tmp.reserve(bytes));
    return cub::DeviceScan::ExclusiveSum(tmp.p, bytes, in, out, n + 1, s);
}

}  // namespace

cudaError_t build_mesh_device(uint32_t nn, uint32_t ne, const uint4* conn, MeshSetupDev& d,
                              MeshSetupHost& h, unsigned* status, int* result, cudaStream_t s) {
    *result = kSetupOk;
    DevBuf<uint32_t> cnt, depth;
    DevBuf<unsigned> scal;  // max_inc, max_deg, ticket
    DevBuf<unsigned char> tmp;
    DevBuf<unsigned long long> keys, keys_sorted;
    SCK(cnt.reserve((size_t)nn + 1));
    SCK(scal.reserve(4));
    SCK(cudaMemsetAsync(scal.p, 0, 4 * sizeof(unsigned), s));

    // incidence: counts, offsets, fill, per-node sort
    SCK(cudaMemsetAsync(cnt.p, 0, ((size_t)nn + 1) * sizeof(uint32_t), s));
    k_inc_count<<<blocks_for(ne, 256), 256, 0, s>>>(ne, conn, cnt.p);
    SCK(d.inc_ptr->reserve((size_t)nn + 1));
    SCK(exclusive_scan(cnt.p, d.inc_ptr->p, nn, tmp, s));
    SCK(d.inc_e->reserve(std::max<size_t>(1, 4 * (size_t)ne)));
    SCK(cudaMemsetAsync(cnt.p, 0, ((size_t)nn + 1) * sizeof(uint32_t), s));
    k_inc_fill<<<blocks_for(ne, 256), 256, 0, s>>>(ne, conn, d.inc_ptr->p, cnt.p, d.inc_e->p);
    k_inc_sort<<<blocks_for((size_t)nn * 32, 256), 256, 0, s>>>(nn, d.inc_ptr->p, d.inc_e->p,
                                                              scal.p);
    unsigned hs[4];
    SCK(cudaMemcpyAsync(hs, scal.p, sizeof hs, cudaMemcpyDeviceToHost, s));
    SCK(cudaStreamSynchronize(s));
    h.max_inc = hs[0];
    if (h.max_inc > 32) {
        *result = kSetupLimits;
        return cudaSuccess;
    }

    // node graph: degrees, offsets, sorted unique neighbour sets
    k_graph_degree<<<blocks_for(nn, kSetupWarps), kSetupWarps * 32, 0, s>>>(
        nn, conn, d.inc_ptr->p, d.inc_e->p, cnt.p, scal.p + 1);
    SCK(d.nbr_ptr->reserve((size_t)nn + 1));
    SCK(exclusive_scan(cnt.p, d.nbr_ptr->p, nn, tmp, s));
    uint32_t total = 0;
    SCK(cudaMemcpyAsync(&total, d.nbr_ptr->p + nn, sizeof total, cudaMemcpyDeviceToHost, s));
    SCK(cudaMemcpyAsync(hs, scal.p, sizeof hs, cudaMemcpyDeviceToHost, s));
    SCK(cudaStreamSynchronize(s));
    h.graph.max_deg = hs[1];
    if (h.graph.max_deg > 32) {
        *result = kSetupLimits;
        return cudaSuccess;
    }
    SCK(d.nbr->reserve(std::max<uint32_t>(total, 1)));
    SCK(d.self_pos->reserve(std::max<uint32_t>(nn, 1)));
    SCK(cudaMemsetAsync(d.self_pos->p, 0, (size_t)nn * sizeof(uint32_t), s));
    k_graph_fill<<<blocks_for(nn, kSetupWarps), kSetupWarps * 32, 0, s>>>(
        nn, conn, d.inc_ptr->p, d.inc_e->p, d.nbr_ptr->p, d.nbr->p, d.self_pos->p);

    // dependency depth both ways and the level lists (stable by node id)
    SCK(depth.reserve(std::max<uint32_t>(nn, 1)));
    SCK(keys.reserve(std::max<uint32_t>(nn, 1)));
    SCK(keys_sorted.reserve(std::max<uint32_t>(nn, 1)));
    SCK(d.node_fwd->reserve(std::max<uint32_t>(nn, 1)));
    SCK(d.node_bwd->reserve(std::max<uint32_t>(nn, 1)));
    SCK(d.node_fwd_rec->reserve(std::max<uint32_t>(nn, 1)));
    SCK(d.node_bwd_rec->reserve(std::max<uint32_t>(nn, 1)));
    int dev = 0, sms = 148;
    SCK(cudaGetDevice(&dev));
    SCK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    for (int lower = 1; lower >= 0; --lower) {
        SCK(cudaMemsetAsync(cnt.p, 0, ((size_t)nn + 1) * sizeof(uint32_t), s));  // flags
        SCK(cudaMemsetAsync(scal.p + 2, 0, sizeof(unsigned), s));               // ticket
        k_node_depth<<<sms * 4, 256, 0, s>>>(nn, lower, d.nbr_ptr->p, d.nbr->p, depth.p, cnt.p,
                                             scal.p + 2, status);
        unsigned flags = 0;
        SCK(cudaMemcpyAsync(&flags, status, sizeof flags, cudaMemcpyDeviceToHost, s));
        SCK(cudaStreamSynchronize(s));
        if (flags & FM_FLAG_TIMEOUT) {
            *result = kSetupTimeout;
            return cudaSuccess;
        }
        // depth histogram (at most nn levels) and the (depth, node) keys
        SCK(cudaMemsetAsync(cnt.p, 0, ((size_t)nn + 1) * sizeof(uint32_t), s));
        k_depth_keys<<<blocks_for(nn, 256), 256, 0, s>>>(nn, depth.p, keys.p, cnt.p);
        size_t bytes = 0;
        SCK(cub::DeviceRadixSort::SortKeys(nullptr, bytes, keys.p, keys_sorted.p, (int)nn, 0, 64,
                                           s));
        SCK(tmp.reserve(bytes));
        SCK(cub::DeviceRadixSort::SortKeys(tmp.p, bytes, keys.p, keys_sorted.p, (int)nn, 0, 64,
                                           s));
        DevBuf<uint32_t>& ord = lower ? *d.node_fwd : *d.node_bwd;
        DevBuf<uint4>& rec = lower ? *d.node_fwd_rec : *d.node_bwd_rec;
        k_node_records<<<blocks_for(nn, 256), 256, 0, s>>>(nn, keys_sorted.p, d.nbr_ptr->p,
                                                           d.self_pos->p, ord.p, rec.p);
        unsigned long long last = 0;
        if (nn)
            SCK(cudaMemcpyAsync(&last, keys_sorted.p + nn - 1, sizeof last,
                                cudaMemcpyDeviceToHost, s));
        SCK(cudaStreamSynchronize(s));
        const uint32_t nl = nn ? (uint32_t)(last >> 32) + 1 : 0;
        std::vector<uint32_t>& lp = lower ? h.lp : h.up;
        std::vector<uint32_t>& lo = lower ? h.lo : h.uo;
        std::vector<uint32_t> hist;
        SCK(down(hist, cnt.p, nl, s));
        SCK(down(lo, ord.p, nn, s));
        SCK(cudaStreamSynchronize(s));
        lp.assign(nl + 1, 0);
        for (uint32_t l = 0; l < nl; ++l) lp[l + 1] = lp[l] + hist[l];
    }

    // ILU(0) update maps and the assembly's scatter structure
    k_emap_count<<<blocks_for(nn, 256), 256, 0, s>>>(nn, d.nbr_ptr->p, d.nbr->p, d.self_pos->p,
                                                     cnt.p);
    SCK(d.emap_ptr->reserve((size_t)nn + 1));
    SCK(exclusive_scan(cnt.p, d.emap_ptr->p, nn, tmp, s));
    uint32_t n_emap = 0;
    SCK(cudaMemcpyAsync(&n_emap, d.emap_ptr->p + nn, sizeof n_emap, cudaMemcpyDeviceToHost, s));
    SCK(cudaStreamSynchronize(s));
    SCK(d.emap->reserve(std::max<uint32_t>(n_emap, 1)));
    k_emap_fill<<<blocks_for(nn, kSetupWarps), kSetupWarps * 32, 0, s>>>(
        nn, d.nbr_ptr->p, d.nbr->p, d.self_pos->p, d.emap_ptr->p, d.emap->p);
    SCK(d.inc_pos->reserve(std::max<size_t>(1, 4 * (size_t)ne)));
    SCK(d.nbr_members->reserve(std::max<uint32_t>(total, 1)));
    k_scatter_struct<<<blocks_for(nn, kSetupWarps), kSetupWarps * 32, 0, s>>>(
        nn, conn, d.inc_ptr->p, d.inc_e->p, d.nbr_ptr->p, d.nbr->p, d.inc_pos->p,
        d.nbr_members->p);
    SCK(cudaGetLastError());

    // host copies of the graph
    h.graph.n_nodes = nn;
    SCK(down(h.graph.ptr, d.nbr_ptr->p, (size_t)nn + 1, s));
    SCK(down(h.graph.nbr, d.nbr->p, total, s));
    SCK(down(h.graph.self, d.self_pos->p, nn, s));
    SCK(cudaStreamSynchronize(s));
    return cudaSuccess;
}

namespace {

// slot[e][(i*3+di)*12 + j*3+dj] of tets e0 .. e0+count-1: the CSR index of
// (3 n_i + di, 3 n_j + dj).  Solve pattern: node n's rows hold every
// neighbour's three columns, row 3n+p at 9 ptr[n] + 3 p deg, neighbour k at
// + 3k.  Reference pattern (its neighbour-major fill, :1109-1119): node n's
// 9 deg entries form one run, entry w = 9k + 3s + q (neighbour k, s = 0..2)
// sits in row 3n + w / (3 deg) with column 3 nbr[k] + q; of the entries that
// land on (row, column) the last wins (:1146-1149), none gives -1.
__global__ void k_slot_map(uint32_t e0, uint32_t count, const uint4* __restrict__ conn,
                           const uint32_t* __restrict__ nbr_ptr, const uint32_t* __restrict__ nbr,
                           int reference, int32_t* __restrict__ slot) {
    const uint64_t total = 144ull * count;
    for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
         t += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t el = (uint32_t)(t / 144), r = (uint32_t)(t % 144);
        const uint4 c = conn[e0 + el];
        const int i = (int)(r / 36), di = (int)(r / 12) % 3, j = (int)(r % 12) / 3, dj = (int)(r % 3);
        const uint32_t ni = vtx(c, i), nj = vtx(c, j);
        const uint32_t b = nbr_ptr[ni], deg = nbr_ptr[ni + 1] - b;
        const uint32_t k = pos_in(nbr + b, deg, nj);
        int32_t out = -1;
        if (k != 0xffu) {
            if (!reference) {
                out = (int32_t)(9u * b + 3u * (uint32_t)di * deg + 3u * k + (uint32_t)dj);
            } else {
                const uint32_t lo = 3u * (uint32_t)di * deg, hi = lo + 3u * deg;
                for (int sd = 2; sd >= 0; --sd) {
                    const uint32_t w = 9u * k + 3u * (uint32_t)sd + (uint32_t)dj;
                    if (w >= lo && w < hi) {
                        out = (int32_t)(9u * b + w);
                        break;
                    }
                }
            }
        }
        slot[t] = out;
    }
}

}  // namespace

void launch_slot_map(uint32_t e0, uint32_t count, const uint4* conn, const uint32_t* nbr_ptr,
                     const uint32_t* nbr, int reference, int32_t* slot, cudaStream_t s) {
    if (!count) return;
    k_slot_map<<<148 * 16, 256, 0, s>>>(e0, count, conn, nbr_ptr, nbr, reference, slot);
}

uint32_t mesh_coloring(uint32_t nn, uint32_t ne, const uint32_t* conn, uint32_t* colors) {
    const Incidence inc = build_incidence(nn, ne, conn);
    // colour of e: the smallest colour absent from the already coloured
    // (lower-numbered) tets that share a node with e
    std::vector<uint32_t> mark;  // mark[c] == e + 1: colour c is taken for e
    uint32_t n_colors = 0;
    for (uint32_t e = 0; e < ne; ++e) {
        for (int q = 0; q < 4; ++q) {
            const uint32_t n = conn[4 * (size_t)e + q];
            for (uint32_t k = inc.ptr[n]; k < inc.ptr[n + 1]; ++k) {
                const uint32_t f = inc.elem[k];
                if (f >= e) break;  // ascending: the rest are not coloured yet
                const uint32_t cf = colors[f];
                if (cf >= mark.size()) mark.resize(cf + 1, 0);
                mark[cf] = e + 1;
            }
        }
        uint32_t c = 0;
        while (c < mark.size() && mark[c] == e + 1) ++c;
        colors[e] = c;
        n_colors = std::max(n_colors, c + 1);
    }
    return n_colors;
}

}  // namespace fm
