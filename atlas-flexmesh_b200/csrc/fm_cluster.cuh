// fm_cluster.cuh — device helpers of the cluster-resident solves: shared
// and distributed shared memory addressing, cp.async and bulk copies with
// mbarrier completion, cluster barriers, and the value slots that carry a
// node's three solve values between the CTAs of a cluster.
#pragma once

#include <cstdint>

#include "fm_sync.cuh"

namespace fm {
namespace clu {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void cp_async4(uint32_t dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async8(uint32_t dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(dst), "l"(src) : "memory");
}
template <typename T>
__device__ __forceinline__ void cp_async_val(uint32_t dst, const T* src) {
    if constexpr (sizeof(T) == 4) cp_async4(dst, src);
    else cp_async8(dst, src);
}
__device__ __forceinline__ void cp_async_commit() {
    asm volatile("cp.async.commit_group;" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}
__device__ __forceinline__ void cluster_barrier() {
    asm volatile(
        "barrier.cluster.arrive.release.aligned;\n\t"
        "barrier.cluster.wait.acquire.aligned;" ::
            : "memory");
}
__device__ __forceinline__ uint32_t mapa(uint32_t addr, uint32_t cta) {
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(addr), "r"(cta));
    return r;
}
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
                 : "memory");
}
// bulk copy global -> this CTA's shared memory, completing on bar
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes,
                                         uint32_t bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
            "r"(dst),
        "l"(src), "r"(bytes), "r"(bar)
        : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait for the phase with the given parity to complete.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, unsigned* status) {
    if (mbar_try_wait(bar, parity)) return true;
    const long long t0 = clock64();
    for (unsigned it = 1;; ++it) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((it & 63u) == 0) {
            if (ld_volatile_u32(status) & FM_FLAG_TIMEOUT) return false;
            if (clock64() - t0 > kWaitCycles) {
                raise_flag(status, FM_FLAG_TIMEOUT);
                return false;
            }
        }
    }
}

// One value slot: the node's three values (padded to 16/32 bytes), each
// written once per lifetime by a relaxed cluster-scope store and polled by
// its readers until no component is the wait sentinel.
template <typename T>
__device__ __forceinline__ void ld_slot(uint32_t addr, T& a, T& b, T& c);
template <>
__device__ __forceinline__ void ld_slot<float>(uint32_t addr, float& a, float& b, float& c) {
    [[maybe_unused]] float d;
    asm volatile("ld.relaxed.cluster.shared::cluster.v4.f32 {%0, %1, %2, %3}, [%4];"
                 : "=f"(a), "=f"(b), "=f"(c), "=f"(d)
                 : "r"(addr)
                 : "memory");
}
template <>
__device__ __forceinline__ void ld_slot<double>(uint32_t addr, double& a, double& b, double& c) {
    [[maybe_unused]] double d;
    asm volatile("ld.relaxed.cluster.shared::cluster.v2.f64 {%0, %1}, [%2];"
                 : "=d"(a), "=d"(b)
                 : "r"(addr)
                 : "memory");
    asm volatile("ld.relaxed.cluster.shared::cluster.v2.f64 {%0, %1}, [%2];"
                 : "=d"(c), "=d"(d)
                 : "r"(addr + 16)
                 : "memory");
}
__device__ __forceinline__ void st_val(uint32_t addr, float v) {
    asm volatile("st.relaxed.cluster.shared::cta.f32 [%0], %1;" ::"r"(addr), "f"(v) : "memory");
}
__device__ __forceinline__ void st_val(uint32_t addr, double v) {
    asm volatile("st.relaxed.cluster.shared::cta.f64 [%0], %1;" ::"r"(addr), "d"(v) : "memory");
}
template <typename T>
__device__ __forceinline__ void st_slot(uint32_t addr, T a, T b, T c) {
    st_val(addr, a);
    st_val(addr + sizeof(T), b);
    st_val(addr + 2 * sizeof(T), c);
}
// A slot of this CTA's own shared memory, polled by its reader while a
// CTA of the cluster (possibly this one) writes it with st_slot_cluster.
template <typename T>
__device__ __forceinline__ void ld_slot_cta(uint32_t addr, T& a, T& b, T& c);
template <>
__device__ __forceinline__ void ld_slot_cta<float>(uint32_t addr, float& a, float& b, float& c) {
    [[maybe_unused]] float d;
    asm volatile("ld.relaxed.cluster.shared::cta.v4.f32 {%0, %1, %2, %3}, [%4];"
                 : "=f"(a), "=f"(b), "=f"(c), "=f"(d)
                 : "r"(addr)
                 : "memory");
}
template <>
__device__ __forceinline__ void ld_slot_cta<double>(uint32_t addr, double& a, double& b,
                                                    double& c) {
    [[maybe_unused]] double d;
    asm volatile("ld.relaxed.cluster.shared::cta.v2.f64 {%0, %1}, [%2];"
                 : "=d"(a), "=d"(b)
                 : "r"(addr)
                 : "memory");
    asm volatile("ld.relaxed.cluster.shared::cta.v2.f64 {%0, %1}, [%2];"
                 : "=d"(c), "=d"(d)
                 : "r"(addr + 16)
                 : "memory");
}
// The three values into a slot of any CTA of the cluster (addr from mapa);
// the fourth word of the slot is padding.
__device__ __forceinline__ void st_slot_cluster(uint32_t addr, float a, float b, float c) {
    asm volatile("st.relaxed.cluster.shared::cluster.v4.f32 [%0], {%1, %2, %3, %4};" ::"r"(addr),
                 "f"(a), "f"(b), "f"(c), "f"(0.f)
                 : "memory");
}
__device__ __forceinline__ void st_slot_cluster(uint32_t addr, double a, double b, double c) {
    asm volatile("st.relaxed.cluster.shared::cluster.v2.f64 [%0], {%1, %2};" ::"r"(addr), "d"(a),
                 "d"(b)
                 : "memory");
    asm volatile("st.relaxed.cluster.shared::cluster.v2.f64 [%0], {%1, %2};" ::"r"(addr + 16),
                 "d"(c), "d"(0.0)
                 : "memory");
}
}  // namespace clu
}  // namespace fm
