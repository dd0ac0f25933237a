// fm_cluster.cuh — device helpers of the push solves: shared and
// distributed shared memory addressing, the cluster barrier, and the value
// slots that carry a node's three solve values between the CTAs of a
// cluster.
#pragma once

#include <cstdint>

#include "fm_sync.cuh"

namespace fm {
namespace clu {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
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
