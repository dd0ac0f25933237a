// fm_sync.cuh — value-sentinel synchronization between warps of one grid.
//
// A consumer spins on a producer's output value itself: outputs are
// pre-filled with a NaN whose payload arithmetic never produces, and the
// producer's relaxed gpu-scope store of the real value is the signal.  Each
// 32/64-bit aligned word is single-copy atomic, so no separate flag (and no
// second round trip) is needed.  Every wait is bounded.
#pragma once

#include "fm_device.cuh"

namespace fm {

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

// Bounded wait for a node's three values: lanes with p != nullptr wait for
// them, and all lanes leave together (warp vote), so the warp stays
// converged for the reduction that follows.  On a timeout FM_FLAG_TIMEOUT
// is set and the values may still be sentinels.  After 16 polls the
// loop sleeps between polls, doubling from 32 ns up to sleep_ns (0: never).
template <typename T>
__device__ __forceinline__ void wait_values3_warp(const T* p, unsigned* status, unsigned sleep_ns,
                                                  T& v0, T& v1, T& v2) {
    bool need = p != nullptr;
    v0 = v1 = v2 = T(0);
    if (need) {
        v0 = ld_relaxed(p);
        v1 = ld_relaxed(p + 1);
        v2 = ld_relaxed(p + 2);
        need = Sentinel<T>::is(v0) | Sentinel<T>::is(v1) | Sentinel<T>::is(v2);
    }
    if (!__any_sync(kFull, need)) return;
    const long long t0 = clock64(), limit = wait_limit(status);
    unsigned ns = 32;
    for (unsigned it = 1;; ++it) {
        if (sleep_ns && it > 16) {
            __nanosleep(ns);
            if (ns < sleep_ns) ns <<= 1;
        }
        if (need) {
            if (Sentinel<T>::is(v0)) v0 = ld_relaxed(p);
            if (Sentinel<T>::is(v1)) v1 = ld_relaxed(p + 1);
            if (Sentinel<T>::is(v2)) v2 = ld_relaxed(p + 2);
            need = Sentinel<T>::is(v0) | Sentinel<T>::is(v1) | Sentinel<T>::is(v2);
        }
        if (!__any_sync(kFull, need)) return;
        if ((it & 63u) == 0 &&
            __any_sync(kFull, (ld_volatile_u32(status) & FM_FLAG_TIMEOUT) ||
                                  clock64() - t0 > limit)) {
            if ((threadIdx.x & 31) == 0) raise_flag(status, FM_FLAG_TIMEOUT);
            return;
        }
    }
}

}  // namespace fm
