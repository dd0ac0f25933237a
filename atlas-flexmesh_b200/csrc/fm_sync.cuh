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

// Spin (bounded) until *p is not the sentinel; returns the value, or the
// sentinel when the wait gave up (FM_FLAG_TIMEOUT then set).
// backoff_ns > 0: sleep between polls, doubling from backoff_ns up to 8x,
// which keeps thousands of early waiters from flooding L2 with polls.
template <typename T>
__device__ __forceinline__ T wait_value(const T* p, unsigned* status, unsigned backoff_ns = 0) {
    T v = ld_relaxed(p);
    if (!Sentinel<T>::is(v)) return v;
    const long long t0 = clock64();
    unsigned ns = backoff_ns;
    for (unsigned it = 1;; ++it) {
        if (ns) {
            __nanosleep(ns);
            if (ns < 8 * backoff_ns) ns <<= 1;
        }
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

// Three consecutive values (one node's block) with the polls in flight
// together: one round trip when they are ready, not three.
template <typename T>
__device__ __forceinline__ void wait_values3(const T* p, unsigned* status, T& v0, T& v1, T& v2) {
    v0 = ld_relaxed(p);
    v1 = ld_relaxed(p + 1);
    v2 = ld_relaxed(p + 2);
    if (!(Sentinel<T>::is(v0) | Sentinel<T>::is(v1) | Sentinel<T>::is(v2))) return;
    const long long t0 = clock64();
    for (unsigned it = 1;; ++it) {
        if (Sentinel<T>::is(v0)) v0 = ld_relaxed(p);
        if (Sentinel<T>::is(v1)) v1 = ld_relaxed(p + 1);
        if (Sentinel<T>::is(v2)) v2 = ld_relaxed(p + 2);
        if (!(Sentinel<T>::is(v0) | Sentinel<T>::is(v1) | Sentinel<T>::is(v2))) return;
        if ((it & 63u) == 0) {
            if (ld_volatile_u32(status) & FM_FLAG_TIMEOUT) return;
            if (clock64() - t0 > kWaitCycles) {
                raise_flag(status, FM_FLAG_TIMEOUT);
                return;
            }
        }
    }
}

// Warp-uniform form of wait_values3: lanes with p != nullptr wait for their
// node's three values, and all lanes leave together (warp vote), so the
// warp stays converged for the reduction that follows.  After 16 polls the
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
    const long long t0 = clock64();
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
                                  clock64() - t0 > kWaitCycles)) {
            if ((threadIdx.x & 31) == 0) raise_flag(status, FM_FLAG_TIMEOUT);
            return;
        }
    }
}

}  // namespace fm
