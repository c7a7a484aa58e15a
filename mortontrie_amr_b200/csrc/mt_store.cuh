// Population storage types shared by the dense and multi-level kernels.
//
// double: unshifted populations, FP64 arithmetic (the reference's precision).
// float / half / bfloat16: the deviation f - s_q from a storage shift is
// stored (s_q = w_q on the dense path; per level on the multi-level path),
// arithmetic is FP32.
// cv converts one stored value to the compute type.
// Index type I of ld/st: uint32_t while an array fits 2^32 elements (one wide
// multiply-add per address), int64_t beyond.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <cstdint>

namespace mt {

template <class S> struct Store;
template <> struct Store<double> {
    using C = double;
    static constexpr bool shifted = false;
    static constexpr int bytes = 8;
    template <class I> __device__ static __forceinline__ double ld(const double *p, I i) { return __ldg(p + i); }
    __device__ static __forceinline__ double cv(double v) { return v; }
    template <class I> __device__ static __forceinline__ void st(double *p, I i, double v) { p[i] = v; }
};
template <> struct Store<float> {
    using C = float;
    static constexpr bool shifted = true;
    static constexpr int bytes = 4;
    template <class I> __device__ static __forceinline__ float ld(const float *p, I i) { return __ldg(p + i); }
    __device__ static __forceinline__ float cv(float v) { return v; }
    template <class I> __device__ static __forceinline__ void st(float *p, I i, float v) { p[i] = v; }
};
template <> struct Store<__half> {
    using C = float;
    static constexpr bool shifted = true;
    static constexpr int bytes = 2;
    template <class I> __device__ static __forceinline__ float ld(const __half *p, I i)
    {
        return __half2float(__ldg(p + i));
    }
    __device__ static __forceinline__ float cv(__half v) { return __half2float(v); }
    template <class I> __device__ static __forceinline__ void st(__half *p, I i, float v) { p[i] = __float2half_rn(v); }
};
template <> struct Store<__nv_bfloat16> {
    using C = float;
    static constexpr bool shifted = true;
    static constexpr int bytes = 2;
    template <class I> __device__ static __forceinline__ float ld(const __nv_bfloat16 *p, I i)
    {
        return __bfloat162float(__ldg(p + i));
    }
    __device__ static __forceinline__ float cv(__nv_bfloat16 v) { return __bfloat162float(v); }
    template <class I> __device__ static __forceinline__ void st(__nv_bfloat16 *p, I i, float v)
    {
        p[i] = __float2bfloat16_rn(v);
    }
};

// full population value of direction k from a stored value, and back, under
// the case's storage shift (u_s = 0: the weights)
template <class S>
__device__ __forceinline__ typename Store<S>::C full_sh(const Shift &sh, typename Store<S>::C v, int k)
{
    using C = typename Store<S>::C;
    if constexpr (Store<S>::shifted)
        return v + (C)sh.v[k];
    else
        return v;
}
template <class S>
__device__ __forceinline__ typename Store<S>::C stored_sh(const Shift &sh, typename Store<S>::C v, int k)
{
    using C = typename Store<S>::C;
    if constexpr (Store<S>::shifted)
        return v - (C)sh.v[k];
    else
        return v;
}
// full value from a stored one under a shift given as its FP32 table
template <class S>
__device__ __forceinline__ typename Store<S>::C full_v(const float *shv, typename Store<S>::C v, int k)
{
    using C = typename Store<S>::C;
    if constexpr (Store<S>::shifted)
        return v + (C)shv[k];
    else
        return v;
}
// the stored value of an FP64 population (subtraction in FP64, one rounding)
template <class S> __device__ __forceinline__ typename Store<S>::C stored_f64(const Shift &sh, double v, int k)
{
    using C = typename Store<S>::C;
    if constexpr (Store<S>::shifted)
        return (C)(v - sh.d[k]);
    else
        return (C)v;
}

}  // namespace mt
