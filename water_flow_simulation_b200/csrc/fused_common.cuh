// fused_common.cuh -- vector load/store helpers shared by the fused step kernels.
// Included inside the anonymous namespace of lbm_kernels.cu.
#pragma once

template <int V> struct Vec;
template <> struct Vec<2> {
    static __device__ __forceinline__ void load(float (&o)[2], const float* p)
    {
        const float2 t = __ldg(reinterpret_cast<const float2*>(p));
        o[0] = t.x; o[1] = t.y;
    }
    static __device__ __forceinline__ void store(float* p, float a, float b)
    {
        __stcs(reinterpret_cast<float2*>(p), make_float2(a, b));
    }
    static __device__ __forceinline__ void loadu(uint32_t (&o)[2], const uint32_t* p)
    {
        const uint2 t = __ldg(reinterpret_cast<const uint2*>(p));
        o[0] = t.x; o[1] = t.y;
    }
};
template <> struct Vec<4> {
    static __device__ __forceinline__ void load(float (&o)[4], const float* p)
    {
        const float4 t = __ldg(reinterpret_cast<const float4*>(p));
        o[0] = t.x; o[1] = t.y; o[2] = t.z; o[3] = t.w;
    }
    static __device__ __forceinline__ void store(float* p, float a, float b, float c, float d)
    {
        __stcs(reinterpret_cast<float4*>(p), make_float4(a, b, c, d));
    }
    static __device__ __forceinline__ void loadu(uint32_t (&o)[4], const uint32_t* p)
    {
        const uint4 t = __ldg(reinterpret_cast<const uint4*>(p));
        o[0] = t.x; o[1] = t.y; o[2] = t.z; o[3] = t.w;
    }
};

template <int V>
__device__ __forceinline__ void vstore(float* p, const float (&v)[V])
{
    if constexpr (V == 2) Vec<2>::store(p, v[0], v[1]);
    else Vec<4>::store(p, v[0], v[1], v[2], v[3]);
}
template <int V>
__device__ __forceinline__ void vstore_plain(float* p, const float (&v)[V])
{
    if constexpr (V == 2) *reinterpret_cast<float2*>(p) = make_float2(v[0], v[1]);
    else *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
}
template <int V>
__device__ __forceinline__ void vload_plain(float (&o)[V], const float* p)
{
    if constexpr (V == 2) { const float2 t = *reinterpret_cast<const float2*>(p); o[0] = t.x; o[1] = t.y; }
    else { const float4 t = *reinterpret_cast<const float4*>(p); o[0] = t.x; o[1] = t.y; o[2] = t.z; o[3] = t.w; }
}


// Per-direction element offsets from a cell to its pull source in an interior row
// (no wall, bed or lid involved): i*cells - cz(i)*ny*pitch - cy(i)*pitch.  Filled on the
// host and passed as a kernel parameter, so each offset is a constant-bank operand.
struct PullOffsets {
    long long d[Q];
};
