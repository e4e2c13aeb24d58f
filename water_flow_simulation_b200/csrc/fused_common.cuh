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
    else if constexpr (V == 4) *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
    else {
        reinterpret_cast<float4*>(p)[0] = make_float4(v[0], v[1], v[2], v[3]);
        reinterpret_cast<float4*>(p)[1] = make_float4(v[4], v[5], v[6], v[7]);
    }
}
template <int V>
__device__ __forceinline__ void vload_plain(float (&o)[V], const float* p)
{
    if constexpr (V == 2) { const float2 t = *reinterpret_cast<const float2*>(p); o[0] = t.x; o[1] = t.y; }
    else {
#pragma unroll
        for (int q = 0; q < V / 4; ++q) {
            const float4 t = reinterpret_cast<const float4*>(p)[q];
            o[4 * q] = t.x; o[4 * q + 1] = t.y; o[4 * q + 2] = t.z; o[4 * q + 3] = t.w;
        }
    }
}

// ---------------------------------------------------------------------------------------------
// Population storage.  The pull code is written once over the element type T of the
// population arrays:
//   float  -- the reference's layout and values;
//   __half -- 16-bit storage: element = fp16_rn((f_i - w_i) * scale), the deviation of the
//             population from its lattice weight times a per-lattice power of two (exact, so
//             the scale moves only the fp16 exponent range: |f_i - w_i| < 65504/scale, and
//             deviations above 2^-14/scale keep the full 11-bit significand).
// ldv/ld1 load raw element values as float (for __half: the scaled deviation); every pull
// phase only moves values, and the weight of the direction a value is read from always equals
// the weight of the direction it lands in (w_opp(i) = w_mirz(i) = w_i), so 16-bit values become
// populations after the pull: f_i = w_i + raw / scale.
// ---------------------------------------------------------------------------------------------
template <int V>
__device__ __forceinline__ void ldv(float (&o)[V], const float* p) { Vec<V>::load(o, p); }
__device__ __forceinline__ float ld1(const float* p) { return __ldg(p); }

__device__ __forceinline__ float2 half2_bits_to_float2(uint32_t b)
{
    __half2 h;
    memcpy(&h, &b, 4);
    return __half22float2(h);
}
__device__ __forceinline__ uint32_t float2_to_half2_bits(float lo, float hi)
{
    const __half2 h = __floats2half2_rn(lo, hi);
    uint32_t b;
    memcpy(&b, &h, 4);
    return b;
}

template <int V>
__device__ __forceinline__ void ldv(float (&o)[V], const __half* p)
{
    static_assert(V == 2 || V == 4, "16-bit general path moves 2 or 4 cells per lane");
    if constexpr (V == 2) {
        const float2 a = half2_bits_to_float2(__ldg(reinterpret_cast<const unsigned int*>(p)));
        o[0] = a.x; o[1] = a.y;
    } else {
        const uint2 t = __ldg(reinterpret_cast<const uint2*>(p));
        const float2 a = half2_bits_to_float2(t.x), b = half2_bits_to_float2(t.y);
        o[0] = a.x; o[1] = a.y; o[2] = b.x; o[3] = b.y;
    }
}
__device__ __forceinline__ float ld1(const __half* p) { return __half2float(__ldg(p)); }

// 16-bit storage read through coherent loads (ld.global.cg, served by L2): for a kernel that
// reads populations which other CTAs wrote earlier in the same launch (the persistent batch
// chunk).  __ldg's read-only path may keep lines from before such writes, so it is only for
// data that stays unchanged for a whole launch.  Same bits and layout as __half.
struct __align__(2) hcoh {
    __half h;
};
template <int V>
__device__ __forceinline__ void ldv(float (&o)[V], const hcoh* p)
{
    static_assert(V == 2 || V == 4, "16-bit general path moves 2 or 4 cells per lane");
    if constexpr (V == 2) {
        const float2 a = half2_bits_to_float2(__ldcg(reinterpret_cast<const unsigned int*>(p)));
        o[0] = a.x; o[1] = a.y;
    } else {
        const uint2 t = __ldcg(reinterpret_cast<const uint2*>(p));
        const float2 a = half2_bits_to_float2(t.x), b = half2_bits_to_float2(t.y);
        o[0] = a.x; o[1] = a.y; o[2] = b.x; o[3] = b.y;
    }
}
__device__ __forceinline__ float ld1(const hcoh* p) { return __half2float(__ldcg(reinterpret_cast<const __half*>(p))); }

// f (after the pull) from raw element values: identity for float storage.
template <typename T, int V>
__device__ __forceinline__ void raw_to_pop(float (&f)[V][Q], float inv_scale)
{
    if constexpr (!std::is_same<T, float>::value) {
#pragma unroll
        for (int k = 0; k < V; ++k)
#pragma unroll
            for (int i = 0; i < Q; ++i) f[k][i] = fmaf(f[k][i], inv_scale, wgt(i));
    }
}

// Streaming store of direction I of V cells.
template <int I, int V>
__device__ __forceinline__ void stv(float* p, const float (&v)[V], float) { vstore<V>(p, v); }
template <int I, int V>
__device__ __forceinline__ void stv(__half* p, const float (&v)[V], float scale);
template <int I, int V>
__device__ __forceinline__ void stv(hcoh* p, const float (&v)[V], float scale)
{
    stv<I, V>(reinterpret_cast<__half*>(p), v, scale);
}
template <int I, int V>
__device__ __forceinline__ void stv(__half* p, const float (&v)[V], float scale)
{
    static_assert(V == 2 || V == 4, "16-bit general path moves 2 or 4 cells per lane");
    constexpr float w = wgt(I);
    if constexpr (V == 2) {
        __stcs(reinterpret_cast<unsigned int*>(p), float2_to_half2_bits((v[0] - w) * scale, (v[1] - w) * scale));
    } else {
        __stcs(reinterpret_cast<uint2*>(p), make_uint2(float2_to_half2_bits((v[0] - w) * scale, (v[1] - w) * scale),
                                                       float2_to_half2_bits((v[2] - w) * scale, (v[3] - w) * scale)));
    }
}


// Per-direction element offsets from a cell to its pull source in an interior row
// (no wall, bed or lid involved): i*cells - cz(i)*ny*pitch - cy(i)*pitch; and in an open
// row under the rigid lid (z = nz-1), where a -z mover takes the cell's own mirrored
// population one row over in y (floodsim/lbm3d.py:54): mirz(i)*cells - cy(i)*pitch.
// Filled on the host and passed as a kernel parameter, so each offset is a constant-bank
// operand.
struct PullOffsets {
    long long d[Q];
    long long lid[Q];
};
template <int I>
__device__ __forceinline__ long long pull_offset(const PullOffsets& po, bool lid)
{
    if constexpr (cz(I) == -1) return lid ? po.lid[I] : po.d[I];
    else return po.d[I];
}

// One population of direction i (scalar; i need not be a compile-time constant).
__device__ __forceinline__ float ldpop(const float* p, int, float) { return *p; }
__device__ __forceinline__ float ldpop(const __half* p, int i, float inv_scale)
{
    return fmaf(__half2float(*p), inv_scale, wgt(i));
}
__device__ __forceinline__ void stpop(float* p, int, float v, float) { *p = v; }
__device__ __forceinline__ void stpop(__half* p, int i, float v, float scale) { *p = __float2half_rn((v - wgt(i)) * scale); }
__device__ __forceinline__ float ldpop(const hcoh* p, int i, float inv_scale)
{
    return fmaf(__half2float(__ldcg(reinterpret_cast<const __half*>(p))), inv_scale, wgt(i));
}
__device__ __forceinline__ void stpop(hcoh* p, int i, float v, float scale)
{
    stpop(reinterpret_cast<__half*>(p), i, v, scale);
}

