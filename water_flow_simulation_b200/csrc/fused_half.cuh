// fused_half.cuh -- the split (work-list) pipeline over 16-bit population storage.
// Included inside the anonymous namespace of lbm_kernels.cu, after fused_split.cuh.
//
// Storage: h_i = fp16_rn((f_i - w_i) * scale) in the SoA layout of the float path
// (h[i*cells + c]), scale a per-lattice power of two.  Collision stays in FP32.  A step
// moves 2 x 19 x 2 = 76 bytes per cell instead of 152.
//
// Work lists are built over row segments of 32*cpl cells (cpl = cells_per_lane 2, 4 or 8:
// 64, 128 or 256 cells), and pitch is a multiple of 8 so every 8-cell group is one aligned
// 16-byte vector.
//   k_rows_h_plain    plain segments: a lane moves VP = 8 (or 4) cells with one 16-byte (8-byte)
//                     load/store per direction, 32*cpl/VP lanes per segment; the +-1 x
//                     neighbours are one shuffle and VP/2 byte permutes on the packed halves;
//                     the collision works on deviations directly (moments of f - w), two
//                     cells at a time.
//   k_rows_edge       edge segments and
//   k_rows_h_general  special segments: the edge and general paths of fused_split.cuh with
//                     T = __half, 2 cells per lane (4-byte accesses) for 64-cell segments,
//                     else 4 (8-byte accesses) in one or two passes.
#pragma once

// Regularized-BGK + Smagorinsky collision without body force, on deviations: `d` holds
// raw storage values (f_i - w_i) * scale on entry and on exit.  Same update as collide():
// with dr = rho - 1 and S = sum c c (f - w) (so that sum c c f = I/3 + S), the
// non-equilibrium stress is Pi = S - rho u u - dr I/3, and the post-collision deviation is
// w_i [ (A0 - 1) + c.B + c.C.c ].
__device__ __forceinline__ void collide_dev(float (&d)[Q], float scale, float inv_scale, float tau0, float csmag2,
                                            float& r, float& ux, float& uy, float& uz)
{
    const float s1 = d[1] + d[2], d1 = d[1] - d[2];
    const float s3 = d[3] + d[4], d3 = d[3] - d[4];
    const float s5 = d[5] + d[6], d5 = d[5] - d[6];
    const float s7 = d[7] + d[8], d7 = d[7] - d[8];
    const float s9 = d[9] + d[10], d9 = d[9] - d[10];
    const float s11 = d[11] + d[12], d11 = d[11] - d[12];
    const float s13 = d[13] + d[14], d13 = d[13] - d[14];
    const float s15 = d[15] + d[16], d15 = d[15] - d[16];
    const float s17 = d[17] + d[18], d17 = d[17] - d[18];
    const float dr = (d[0] + (s1 + s3 + s5) + (s7 + s9 + s11) + (s13 + s15 + s17)) * inv_scale;
    r = 1.0f + dr;
    const float jx = (d1 + d7 + d9 + d11 + d13) * inv_scale;
    const float jy = (d3 + d7 - d9 + d15 + d17) * inv_scale;
    const float jz = (d5 + d11 - d13 + d15 - d17) * inv_scale;
    const float sxx = (s1 + s7 + s9 + s11 + s13) * inv_scale;
    const float syy = (s3 + s7 + s9 + s15 + s17) * inv_scale;
    const float szz = (s5 + s11 + s13 + s15 + s17) * inv_scale;
    const float sxy = (s7 - s9) * inv_scale, sxz = (s11 - s13) * inv_scale, syz = (s15 - s17) * inv_scale;

    const float ir = 1.0f / r;
    ux = jx * ir;
    uy = jy * ir;
    uz = jz * ir;
    const float dr3 = dr * (1.0f / 3.0f);
    const float pxx = sxx - r * ux * ux - dr3, pyy = syy - r * uy * uy - dr3, pzz = szz - r * uz * uz - dr3;
    const float pxy = sxy - r * ux * uy, pxz = sxz - r * ux * uz, pyz = syz - r * uy * uz;

    const float qn = sqrtf(pxx * pxx + pyy * pyy + pzz * pzz + 2.0f * (pxy * pxy + pxz * pxz + pyz * pyz));
    // tau0^2 and 18 sqrt(2) Cs^2 are rounded explicitly: they are lattice constants, and a compiler
    // that hoists them out of a loop (or not) must not change how they fuse into what follows
    const float tau0sq = mul_rn(tau0, tau0), smag = mul_rn(18.0f * 1.41421356f, csmag2);
    const float tau = 0.5f * (tau0 + sqrtf(tau0sq + smag * qn * ir));
    const float om = 1.0f / tau;
    const float k1 = 1.0f - om;

    const float usq = ux * ux + uy * uy + uz * uz;
    const float A0 = dr - 1.5f * (r * usq + k1 * (pxx + pyy + pzz));
    const float Bx = 3.0f * r * ux, By = 3.0f * r * uy, Bz = 3.0f * r * uz;
    const float Cxx = 4.5f * (r * ux * ux + k1 * pxx);
    const float Cyy = 4.5f * (r * uy * uy + k1 * pyy);
    const float Czz = 4.5f * (r * uz * uz + k1 * pzz);
    const float Cxy2 = 9.0f * (r * ux * uy + k1 * pxy);
    const float Cxz2 = 9.0f * (r * ux * uz + k1 * pxz);
    const float Cyz2 = 9.0f * (r * uy * uz + k1 * pyz);

    const float w0 = wgt(0) * scale, w1 = wgt(1) * scale, w2 = wgt(7) * scale;
    d[0] = w0 * A0;
    float b;
    b = A0 + Cxx;                 d[1] = w1 * (b + Bx);  d[2] = w1 * (b - Bx);
    b = A0 + Cyy;                 d[3] = w1 * (b + By);  d[4] = w1 * (b - By);
    b = A0 + Czz;                 d[5] = w1 * (b + Bz);  d[6] = w1 * (b - Bz);
    b = A0 + Cxx + Cyy + Cxy2;    d[7] = w2 * (b + (Bx + By));  d[8] = w2 * (b - (Bx + By));
    b = A0 + Cxx + Cyy - Cxy2;    d[9] = w2 * (b + (Bx - By));  d[10] = w2 * (b - (Bx - By));
    b = A0 + Cxx + Czz + Cxz2;    d[11] = w2 * (b + (Bx + Bz)); d[12] = w2 * (b - (Bx + Bz));
    b = A0 + Cxx + Czz - Cxz2;    d[13] = w2 * (b + (Bx - Bz)); d[14] = w2 * (b - (Bx - Bz));
    b = A0 + Cyy + Czz + Cyz2;    d[15] = w2 * (b + (By + Bz)); d[16] = w2 * (b - (By + Bz));
    b = A0 + Cyy + Czz - Cyz2;    d[17] = w2 * (b + (By - Bz)); d[18] = w2 * (b - (By - Bz));
}

// Pull of direction I for the VP cells (VP = 4 or 8) of a lane in an interior row, packed:
// word j of h[I] holds cells 2j (low half) and 2j+1 (high half).  A +x mover takes element
// x-1: word j = (high half of source word j-1, low half of source word j); word -1 is the
// left lane's last word (at a segment's first lane: the 4-byte word just left of the
// segment).  A -x mover takes element x+1 symmetrically, word VP/2 from the right lane.
// G lanes share a segment (shuffles of width G).
template <int VP> struct HVec;
template <> struct HVec<4> {
    static __device__ __forceinline__ void load(uint32_t (&t)[2], const __half* p)
    {
        const uint2 v = __ldg(reinterpret_cast<const uint2*>(p));
        t[0] = v.x; t[1] = v.y;
    }
    static __device__ __forceinline__ void store(__half* p, const uint32_t (&t)[2])
    {
        *reinterpret_cast<uint2*>(p) = make_uint2(t[0], t[1]);
    }
};
// Stores are plain write-back stores: for this kernel they measured 2.7 % faster than
// streaming (.cs) stores on reach36m, while the float32 kernels keep .cs stores (6 % slower
// without); .cs, .nc.L1::no_allocate loads were 9-11 % slower than the default __ldg.
template <> struct HVec<8> {
    static __device__ __forceinline__ void load(uint32_t (&t)[4], const __half* p)
    {
        const uint4 v = __ldg(reinterpret_cast<const uint4*>(p));
        t[0] = v.x; t[1] = v.y; t[2] = v.z; t[3] = v.w;
    }
    static __device__ __forceinline__ void store(__half* p, const uint32_t (&t)[4])
    {
        *reinterpret_cast<uint4*>(p) = make_uint4(t[0], t[1], t[2], t[3]);
    }
};

// Packed loads of VP cells and of one 4-byte word: read-only path for __half, coherent for hcoh.
template <int VP>
__device__ __forceinline__ void hload(uint32_t (&t)[VP / 2], const __half* p) { HVec<VP>::load(t, p); }
template <int VP>
__device__ __forceinline__ void hload(uint32_t (&t)[VP / 2], const hcoh* p)
{
    if constexpr (VP == 8) {
        const uint4 v = __ldcg(reinterpret_cast<const uint4*>(p));
        t[0] = v.x; t[1] = v.y; t[2] = v.z; t[3] = v.w;
    } else {
        const uint2 v = __ldcg(reinterpret_cast<const uint2*>(p));
        t[0] = v.x; t[1] = v.y;
    }
}
__device__ __forceinline__ uint32_t hword(const __half* p) { return __ldg(reinterpret_cast<const unsigned int*>(p)); }
__device__ __forceinline__ uint32_t hword(const hcoh* p) { return __ldcg(reinterpret_cast<const unsigned int*>(p)); }

template <int I, int VP, int G, typename T>
__device__ __forceinline__ void hpull_dir(uint32_t (&h)[Q][VP / 2], const T* __restrict__ own_ptr,
                                          const PullOffsets& po, int gl, bool lid)
{
    constexpr int CXI = cx(I), NW = VP / 2;
    const T* src = own_ptr + pull_offset<I>(po, lid);
    uint32_t t[NW];
    hload<VP>(t, src);
    if constexpr (CXI == 0) {
#pragma unroll
        for (int j = 0; j < NW; ++j) h[I][j] = t[j];
    } else if constexpr (CXI == 1) {
        uint32_t prev = __shfl_up_sync(0xffffffffu, t[NW - 1], 1, G);
        if (gl == 0) prev = hword(src - 2);
        h[I][0] = __byte_perm(prev, t[0], 0x5432);
#pragma unroll
        for (int j = 1; j < NW; ++j) h[I][j] = __byte_perm(t[j - 1], t[j], 0x5432);
    } else {
        uint32_t next = __shfl_down_sync(0xffffffffu, t[0], 1, G);
        if (gl == G - 1) next = hword(src + VP);
#pragma unroll
        for (int j = 0; j < NW - 1; ++j) h[I][j] = __byte_perm(t[j], t[j + 1], 0x5432);
        h[I][NW - 1] = __byte_perm(t[NW - 1], next, 0x5432);
    }
}
template <int VP, int G, typename T, int... Is>
__device__ __forceinline__ void hpull_all(std::integer_sequence<int, Is...>, uint32_t (&h)[Q][VP / 2],
                                          const T* __restrict__ own_ptr, const PullOffsets& po, int gl,
                                          bool lid)
{
    (hpull_dir<Is, VP, G, T>(h, own_ptr, po, gl, lid), ...);
}

// One plain segment (row-segment id `id`) for the G lanes of a group: lane gl of the group
// moves VP cells.  Every lane of the warp calls it together (shuffles); `store` false: the
// group recomputes a segment another group owns and writes nothing.
template <int VP, int G, bool OUT, bool AVG, typename T = __half>
__device__ __forceinline__ void h_plain_segment(const lbm_lattice& L, const PullOffsets& po,
                                                const T* __restrict__ fs, T* __restrict__ fd, float scale,
                                                uint32_t id, int gl, bool store)
{
    constexpr int NW = VP / 2, SEG = VP * G;
    const int nseg = (L.pitch + SEG - 1) / SEG;
    const long long S = L.cells;
    const float inv_scale = 1.0f / scale;
    int seg, y, z;
    decode_row(id, nseg, L.ny, seg, y, z);
    const long long own = ((long long)z * L.ny + y) * L.pitch + seg * SEG + gl * VP;
    uint32_t h[Q][NW];
    hpull_all<VP, G, T>(std::make_integer_sequence<int, Q>{}, h, fs + own, po, gl, z == L.nz - 1);
    float R[VP], UX[VP], UY[VP], UZ[VP];
#pragma unroll
    for (int p = 0; p < NW; ++p) {
        float a[Q], c[Q];
#pragma unroll
        for (int i = 0; i < Q; ++i) {
            const float2 v = half2_bits_to_float2(h[i][p]);
            a[i] = v.x; c[i] = v.y;
        }
        collide_dev(a, scale, inv_scale, L.tau0, L.csmag2, R[2 * p], UX[2 * p], UY[2 * p], UZ[2 * p]);
        collide_dev(c, scale, inv_scale, L.tau0, L.csmag2, R[2 * p + 1], UX[2 * p + 1], UY[2 * p + 1], UZ[2 * p + 1]);
#pragma unroll
        for (int i = 0; i < Q; ++i) h[i][p] = float2_to_half2_bits(a[i], c[i]);
    }
    if (!store) return;
#pragma unroll
    for (int i = 0; i < Q; ++i) HVec<VP>::store(reinterpret_cast<__half*>(fd) + (long long)i * S + own, h[i]);
    if constexpr (OUT) {
        store_fields<VP, AVG>(L, own, R, UX, UY, UZ);
        bool bad = false;
#pragma unroll
        for (int k = 0; k < VP; ++k) bad |= !(R[k] > 0.f && R[k] < 3.4e38f);
        if (bad) atomicOr(L.status, 1);
    }
}

// Plain list over segments of VP*G cells: a warp takes 32/G consecutive list entries per
// pass, G lanes (VP cells each) per segment.  In the last pass, groups past the end of the
// list repeat the pass's first segment and store nothing (every lane still takes part in
// the shuffles).
template <int VP, int G, bool OUT, bool AVG>
__global__ void __launch_bounds__(128, VP == 8 ? 3 : 4) k_rows_h_plain(const lbm_lattice L, const PullOffsets po,
                                                                      const uint32_t* __restrict__ list, int nlist,
                                                                      const __half* __restrict__ fs,
                                                                      __half* __restrict__ fd, float scale)
{
    constexpr int PER_WARP = 32 / G;
    const int lane = threadIdx.x & 31, gl = lane % G, grp = lane / G;
    const int gw = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), W = (int)((gridDim.x * blockDim.x) >> 5);
    for (long long b = (long long)gw * PER_WARP; b < nlist; b += (long long)W * PER_WARP) {
        const bool valid = b + grp < nlist;
        const uint32_t id = __ldg(list + (valid ? b + grp : b));
        h_plain_segment<VP, G, OUT, AVG>(L, po, fs, fd, scale, id, gl, valid);
    }
}

// 16-bit start state: the float path's initial populations (k_init_equilibrium), stored as
// scaled deviations.
__global__ void k_init_equilibrium_h(const lbm_lattice L, __half* __restrict__ h, float scale)
{
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= L.cells) return;
    const int x = (int)(c % L.pitch), y = (int)((c / L.pitch) % L.ny), z = (int)(c / ((long long)L.pitch * L.ny));
    const bool fluid = x < L.nx && !(L.flags[c] & FLAG_SOLID);
    const float u = fluid ? L.uin[y + (long long)L.ny * z] : 0.f;
    const double ud = (double)u;
    const float q = __fmul_rn(__fmul_rn(1.5f, u), u);
#pragma unroll
    for (int i = 0; i < Q; ++i) {
        const double cu = __dmul_rn((double)(3 * cx(i)), ud);
        const double poly = __dsub_rn(__dadd_rn(__dadd_rn(1.0, cu), __dmul_rn(__dmul_rn(0.5, cu), cu)), (double)q);
        const float f = __double2float_rn(__dmul_rn(wgt64(i), poly));
        h[(long long)i * L.cells + c] = __float2half_rn(__fmul_rn(__fsub_rn(f, wgt(i)), scale));
    }
}

// float populations <-> 16-bit storage, n = 19*cells elements (direction i = element / cells).
__global__ void k_pack_populations(const float* __restrict__ f, __half* __restrict__ h, long long cells, float scale)
{
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (long long)Q * cells) return;
    const int i = (int)(e / cells);
    const float w = i == 0 ? wgt(0) : (i < 7 ? wgt(1) : wgt(7));
    h[e] = __float2half_rn(__fmul_rn(__fsub_rn(f[e], w), scale));
}
__global__ void k_unpack_populations(const __half* __restrict__ h, float* __restrict__ f, long long cells,
                                     float inv_scale)
{
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (long long)Q * cells) return;
    const int i = (int)(e / cells);
    const float w = i == 0 ? wgt(0) : (i < 7 ? wgt(1) : wgt(7));
    f[e] = __fadd_rn(w, __fmul_rn(__half2float(h[e]), inv_scale));
}
