// fused_reg.cuh -- register/shuffle pipeline of the fused step (lbm_tile.pipeline = 0).
// Included inside the anonymous namespace of lbm_kernels.cu.
//
// A warp covers 32*V consecutive x cells of one (y,z) row; each lane owns V cells and
// moves them with V-wide loads and stores, the +-1 x neighbours arriving by warp shuffle.
#pragma once

// ---------------------------------------------------------------------------------------------
// Pull streaming for the V cells of a lane (floodsim/lbm3d.py:50-60 semantics), in phases so
// that all 19 row loads (and the 10 halo loads) are in flight together:
//   A  branch-free: per direction, the source row (or, for a row outside the domain, the
//      cell's own opposite population) as one V-wide load, plus a scalar halo load;
//   B  shuffles: x-shifted directions take the neighbour lane's element (halo at the
//      segment's first/last lane);
//   C  bounce-back from solid neighbours, only in lanes whose cells have any;
//   D  x edges: a direction whose source lies outside [0, nx) keeps the own population.
// ---------------------------------------------------------------------------------------------
template <typename T>
struct PullCtxT {
    const T* fs;
    long long S, rowc, own;   // own = rowc + x0c (load start, clamped into the row)
    int x0, x0c, y, z, lane;
};
using PullCtx = PullCtxT<float>;

template <int I, int V, typename T>
__device__ __forceinline__ void pull_load(float (&t)[Q][V], float (&hv)[Q], uint32_t& rwm, const lbm_lattice& L,
                                          const PullCtxT<T>& c)
{
    constexpr int CXI = cx(I), CYI = cy(I), CZI = cz(I);
    if constexpr (I == 0) {
        ldv<V>(t[0], c.fs + c.own);
    } else {
        int ys = c.y - CYI, zs = c.z - CZI, di = I;
        if (CZI == -1 && c.z == L.nz - 1) { zs = c.z; di = mirz(I); }   // rigid lid: mirrored population
        const bool rowwall = (ys < 0) || (ys >= L.ny) || (zs < 0);      // warp-uniform
        const T* row = rowwall ? c.fs + (long long)opp(I) * c.S + c.rowc
                               : c.fs + (long long)di * c.S + ((long long)zs * L.ny + ys) * L.pitch;
        ldv<V>(t[I], row + c.x0c);
        if constexpr (CXI == 1) hv[I] = ld1(row + (c.x0c > 0 ? c.x0c - 1 : 0));
        if constexpr (CXI == -1) hv[I] = ld1(row + (c.x0c + V < L.pitch ? c.x0c + V : L.pitch - 1));
        rwm |= rowwall ? (1u << I) : 0u;
    }
}

template <int I, int V>
__device__ __forceinline__ void pull_shift(float (&f)[V][Q], float (&t)[Q][V], const float (&hv)[Q], uint32_t rwm,
                                           int lane)
{
    constexpr int CXI = cx(I);
    if constexpr (CXI == 0) {
#pragma unroll
        for (int k = 0; k < V; ++k) f[k][I] = t[I][k];
    } else if constexpr (CXI == 1) {
        float h = __shfl_up_sync(0xffffffffu, t[I][V - 1], 1);
        if (lane == 0) h = hv[I];
        const bool rw = rwm & (1u << I);
        f[0][I] = rw ? t[I][0] : h;
#pragma unroll
        for (int k = 1; k < V; ++k) f[k][I] = rw ? t[I][k] : t[I][k - 1];
    } else {
        float h = __shfl_down_sync(0xffffffffu, t[I][0], 1);
        if (lane == 31) h = hv[I];
        const bool rw = rwm & (1u << I);
#pragma unroll
        for (int k = 0; k < V - 1; ++k) f[k][I] = rw ? t[I][k] : t[I][k + 1];
        f[V - 1][I] = rw ? t[I][V - 1] : h;
    }
}

template <int I, int V, typename T>
__device__ __forceinline__ void pull_bounce(float (&f)[V][Q], const uint32_t (&fl)[V], uint32_t bb,
                                            const PullCtxT<T>& c)
{
    if constexpr (I > 0) {
        if (bb & (1u << I)) {
            float b[V];
            ldv<V>(b, c.fs + (long long)opp(I) * c.S + c.own);
#pragma unroll
            for (int k = 0; k < V; ++k)
                if (fl[k] & (1u << I)) f[k][I] = b[k];
        }
    }
}

template <int I, int V, typename T>
__device__ __forceinline__ void pull_edge(float (&f)[V][Q], const lbm_lattice& L, const PullCtxT<T>& c)
{
    constexpr int CXI = cx(I);
    if constexpr (CXI == 1) {
        if (c.x0 == 0) f[0][I] = ld1(c.fs + (long long)I * c.S + c.rowc);
    } else if constexpr (CXI == -1) {
#pragma unroll
        for (int k = 0; k < V; ++k)
            if (c.x0 + k == L.nx - 1) f[k][I] = ld1(c.fs + (long long)I * c.S + c.rowc + L.nx - 1);
    }
}

// Rows on the y walls, the bed or the lid: per-direction source rows (phases A and B).
// Returns the mask of directions whose source row lies outside the domain.
template <int V, typename T, int... Is>
__device__ __forceinline__ uint32_t pull_rows(std::integer_sequence<int, Is...>, float (&f)[V][Q],
                                              const lbm_lattice& L, const PullCtxT<T>& c)
{
    float t[Q][V];
    float hv[Q];
    uint32_t rwm = 0;
    (pull_load<Is, V, T>(t, hv, rwm, L, c), ...);
    (pull_shift<Is, V>(f, t, hv, rwm, c.lane), ...);
    return rwm;
}
template <int V, typename T, int... Is>
__device__ __forceinline__ void pull_edges(std::integer_sequence<int, Is...>, float (&f)[V][Q], const lbm_lattice& L,
                                           const PullCtxT<T>& c)
{
    (pull_edge<Is, V, T>(f, L, c), ...);                            // phase D only
}
template <int V, typename T, int... Is>
__device__ __forceinline__ void pull_fixups(std::integer_sequence<int, Is...>, float (&f)[V][Q], const lbm_lattice& L,
                                            const PullCtxT<T>& c, const uint32_t (&fl)[V], uint32_t bb)
{
    if (bb) { (pull_bounce<Is, V, T>(f, fl, bb, c), ...); }         // phase C
    const bool edge = (c.x0 == 0) || (c.x0 <= L.nx - 1 && L.nx - 1 < c.x0 + V);
    if (edge) { (pull_edge<Is, V, T>(f, L, c), ...); }              // phase D
}

// Pull for the segment of an interior row (no y wall or bed involved; `lid`: the row under
// the rigid lid): every source is own + a constant offset; the segment's first/last lane
// fetch the one halo element.  At the x
// edges and in padding lanes the values are fixed up (or discarded) afterwards; every
// address stays inside the population array because an interior row has rows on both sides.
template <int I, int V, typename T>
__device__ __forceinline__ void pull_fast_dir(float (&f)[V][Q], const T* __restrict__ own_ptr,
                                              const PullOffsets& po, int lane, bool lid)
{
    constexpr int CXI = cx(I);
    const T* src = own_ptr + pull_offset<I>(po, lid);
    float t[V];
    ldv<V>(t, src);
    if constexpr (CXI == 0) {
#pragma unroll
        for (int k = 0; k < V; ++k) f[k][I] = t[k];
    } else if constexpr (CXI == 1) {
        float h = __shfl_up_sync(0xffffffffu, t[V - 1], 1);
        if (lane == 0) h = ld1(src - 1);
        f[0][I] = h;
#pragma unroll
        for (int k = 1; k < V; ++k) f[k][I] = t[k - 1];
    } else {
        float h = __shfl_down_sync(0xffffffffu, t[0], 1);
        if (lane == 31) h = ld1(src + V);
#pragma unroll
        for (int k = 0; k < V - 1; ++k) f[k][I] = t[k + 1];
        f[V - 1][I] = h;
    }
}
template <int V, typename T, int... Is>
__device__ __forceinline__ void pull_fast_all(std::integer_sequence<int, Is...>, float (&f)[V][Q],
                                              const T* __restrict__ own_ptr, const PullOffsets& po, int lane,
                                              bool lid = false)
{
    (pull_fast_dir<Is, V, T>(f, own_ptr, po, lane, lid), ...);
}

template <int V, bool OUT, bool UCOL, bool AVG>
__global__ void __launch_bounds__(128, V == 4 ? 3 : 4) k_fused(const lbm_lattice L, const PullOffsets po,
                                                              const float* __restrict__ fs, float* __restrict__ fd)
{
    extern __shared__ float sh[];  // column partial sums, only for OUT && UCOL
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    constexpr int SEG = 32 * V;
    const int nseg = (L.pitch + SEG - 1) / SEG;
    const int nitems = nseg * L.ny;
    const long long S = L.cells;

    for (int item = blockIdx.x; item < nitems; item += gridDim.x) {
        const int seg = item % nseg, y = item / nseg;
        const int x0 = seg * SEG + lane * V;
        const bool active = x0 < L.pitch;
        const int x0c = active ? x0 : L.pitch - V;   // inactive lanes load (and discard) the row's last vector
        float csx[V], csy[V], ccn[V];
#pragma unroll
        for (int k = 0; k < V; ++k) { csx[k] = 0.f; csy[k] = 0.f; ccn[k] = 0.f; }

        // flag words are fetched one row ahead, so a row's special cases are known before
        // its populations are requested
        uint32_t fl_next[V];
#pragma unroll
        for (int k = 0; k < V; ++k) fl_next[k] = FLAG_GHOST | FLAG_SOLID;
        if (warp < L.nz) Vec<V>::loadu(fl_next, L.flags + ((long long)warp * L.ny + y) * L.pitch + x0c);

        for (int z = warp; z < L.nz; z += nwarps) {
            const long long rowc = ((long long)z * L.ny + y) * L.pitch;
            const long long own = rowc + x0;
            PullCtx pc{fs, S, rowc, rowc + x0c, x0, x0c, y, z, lane};
            uint32_t fl[V];
#pragma unroll
            for (int k = 0; k < V; ++k) fl[k] = active ? fl_next[k] : (FLAG_GHOST | FLAG_SOLID);
            if (z + nwarps < L.nz)
                Vec<V>::loadu(fl_next, L.flags + ((long long)(z + nwarps) * L.ny + y) * L.pitch + x0c);

            // a segment of solid cells moves no populations (solid cells are never read and both
            // population buffers hold their rest state); output steps still write its fields
            bool lane_solid = true;
#pragma unroll
            for (int k = 0; k < V; ++k) lane_solid &= (fl[k] & FLAG_SOLID) != 0;
            if (__all_sync(0xffffffffu, lane_solid)) {
                if constexpr (OUT) {
                    if (active) {
                        float one[V], zero[V];
#pragma unroll
                        for (int k = 0; k < V; ++k) { one[k] = 1.f; zero[k] = 0.f; }
                        vstore_plain<V>(L.rho + own, one);
                        vstore_plain<V>(L.ux + own, zero);
                        vstore_plain<V>(L.uy + own, zero);
                        vstore_plain<V>(L.uz + own, zero);
                        if constexpr (AVG) {
                            float a[V];
                            vload_plain<V>(a, L.avg + 3 * S + own);
#pragma unroll
                            for (int k = 0; k < V; ++k) a[k] += 1.f;
                            vstore_plain<V>(L.avg + 3 * S + own, a);
                        }
                    }
                }
                continue;
            }

            float f[V][Q];
            float R[V], UX[V], UY[V], UZ[V];
            const bool interior = y >= 1 && y <= L.ny - 2 && z >= 1 && z <= L.nz - 2;   // warp-uniform
            uint32_t rwm = 0;
            if (interior) pull_fast_all<V>(std::make_integer_sequence<int, Q>{}, f, fs + pc.own, po, lane);
            else rwm = pull_rows<V>(std::make_integer_sequence<int, Q>{}, f, L, pc);
            uint32_t flany = 0;
#pragma unroll
            for (int k = 0; k < V; ++k) flany |= fl[k];
            pull_fixups<V>(std::make_integer_sequence<int, Q>{}, f, L, pc, fl, flany & FLAG_WALLS & ~rwm);

            if (!__any_sync(0xffffffffu, flany & (FLAG_SOLID | FLAG_WALLFN | FLAG_FORCE))) {
#pragma unroll
                for (int k = 0; k < V; ++k)
                    collide(f[k], 0.f, 0.f, 0.f, L.tau0, L.csmag2, R[k], UX[k], UY[k], UZ[k]);
            } else {
#pragma unroll
                for (int k = 0; k < V; ++k) {
                    const uint32_t fk = fl[k];
                    const long long c = own + k;
                    if (fk & FLAG_SOLID) {
#pragma unroll
                        for (int i = 0; i < Q; ++i) f[k][i] = wgt(i);
                        R[k] = 1.f; UX[k] = 0.f; UY[k] = 0.f; UZ[k] = 0.f;
                    } else {
                        if (fk & FLAG_WALLFN) {
                            float U;
                            if constexpr (UCOL) U = (fk & FLAG_BEDWALL) ? L.colU[(long long)y * L.pitch + x0 + k] : 0.f;
                            else U = L.uref[c];
                            wall_function(f[k], fk & FLAG_WALLS, L.cfw[c], L.ux[c], L.uy[c], L.uz[c], L.rho[c], U);
                        }
                        float fx = 0.f, fy = 0.f, fz = 0.f;
                        if (fk & FLAG_FORCE) {
                            fx = L.Fx[c] * L.force_scale;
                            fy = L.Fy[c] * L.force_scale;
                            fz = L.Fz[c] * L.force_scale;
                        }
                        collide(f[k], fx, fy, fz, L.tau0, L.csmag2, R[k], UX[k], UY[k], UZ[k]);
                    }
                }
            }
            // inlet (x=0 from x=1) and outlet (x=nx-1 from x=nx-2), both inside this lane
            if (x0 == 0 && !(fl[0] & FLAG_SOLID) && !(fl[1] & FLAG_SOLID))
                nebb<true>(f[1], f[0], L.uin[y + (long long)L.ny * z], L.rho_out);
#pragma unroll
            for (int k = 1; k < V; ++k)
                if (x0 + k == L.nx - 1 && !(fl[k] & FLAG_SOLID) && !(fl[k - 1] & FLAG_SOLID))
                    nebb<false>(f[k - 1], f[k], 0.f, L.rho_out);

            if (active) {
#pragma unroll
                for (int i = 0; i < Q; ++i) {
                    float v[V];
#pragma unroll
                    for (int k = 0; k < V; ++k) v[k] = f[k][i];
                    vstore<V>(fd + (long long)i * S + own, v);
                }
                if constexpr (OUT) {
                    vstore_plain<V>(L.rho + own, R);
                    vstore_plain<V>(L.ux + own, UX);
                    vstore_plain<V>(L.uy + own, UY);
                    vstore_plain<V>(L.uz + own, UZ);
                    bool bad = false;
#pragma unroll
                    for (int k = 0; k < V; ++k) bad |= !(R[k] > 0.f && R[k] < 3.4e38f);
                    if (bad) atomicOr(L.status, 1);
                    if constexpr (AVG) {
                        float a[V], s[V];
#define WFS_ACC(M, EXPR)                                                   \
                        vload_plain<V>(a, L.avg + (long long)(M) * S + own); \
                        _Pragma("unroll") for (int k = 0; k < V; ++k) {     \
                            s[k] = a[k] + (EXPR);                           \
                        }                                                   \
                        vstore_plain<V>(L.avg + (long long)(M) * S + own, s);
                        WFS_ACC(0, UX[k])
                        WFS_ACC(1, UY[k])
                        WFS_ACC(2, UZ[k])
                        WFS_ACC(3, R[k])
                        WFS_ACC(4, sqrtf(UX[k] * UX[k] + UY[k] * UY[k] + UZ[k] * UZ[k]))
                        WFS_ACC(5, UX[k] * UX[k])
#undef WFS_ACC
                    }
                    if constexpr (UCOL) {
#pragma unroll
                        for (int k = 0; k < V; ++k)
                            if (!(fl[k] & FLAG_SOLID)) { csx[k] += UX[k]; csy[k] += UY[k]; ccn[k] += 1.f; }
                    }
                } else {
#pragma unroll
                    for (int k = 0; k < V; ++k)
                        if (fl[k] & FLAG_WALLFN) {
                            L.rho[own + k] = R[k]; L.ux[own + k] = UX[k];
                            L.uy[own + k] = UY[k]; L.uz[own + k] = UZ[k];
                        }
                }
            }
        }

        if constexpr (OUT && UCOL) {   // depth-mean speed of the item's columns (floodsim/reach3d.py:412-417)
            float* shx = sh;
            float* shy = sh + nwarps * SEG;
            float* shn = sh + 2 * nwarps * SEG;
#pragma unroll
            for (int k = 0; k < V; ++k) {
                shx[warp * SEG + lane * V + k] = csx[k];
                shy[warp * SEG + lane * V + k] = csy[k];
                shn[warp * SEG + lane * V + k] = ccn[k];
            }
            __syncthreads();
            for (int col = threadIdx.x; col < SEG; col += blockDim.x) {
                float sx = 0.f, sy = 0.f, n = 0.f;
                for (int w = 0; w < nwarps; ++w) { sx += shx[w * SEG + col]; sy += shy[w * SEG + col]; n += shn[w * SEG + col]; }
                const int x = seg * SEG + col;
                if (x < L.nx) L.colU[(long long)y * L.pitch + x] = sqrtf(sx * sx + sy * sy) / fmaxf(n, 1.f);
            }
            __syncthreads();
        }
    }
}

