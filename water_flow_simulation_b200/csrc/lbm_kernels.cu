// lbm_kernels.cu -- sm_100a kernels and C ABI of liblbm_b200.so (declared in include/lbm_b200.h).
//
// Hot path: k_fused, one launch per D3Q19 time step.
//   * Persistent CTAs walk work items (x segment, y row); a CTA owns every z of
//     its item, so z-column sums (the wall model's depth-mean speed) reduce
//     inside the CTA, deterministically, with no atomics.
//   * A warp covers 32*V consecutive x cells of one (y,z) row; each lane owns V
//     cells and moves them with V-wide (64/128-bit) loads and stores.  A pull
//     from x-1 / x+1 takes the neighbour lane's element by warp shuffle; only
//     the segment's first / last lane issues one extra scalar load.
//   * Walls are a per-cell 19-bit mask in a uint32 flag word (built once):
//     rows outside the domain (y walls, bed) bounce back warp-uniformly, solid
//     neighbours per cell with one extra load of the own-row opposite direction.
//   * Inlet/outlet non-equilibrium extrapolation runs in-thread on the
//     post-collision registers of x=1 / x=nx-2 (same lane), so the reference's
//     second kernel disappears.
//   * Macroscopic fields are written every step only where the next step's
//     wall function reads them; the last step of a chunk writes them everywhere,
//     refreshes the column-mean speed and adds the time averages.
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <utility>

#include "d3q19.cuh"
#include "../../include/lbm_b200.h"

using namespace wfs;

namespace {

thread_local char g_err[512] = "";

int fail(int code, const char* fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof g_err, fmt, ap);
    va_end(ap);
    return code;
}

int check_launch(const char* what)
{
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(LBM_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
    return LBM_OK;
}

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

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
struct PullCtx {
    const float* fs;
    long long S, rowc, own;   // own = rowc + x0c (load start, clamped into the row)
    int x0, x0c, y, z, lane;
};

template <int I, int V>
__device__ __forceinline__ void pull_load(float (&t)[Q][V], float (&hv)[Q], uint32_t& rwm, const lbm_lattice& L,
                                          const PullCtx& c)
{
    constexpr int CXI = cx(I), CYI = cy(I), CZI = cz(I);
    if constexpr (I == 0) {
        Vec<V>::load(t[0], c.fs + c.own);
    } else {
        int ys = c.y - CYI, zs = c.z - CZI, di = I;
        if (CZI == -1 && c.z == L.nz - 1) { zs = c.z; di = mirz(I); }   // rigid lid: mirrored population
        const bool rowwall = (ys < 0) || (ys >= L.ny) || (zs < 0);      // warp-uniform
        const float* row = rowwall ? c.fs + (long long)opp(I) * c.S + c.rowc
                                   : c.fs + (long long)di * c.S + ((long long)zs * L.ny + ys) * L.pitch;
        Vec<V>::load(t[I], row + c.x0c);
        if constexpr (CXI == 1) hv[I] = __ldg(row + (c.x0c > 0 ? c.x0c - 1 : 0));
        if constexpr (CXI == -1) hv[I] = __ldg(row + (c.x0c + V < L.pitch ? c.x0c + V : L.pitch - 1));
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

template <int I, int V>
__device__ __forceinline__ void pull_bounce(float (&f)[V][Q], const uint32_t (&fl)[V], uint32_t bb, const PullCtx& c)
{
    if constexpr (I > 0) {
        if (bb & (1u << I)) {
            float b[V];
            Vec<V>::load(b, c.fs + (long long)opp(I) * c.S + c.own);
#pragma unroll
            for (int k = 0; k < V; ++k)
                if (fl[k] & (1u << I)) f[k][I] = b[k];
        }
    }
}

template <int I, int V>
__device__ __forceinline__ void pull_edge(float (&f)[V][Q], const lbm_lattice& L, const PullCtx& c)
{
    constexpr int CXI = cx(I);
    if constexpr (CXI == 1) {
        if (c.x0 == 0) f[0][I] = __ldg(c.fs + (long long)I * c.S + c.rowc);
    } else if constexpr (CXI == -1) {
#pragma unroll
        for (int k = 0; k < V; ++k)
            if (c.x0 + k == L.nx - 1) f[k][I] = __ldg(c.fs + (long long)I * c.S + c.rowc + L.nx - 1);
    }
}

template <int V, int... Is>
__device__ __forceinline__ void pull_all(std::integer_sequence<int, Is...>, float (&f)[V][Q], const lbm_lattice& L,
                                         const PullCtx& c, const uint32_t (&fl)[V], uint32_t flany)
{
    float t[Q][V];
    float hv[Q];
    uint32_t rwm = 0;
    (pull_load<Is, V>(t, hv, rwm, L, c), ...);
    (pull_shift<Is, V>(f, t, hv, rwm, c.lane), ...);
    const uint32_t bb = flany & FLAG_WALLS & ~rwm;
    if (bb) { (pull_bounce<Is, V>(f, fl, bb, c), ...); }
    const bool edge = (c.x0 == 0) || (c.x0 <= L.nx - 1 && L.nx - 1 < c.x0 + V);
    if (edge) { (pull_edge<Is, V>(f, L, c), ...); }
}

template <int V, bool OUT, bool UCOL, bool AVG>
__global__ void __launch_bounds__(256) k_fused(const lbm_lattice L, const float* __restrict__ fs,
                                                float* __restrict__ fd)
{
    extern __shared__ float sh[];  // column partial sums, only for OUT && UCOL
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    constexpr int SEG = 32 * V;
    const int nseg = (L.pitch + SEG - 1) / SEG;
    const long long nitems = (long long)nseg * L.ny;
    const long long S = L.cells;

    for (long long item = blockIdx.x; item < nitems; item += gridDim.x) {
        const int seg = (int)(item % nseg), y = (int)(item / nseg);
        const int x0 = seg * SEG + lane * V;
        const bool active = x0 < L.pitch;
        const int x0c = active ? x0 : L.pitch - V;   // inactive lanes load (and discard) the row's last vector
        float csx[V], csy[V], ccn[V];
#pragma unroll
        for (int k = 0; k < V; ++k) { csx[k] = 0.f; csy[k] = 0.f; ccn[k] = 0.f; }

        for (int z = warp; z < L.nz; z += nwarps) {
            const long long rowc = ((long long)z * L.ny + y) * L.pitch;
            const long long own = rowc + x0;
            PullCtx pc{fs, S, rowc, rowc + x0c, x0, x0c, y, z, lane};
            uint32_t fl[V];
            Vec<V>::loadu(fl, L.flags + pc.own);
            if (!active) {
#pragma unroll
                for (int k = 0; k < V; ++k) fl[k] = FLAG_GHOST | FLAG_SOLID;
            }
            uint32_t flany = 0;
#pragma unroll
            for (int k = 0; k < V; ++k) flany |= fl[k];

            float f[V][Q];
            pull_all<V>(std::make_integer_sequence<int, Q>{}, f, L, pc, fl, flany);

            float R[V], UX[V], UY[V], UZ[V];
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

// Outlet/inlet rows on the pitched layout, for lattices whose x=nx-2 and x=nx-1 do not
// share a lane of k_fused (nx % V == 1).  side bit 0 = inlet, bit 1 = outlet.
__global__ void k_bc_rows(const lbm_lattice L, float* __restrict__ fd, int side)
{
    const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= (long long)L.ny * L.nz) return;
    const int y = (int)(j % L.ny), z = (int)(j / L.ny);
    const long long row = ((long long)z * L.ny + y) * L.pitch;
    for (int s = 0; s < 2; ++s) {
        if (!(side & (1 << s))) continue;
        const long long c0 = s == 0 ? row : row + L.nx - 1;
        const long long c1 = s == 0 ? row + 1 : row + L.nx - 2;
        if ((L.flags[c0] & FLAG_SOLID) || (L.flags[c1] & FLAG_SOLID)) continue;
        float g[Q], o[Q];
#pragma unroll
        for (int i = 0; i < Q; ++i) g[i] = fd[(long long)i * L.cells + c1];
        if (s == 0) nebb<true>(g, o, L.uin[j], L.rho_out);
        else nebb<false>(g, o, 0.f, L.rho_out);
#pragma unroll
        for (int i = 0; i < Q; ++i) fd[(long long)i * L.cells + c0] = o[i];
    }
}

// ---------------------------------------------------------------------------------------------
// Reference-layout kernels: the exact interface of floodsim/lbm3d.py's lbm_step / lbm_bc.
// ---------------------------------------------------------------------------------------------
template <int I>
__device__ __forceinline__ void ref_pull(float (&f)[Q], uint32_t& wm, const float* __restrict__ fs,
                                         const uint8_t* __restrict__ solid, long long N, long long c, int x, int y,
                                         int z, int nx, int ny, int nz)
{
    const int xs = x - cx(I), ys = y - cy(I);
    int zs = z - cz(I), ii = I;
    if (xs < 0 || xs >= nx) { f[I] = fs[(long long)I * N + c]; return; }
    if (zs >= nz) { zs = z; ii = mirz(I); }
    bool wall = (ys < 0 || ys >= ny || zs < 0);
    long long s = 0;
    if (!wall) { s = xs + (long long)nx * (ys + (long long)ny * zs); wall = solid[s] != 0; }
    if (wall) wm |= (1u << I);
    f[I] = wall ? fs[(long long)opp(I) * N + c] : fs[(long long)ii * N + s];
}
template <int... Is>
__device__ __forceinline__ void ref_pull_all(std::integer_sequence<int, Is...>, float (&f)[Q], uint32_t& wm,
                                             const float* __restrict__ fs, const uint8_t* __restrict__ solid,
                                             long long N, long long c, int x, int y, int z, int nx, int ny, int nz)
{
    (ref_pull<Is>(f, wm, fs, solid, N, c, x, y, z, nx, ny, nz), ...);
}

__global__ void __launch_bounds__(256) k_ref_step(const float* __restrict__ fs, float* __restrict__ fd,
        const uint8_t* __restrict__ solid, const float* __restrict__ Fx, const float* __restrict__ Fy,
        const float* __restrict__ Fz, float* __restrict__ rho, float* __restrict__ ux, float* __restrict__ uy,
        float* __restrict__ uz, const float* __restrict__ cfw, const float* __restrict__ uref,
        int nx, int ny, int nz, float tau0, float csmag2)
{
    const long long N = (long long)nx * ny * nz;
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= N) return;
    const int x = (int)(c % nx), y = (int)((c / nx) % ny), z = (int)(c / ((long long)nx * ny));
    if (solid[c]) { rho[c] = 1.f; ux[c] = 0.f; uy[c] = 0.f; uz[c] = 0.f; return; }
    float f[Q];
    uint32_t wm = 0;
    ref_pull_all(std::make_integer_sequence<int, Q>{}, f, wm, fs, solid, N, c, x, y, z, nx, ny, nz);
    const float cf = cfw[c];
    if (wm && cf > 0.f) wall_function(f, wm, cf, ux[c], uy[c], uz[c], rho[c], uref[c]);
    float r, u, v, w;
    collide(f, Fx[c], Fy[c], Fz[c], tau0, csmag2, r, u, v, w);
#pragma unroll
    for (int i = 0; i < Q; ++i) fd[(long long)i * N + c] = f[i];
    rho[c] = r; ux[c] = u; uy[c] = v; uz[c] = w;
}

__global__ void k_ref_bc(float* __restrict__ fd, const uint8_t* __restrict__ solid, const float* __restrict__ uin,
                         int nx, int ny, int nz, float rho_out)
{
    const long long N = (long long)nx * ny * nz;
    const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= (long long)ny * nz) return;
    const int y = (int)(j % ny), z = (int)(j / ny);
    const long long row = (long long)nx * (y + (long long)ny * z);
    for (int s = 0; s < 2; ++s) {
        const long long c0 = s == 0 ? row : row + nx - 1;
        const long long c1 = s == 0 ? row + 1 : row + nx - 2;
        if (solid[c0] || solid[c1]) continue;
        float g[Q], o[Q];
#pragma unroll
        for (int i = 0; i < Q; ++i) g[i] = fd[(long long)i * N + c1];
        if (s == 0) nebb<true>(g, o, uin[j], rho_out);
        else nebb<false>(g, o, 0.f, rho_out);
#pragma unroll
        for (int i = 0; i < Q; ++i) fd[(long long)i * N + c0] = o[i];
    }
}

// ---------------------------------------------------------------------------------------------
// Set-up kernels
// ---------------------------------------------------------------------------------------------
template <int I>
__device__ __forceinline__ void flag_dir(uint32_t& wm, const uint8_t* __restrict__ solid, const lbm_lattice& L,
                                         int x, int y, int z)
{
    const int xs = x - cx(I), ys = y - cy(I);
    int zs = z - cz(I);
    if (xs < 0 || xs >= L.nx) return;
    if (zs >= L.nz) zs = z;
    bool wall = (ys < 0 || ys >= L.ny || zs < 0);
    if (!wall) wall = solid[xs + (long long)L.pitch * (ys + (long long)L.ny * zs)] != 0;
    if (wall) wm |= (1u << I);
}
template <int... Is>
__device__ __forceinline__ void flag_all(std::integer_sequence<int, Is...>, uint32_t& wm,
                                         const uint8_t* __restrict__ solid, const lbm_lattice& L, int x, int y, int z)
{
    (flag_dir<Is>(wm, solid, L, x, y, z), ...);
}

__global__ void k_build_flags(const lbm_lattice L, const uint8_t* __restrict__ solid,
                              const uint8_t* __restrict__ bedwall, uint32_t* __restrict__ flags)
{
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= L.cells) return;
    const int x = (int)(c % L.pitch), y = (int)((c / L.pitch) % L.ny), z = (int)(c / ((long long)L.pitch * L.ny));
    if (x >= L.nx) { flags[c] = FLAG_GHOST | FLAG_SOLID; return; }
    if (solid[c]) { flags[c] = FLAG_SOLID; return; }
    uint32_t wm = 0;
    flag_all(std::make_integer_sequence<int, Q>{}, wm, solid, L, x, y, z);
    uint32_t fw = wm;
    if (L.Fx[c] != 0.f || L.Fy[c] != 0.f || L.Fz[c] != 0.f) fw |= FLAG_FORCE;
    if (wm && L.cfw[c] > 0.f) {
        int nwx = 0, nwy = 0, nwz = 0;
        for (int i = 1; i < Q; ++i)
            if (wm & (1u << i)) { nwx -= cx(i); nwy -= cy(i); nwz -= cz(i); }
        const int ax = ((wm >> 1) & 1) + ((wm >> 2) & 1), ay = ((wm >> 3) & 1) + ((wm >> 4) & 1),
                  az = ((wm >> 5) & 1) + ((wm >> 6) & 1);
        if (nwx * nwx + nwy * nwy + nwz * nwz > 0 && ax * ax + ay * ay + az * az > 0) fw |= FLAG_WALLFN;
    }
    if (bedwall && bedwall[c]) fw |= FLAG_BEDWALL;
    flags[c] = fw;
}

// f = feq(1, (u,0,0)) evaluated with the operation order and float64/float32 mix of the
// reference's NumPy start (floodsim/lbm3d.py:377-384): cu = (3*c_x)*u and the quadratic
// in float64, 1.5*u*u in float32, rounded once to float32 at the end.
__global__ void k_init_equilibrium(const lbm_lattice L, float* __restrict__ f)
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
        f[(long long)i * L.cells + c] = __double2float_rn(__dmul_rn(__dmul_rn(wgt64(i), 1.0), poly));
    }
}

// ---------------------------------------------------------------------------------------------
// Launch helpers
// ---------------------------------------------------------------------------------------------
int g_sm_count = 0;

int sm_count()
{
    if (g_sm_count == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&g_sm_count, cudaDevAttrMultiProcessorCount, dev);
        if (g_sm_count <= 0) g_sm_count = 1;
    }
    return g_sm_count;
}

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

int check_lattice(const lbm_lattice* L)
{
    if (!L) return fail(LBM_ERR_ARG, "lattice is NULL");
    if (L->nx < 4 || L->ny < 1 || L->nz < 1) return fail(LBM_ERR_ARG, "lattice %dx%dx%d too small (nx >= 4)", L->nx, L->ny, L->nz);
    if (L->pitch < L->nx || (L->pitch & 3)) return fail(LBM_ERR_ARG, "pitch %d must be >= nx and a multiple of 4", L->pitch);
    if (L->cells != (long long)L->pitch * L->ny * L->nz) return fail(LBM_ERR_ARG, "cells != pitch*ny*nz");
    if (!L->flags || !L->uin) return fail(LBM_ERR_ARG, "flags/uin pointer is NULL");
    return LBM_OK;
}

template <int V, bool OUT, bool UCOL, bool AVG>
int launch_fused_t(const lbm_lattice& L, const float* fs, float* fd, const lbm_tile& t, cudaStream_t st)
{
    auto kern = k_fused<V, OUT, UCOL, AVG>;
    const int threads = 32 * t.warps;
    const size_t smem = (OUT && UCOL) ? (size_t)3 * t.warps * 32 * V * sizeof(float) : 0;
    int per_sm = t.ctas_per_sm;
    if (per_sm <= 0) {
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem) != cudaSuccess || per_sm < 1)
            per_sm = 1;
    }
    const long long nseg = (L.pitch + 32 * V - 1) / (32 * V);
    const long long items = nseg * L.ny;
    long long grid = (long long)sm_count() * per_sm;
    if (grid > items) grid = items;
    kern<<<(unsigned)grid, threads, smem, st>>>(L, fs, fd);
    return check_launch("k_fused");
}

template <int V>
int launch_fused_v(const lbm_lattice& L, const float* fs, float* fd, uint32_t mode, const lbm_tile& t,
                   cudaStream_t st)
{
    const bool out = mode & LBM_STEP_OUTPUT, ucol = mode & LBM_STEP_UREF_COLUMN, avg = mode & LBM_STEP_ACCUMULATE;
    if (!out) return ucol ? launch_fused_t<V, false, true, false>(L, fs, fd, t, st)
                          : launch_fused_t<V, false, false, false>(L, fs, fd, t, st);
    if (ucol) return avg ? launch_fused_t<V, true, true, true>(L, fs, fd, t, st)
                         : launch_fused_t<V, true, true, false>(L, fs, fd, t, st);
    return avg ? launch_fused_t<V, true, false, true>(L, fs, fd, t, st)
               : launch_fused_t<V, true, false, false>(L, fs, fd, t, st);
}

}  // namespace

// =============================================================================================
// C ABI
// =============================================================================================
extern "C" {

const char* lbm_last_error(void) { return g_err; }

int lbm_abi_version(void) { return 100; }

int lbm_device_sm_count(void) { return sm_count(); }

int lbm_step(const float* fs, float* fd, const uint8_t* solid, const float* Fx, const float* Fy, const float* Fz,
             float* rho, float* ux, float* uy, float* uz, const float* cfw, const float* uref,
             int nx, int ny, int nz, float tau0, float csmag2, void* stream)
{
    g_err[0] = 0;
    if (!fs || !fd || !solid || !Fx || !Fy || !Fz || !rho || !ux || !uy || !uz || !cfw || !uref)
        return fail(LBM_ERR_ARG, "lbm_step: NULL array");
    if (nx < 3 || ny < 1 || nz < 1) return fail(LBM_ERR_ARG, "lbm_step: bad lattice %dx%dx%d", nx, ny, nz);
    if (fs == fd) return fail(LBM_ERR_ARG, "lbm_step: fs and fd must differ");
    const long long N = (long long)nx * ny * nz;
    const unsigned grid = (unsigned)((N + 255) / 256);
    k_ref_step<<<grid, 256, 0, as_stream(stream)>>>(fs, fd, solid, Fx, Fy, Fz, rho, ux, uy, uz, cfw, uref, nx, ny,
                                                     nz, tau0, csmag2);
    return check_launch("lbm_step");
}

int lbm_bc(float* fd, const uint8_t* solid, const float* uin, int nx, int ny, int nz, float rho_out, void* stream)
{
    g_err[0] = 0;
    if (!fd || !solid || !uin) return fail(LBM_ERR_ARG, "lbm_bc: NULL array");
    if (nx < 3 || ny < 1 || nz < 1) return fail(LBM_ERR_ARG, "lbm_bc: bad lattice %dx%dx%d", nx, ny, nz);
    const long long M = (long long)ny * nz;
    k_ref_bc<<<(unsigned)((M + 127) / 128), 128, 0, as_stream(stream)>>>(fd, solid, uin, nx, ny, nz, rho_out);
    return check_launch("lbm_bc");
}

int lbm_build_flags(const lbm_lattice* lat, const uint8_t* solid, const uint8_t* bedwall, uint32_t* flags,
                    void* stream)
{
    g_err[0] = 0;
    if (!lat) return fail(LBM_ERR_ARG, "lattice is NULL");
    lbm_lattice L = *lat;
    L.flags = flags;
    if (int e = check_lattice(&L)) return e;
    if (!solid || !L.Fx || !L.Fy || !L.Fz || !L.cfw) return fail(LBM_ERR_ARG, "lbm_build_flags: NULL array");
    k_build_flags<<<(unsigned)((L.cells + 255) / 256), 256, 0, as_stream(stream)>>>(L, solid, bedwall, flags);
    return check_launch("lbm_build_flags");
}

int lbm_init_equilibrium(const lbm_lattice* lat, float* f, void* stream)
{
    g_err[0] = 0;
    if (int e = check_lattice(lat)) return e;
    if (!f) return fail(LBM_ERR_ARG, "lbm_init_equilibrium: NULL f");
    k_init_equilibrium<<<(unsigned)((lat->cells + 255) / 256), 256, 0, as_stream(stream)>>>(*lat, f);
    return check_launch("lbm_init_equilibrium");
}

int lbm_fused_step(const lbm_lattice* lat, const float* fs, float* fd, uint32_t mode, const lbm_tile* tile,
                   void* stream)
{
    g_err[0] = 0;
    if (int e = check_lattice(lat)) return e;
    const lbm_lattice& L = *lat;
    if (!fs || !fd || fs == fd) return fail(LBM_ERR_ARG, "lbm_fused_step: fs/fd NULL or equal");
    if (!L.Fx || !L.Fy || !L.Fz || !L.cfw || !L.rho || !L.ux || !L.uy || !L.uz || !L.status)
        return fail(LBM_ERR_ARG, "lbm_fused_step: NULL field");
    if ((mode & LBM_STEP_UREF_COLUMN) ? !L.colU : !L.uref) return fail(LBM_ERR_ARG, "lbm_fused_step: NULL uref/colU");
    if ((mode & LBM_STEP_ACCUMULATE) && !L.avg) return fail(LBM_ERR_ARG, "lbm_fused_step: NULL avg");
    if (!aligned16(fs) || !aligned16(fd) || !aligned16(L.flags) || !aligned16(L.rho) || !aligned16(L.ux) ||
        !aligned16(L.uy) || !aligned16(L.uz) || (L.avg && !aligned16(L.avg)))
        return fail(LBM_ERR_ARG, "lbm_fused_step: arrays must be 16-byte aligned");
    lbm_tile t = tile ? *tile : lbm_tile{4, 4, 0};
    if ((t.cells_per_lane != 2 && t.cells_per_lane != 4) || t.warps < 1 || t.warps > 8 || t.ctas_per_sm < 0)
        return fail(LBM_ERR_ARG, "lbm_fused_step: bad tile (%d cells/lane, %d warps)", t.cells_per_lane, t.warps);
    cudaStream_t st = as_stream(stream);
    int e = t.cells_per_lane == 4 ? launch_fused_v<4>(L, fs, fd, mode, t, st) : launch_fused_v<2>(L, fs, fd, mode, t, st);
    if (e) return e;
    if (L.nx % t.cells_per_lane == 1) {   // x=nx-2 and x=nx-1 sit in different lanes: outlet in its own pass
        const long long M = (long long)L.ny * L.nz;
        k_bc_rows<<<(unsigned)((M + 127) / 128), 128, 0, st>>>(L, fd, 2);
        return check_launch("k_bc_rows");
    }
    return LBM_OK;
}

}  // extern "C"
