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
#include <cuda.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <cmath>
#include <mutex>
#include <type_traits>
#include <utility>

#include "d3q19.cuh"
#include "errors.cuh"
#include "../../include/lbm_b200.h"

using namespace wfs;

namespace wfs {
thread_local char g_err[512] = "";
}

namespace {

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

#include "fused_common.cuh"
#include "fused_reg.cuh"
#include "fused_tma.cuh"
#include "fused_async.cuh"
#include "fused_split.cuh"
#include "fused_half.cuh"
#include "readouts.cuh"

// Outlet/inlet rows on the pitched layout, for lattices whose x=nx-2 and x=nx-1 do not
// share a lane of k_fused (nx % V == 1).  side bit 0 = inlet, bit 1 = outlet.
template <typename T>
__device__ __forceinline__ void bc_row(const lbm_lattice& L, T* __restrict__ fd, int side, float scale, long long j)
{
    const float inv_scale = 1.0f / scale;
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
        for (int i = 0; i < Q; ++i) g[i] = ldpop(fd + (long long)i * L.cells + c1, i, inv_scale);
        if (s == 0) nebb<true>(g, o, L.uin[j], L.rho_out);
        else nebb<false>(g, o, 0.f, L.rho_out);
#pragma unroll
        for (int i = 0; i < Q; ++i) stpop(fd + (long long)i * L.cells + c0, i, o[i], scale);
    }
}

template <typename T>
__global__ void k_bc_rows(const lbm_lattice L, T* __restrict__ fd, int side, float scale)
{
    bc_row<T>(L, fd, side, scale, (long long)blockIdx.x * blockDim.x + threadIdx.x);
}

#include "fused_batch.cuh"

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

// Start state from a coarse flow prediction (the learned warm start): per fluid cell, the
// prediction (du, v, w, drho) of the cell's position, trilinear between coarse voxel centres
// (voxels of `factor`^3 cells), gives u = (uin(y, z) + du*su, v*su, w*su), rho = 1 + drho*srho,
// and the populations are the second-order equilibrium feq(rho, u) (the same formula as the
// collision's equilibrium part); the fields rho/ux/uy/uz are set to match.  Solid and padding
// cells get the rest state.  coarse: float (Z*Y*X, stride) channels-last.
__global__ void k_lift_coarse(const lbm_lattice L, const float* __restrict__ coarse, int stride, int X, int Y, int Z,
                              int factor, float su, float srho, float* __restrict__ f)
{
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= L.cells) return;
    const int x = (int)(c % L.pitch), y = (int)((c / L.pitch) % L.ny), z = (int)(c / ((long long)L.pitch * L.ny));
    float r = 1.f, ux = 0.f, uy = 0.f, uz = 0.f;
    if (x < L.nx && !(L.flags[c] & FLAG_SOLID)) {
        const float gx = fminf(fmaxf((x + 0.5f) / factor - 0.5f, 0.f), (float)(X - 1));
        const float gy = fminf(fmaxf((y + 0.5f) / factor - 0.5f, 0.f), (float)(Y - 1));
        const float gz = fminf(fmaxf((z + 0.5f) / factor - 0.5f, 0.f), (float)(Z - 1));
        const int x0 = min((int)gx, X - 1), y0 = min((int)gy, Y - 1), z0 = min((int)gz, Z - 1);
        const int x1 = min(x0 + 1, X - 1), y1 = min(y0 + 1, Y - 1), z1 = min(z0 + 1, Z - 1);
        const float tx = gx - x0, ty = gy - y0, tz = gz - z0;
        float p[4] = {0.f, 0.f, 0.f, 0.f};
        for (int k = 0; k < 8; ++k) {
            const int xi = (k & 1) ? x1 : x0, yi = (k & 2) ? y1 : y0, zi = (k & 4) ? z1 : z0;
            const float w = ((k & 1) ? tx : 1.f - tx) * ((k & 2) ? ty : 1.f - ty) * ((k & 4) ? tz : 1.f - tz);
            const float* q = coarse + ((long long)xi + (long long)X * (yi + (long long)Y * zi)) * stride;
            for (int j = 0; j < 4; ++j) p[j] += w * q[j];
        }
        ux = L.uin[y + (long long)L.ny * z] + p[0] * su;
        uy = p[1] * su;
        uz = p[2] * su;
        r = 1.f + p[3] * srho;
    }
    const float usq = ux * ux + uy * uy + uz * uz;
#pragma unroll
    for (int i = 0; i < Q; ++i) {
        const float cu = 3.f * ((float)cx(i) * ux + (float)cy(i) * uy + (float)cz(i) * uz);
        f[(long long)i * L.cells + c] = wgt(i) * r * (1.f + cu + 0.5f * cu * cu - 1.5f * usq);
    }
    L.rho[c] = r;
    L.ux[c] = ux;
    L.uy[c] = uy;
    L.uz[c] = uz;
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

// Context ids (cuCtxGetId; unique within the process, never reused) key the per-context
// resources of the library: the no-alloc scratch address and the overlap side stream.  The
// driver functions come from cudaGetDriverEntryPointByVersion, so the library does not link
// libcuda itself.
using PfnCtxGetCurrent = CUresult (*)(CUcontext*);
using PfnCtxGetId = CUresult (*)(CUcontext, unsigned long long*);
PfnCtxGetCurrent g_ctx_get_current = nullptr;
PfnCtxGetId g_ctx_get_id = nullptr;
bool g_ctx_fns_resolved = false;

// Unique id of the calling thread's current context; 0 if none is current (or the driver
// cannot say).
std::mutex g_ctx_fns_mu;
unsigned long long current_context_id()
{
    std::lock_guard<std::mutex> lock(g_ctx_fns_mu);
    if (!g_ctx_fns_resolved) {
        g_ctx_fns_resolved = true;
        void* fn = nullptr;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &fn, 12000, cudaEnableDefault, nullptr) == cudaSuccess)
            g_ctx_get_current = reinterpret_cast<PfnCtxGetCurrent>(fn);
        fn = nullptr;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetId", &fn, 12000, cudaEnableDefault, nullptr) == cudaSuccess)
            g_ctx_get_id = reinterpret_cast<PfnCtxGetId>(fn);
    }
    if (!g_ctx_get_current || !g_ctx_get_id) return 0;
    CUcontext ctx = nullptr;
    unsigned long long id = 0;
    if (g_ctx_get_current(&ctx) != CUDA_SUCCESS || !ctx) return 0;
    if (g_ctx_get_id(ctx, &id) != CUDA_SUCCESS) return 0;
    return id;
}


// ---------------------------------------------------------------------------------------------
// LBM_STEP_OVERLAP: the edge and special kernels of a split step run on a side stream of the
// library, forked from the caller's stream before the plain kernel and joined back after, so
// that their latency-bound work shares the SMs with the bandwidth-bound plain kernel.  One side
// stream and one fork/join event pair per CUDA context, created on the first overlapped step in
// that context (make it before any stream capture); a mutex holds the pair from the fork to the
// join, so host threads that step concurrently take turns through that short window.
// ---------------------------------------------------------------------------------------------
struct SideStream {
    unsigned long long key;
    cudaStream_t s;
    cudaEvent_t fork, join;
};
constexpr int kSideStreams = 16;
std::mutex g_side_mu;
SideStream g_side[kSideStreams] = {};
int g_side_next = 0;

// Forks: `side` becomes the context's side stream, ordered after all work enqueued on st so far.
// On success the lock is held until overlap_join.
int overlap_fork(cudaStream_t st, cudaStream_t* side, std::unique_lock<std::mutex>& lk)
{
    lk = std::unique_lock<std::mutex>(g_side_mu);
    unsigned long long key = current_context_id();
    if (key == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        key = (1ULL << 63) | (unsigned long long)dev;
    }
    SideStream* ss = nullptr;
    for (SideStream& e : g_side)
        if (e.s && e.key == key) ss = &e;
    if (!ss) {
        SideStream n{key, nullptr, nullptr, nullptr};
        if (cudaStreamCreateWithFlags(&n.s, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&n.fork, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&n.join, cudaEventDisableTiming) != cudaSuccess) {
            lk.unlock();
            return fail(LBM_ERR_CUDA, "LBM_STEP_OVERLAP: side stream or events: %s",
                        cudaGetErrorString(cudaGetLastError()));
        }
        ss = &g_side[g_side_next];        // an entry of a context that is gone is simply replaced
        g_side_next = (g_side_next + 1) % kSideStreams;
        *ss = n;
    }
    cudaError_t e = cudaEventRecord(ss->fork, st);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(ss->s, ss->fork, 0);
    if (e != cudaSuccess) {
        lk.unlock();
        return fail(LBM_ERR_CUDA, "LBM_STEP_OVERLAP: fork: %s", cudaGetErrorString(e));
    }
    *side = ss->s;
    return LBM_OK;
}

// Joins: st waits for everything enqueued on the side stream; releases the lock.
int overlap_join(cudaStream_t st, cudaStream_t side, std::unique_lock<std::mutex>& lk)
{
    SideStream* ss = nullptr;
    for (SideStream& e : g_side)
        if (e.s == side) ss = &e;
    cudaError_t e = ss ? cudaEventRecord(ss->join, side) : cudaErrorInvalidResourceHandle;
    if (e == cudaSuccess) e = cudaStreamWaitEvent(st, ss->join, 0);
    lk.unlock();
    if (e != cudaSuccess) return fail(LBM_ERR_CUDA, "LBM_STEP_OVERLAP: join: %s", cudaGetErrorString(e));
    return LBM_OK;
}

int check_lattice(const lbm_lattice* L)
{
    if (!L) return fail(LBM_ERR_ARG, "lattice is NULL");
    if (L->nx < 4 || L->ny < 1 || L->nz < 1) return fail(LBM_ERR_ARG, "lattice %dx%dx%d too small (nx >= 4)", L->nx, L->ny, L->nz);
    if (L->pitch < L->nx || (L->pitch & 3)) return fail(LBM_ERR_ARG, "pitch %d must be >= nx and a multiple of 4", L->pitch);
    if (L->cells != (long long)L->pitch * L->ny * L->nz) return fail(LBM_ERR_ARG, "cells != pitch*ny*nz");
    if (!L->flags || !L->uin) return fail(LBM_ERR_ARG, "flags/uin pointer is NULL");
    if (L->sponge_cols < 0 || L->sponge_cols > L->nx - 2)
        return fail(LBM_ERR_ARG, "sponge_cols %d outside [0, nx-2]", L->sponge_cols);
    if (L->sponge_cols > 0 && !(L->sponge_tau >= L->tau0 && L->sponge_tau < 2.0f))
        return fail(LBM_ERR_ARG, "sponge_tau %g must be >= tau0 and < 2", (double)L->sponge_tau);
    return LBM_OK;
}

PullOffsets pull_offsets(const lbm_lattice& L)
{
    PullOffsets po;
    for (int i = 0; i < Q; ++i) {
        po.d[i] = (long long)i * L.cells - (long long)cz(i) * L.ny * L.pitch - (long long)cy(i) * L.pitch;
        po.lid[i] = cz(i) == -1 ? (long long)mirz(i) * L.cells - (long long)cy(i) * L.pitch : po.d[i];
    }
    return po;
}

template <typename K>
int occupancy(K kern, int threads, size_t smem, int requested)
{
    if (requested > 0) return requested;
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem) != cudaSuccess || per_sm < 1)
        per_sm = 1;
    return per_sm;
}

template <int V, bool OUT, bool UCOL, bool AVG>
int launch_reg_t(const lbm_lattice& L, const float* fs, float* fd, const lbm_tile& t, cudaStream_t st)
{
    auto kern = k_fused<V, OUT, UCOL, AVG>;
    const int threads = 32 * t.warps;
    const size_t smem = (OUT && UCOL) ? (size_t)3 * t.warps * 32 * V * sizeof(float) : 0;
    const int per_sm = occupancy(kern, threads, smem, t.ctas_per_sm);
    const long long nseg = (L.pitch + 32 * V - 1) / (32 * V);
    const long long items = nseg * L.ny;
    long long grid = (long long)sm_count() * per_sm;
    if (grid > items) grid = items;
    kern<<<(unsigned)grid, threads, smem, st>>>(L, pull_offsets(L), fs, fd);
    return check_launch("k_fused");
}

template <int C, bool OUT, bool UCOL, bool AVG>
int launch_tma_t(const lbm_lattice& L, const float* fs, float* fd, const lbm_tile& t, int outlet_fused,
                 cudaStream_t st)
{
    auto kern = k_fused_tma<C, OUT, UCOL, AVG>;
    const int threads = 32 * (C + 1);
    const TmaLayout lay(32 * C, t.stages);
    static size_t configured = 0;   // dynamic shared memory already granted to this instantiation
    if (lay.bytes > configured) {
        if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)lay.bytes) != cudaSuccess)
            return fail(LBM_ERR_ARG, "k_fused_tma: %zu bytes of shared memory not available", lay.bytes);
        configured = lay.bytes;
    }
    const int per_sm = occupancy(kern, threads, lay.bytes, t.ctas_per_sm);
    const long long nseg = (L.pitch + 32 * C - 1) / (32 * C);
    const long long items = nseg * L.ny;
    long long grid = (long long)sm_count() * per_sm;
    if (grid > items) grid = items;
    kern<<<(unsigned)grid, threads, lay.bytes, st>>>(L, fs, fd, t.stages, outlet_fused);
    return check_launch("k_fused_tma");
}

template <int C>
int launch_tma_c(const lbm_lattice& L, const float* fs, float* fd, uint32_t mode, const lbm_tile& t, int ofused,
                 cudaStream_t st)
{
    const bool out = mode & LBM_STEP_OUTPUT, ucol = mode & LBM_STEP_UREF_COLUMN, avg = mode & LBM_STEP_ACCUMULATE;
    if (!out) return ucol ? launch_tma_t<C, false, true, false>(L, fs, fd, t, ofused, st)
                          : launch_tma_t<C, false, false, false>(L, fs, fd, t, ofused, st);
    if (ucol) return avg ? launch_tma_t<C, true, true, true>(L, fs, fd, t, ofused, st)
                         : launch_tma_t<C, true, true, false>(L, fs, fd, t, ofused, st);
    return avg ? launch_tma_t<C, true, false, true>(L, fs, fd, t, ofused, st)
               : launch_tma_t<C, true, false, false>(L, fs, fd, t, ofused, st);
}

template <int V>
int launch_reg_v(const lbm_lattice& L, const float* fs, float* fd, uint32_t mode, const lbm_tile& t, cudaStream_t st)
{
    const bool out = mode & LBM_STEP_OUTPUT, ucol = mode & LBM_STEP_UREF_COLUMN, avg = mode & LBM_STEP_ACCUMULATE;
    if (!out) return ucol ? launch_reg_t<V, false, true, false>(L, fs, fd, t, st)
                          : launch_reg_t<V, false, false, false>(L, fs, fd, t, st);
    if (ucol) return avg ? launch_reg_t<V, true, true, true>(L, fs, fd, t, st)
                         : launch_reg_t<V, true, true, false>(L, fs, fd, t, st);
    return avg ? launch_reg_t<V, true, false, true>(L, fs, fd, t, st)
               : launch_reg_t<V, true, false, false>(L, fs, fd, t, st);
}

template <bool OUT, bool UCOL, bool AVG, int D>
int launch_async_t(const lbm_lattice& L, const float* fs, float* fd, const lbm_tile& t, int outlet_fused,
                   cudaStream_t st)
{
    auto kern = k_fused_async<OUT, UCOL, AVG, D>;
    const int threads = 32 * t.warps;
    const AsyncLayout lay(t.warps, D);
    static size_t configured = 0;
    if (lay.bytes > configured) {
        if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)lay.bytes) != cudaSuccess)
            return fail(LBM_ERR_ARG, "k_fused_async: %zu bytes of shared memory not available", lay.bytes);
        configured = lay.bytes;
    }
    const PullOffsets po = pull_offsets(L);
    const int per_sm = occupancy(kern, threads, lay.bytes, t.ctas_per_sm);
    const long long nseg = (L.pitch + kSegA - 1) / kSegA;
    const long long warps_needed = nseg * L.ny;
    long long grid = (long long)sm_count() * per_sm;
    const long long grid_max = (warps_needed + t.warps - 1) / t.warps;
    if (grid > grid_max) grid = grid_max;
    kern<<<(unsigned)grid, threads, lay.bytes, st>>>(L, po, fs, fd, outlet_fused);
    return check_launch("k_fused_async");
}

template <int D>
int launch_async_d(const lbm_lattice& L, const float* fs, float* fd, uint32_t mode, const lbm_tile& t, int ofused,
                   cudaStream_t st)
{
    const bool out = mode & LBM_STEP_OUTPUT, ucol = mode & LBM_STEP_UREF_COLUMN, avg = mode & LBM_STEP_ACCUMULATE;
    if (!out) return ucol ? launch_async_t<false, true, false, D>(L, fs, fd, t, ofused, st)
                          : launch_async_t<false, false, false, D>(L, fs, fd, t, ofused, st);
    if (ucol) return avg ? launch_async_t<true, true, true, D>(L, fs, fd, t, ofused, st)
                         : launch_async_t<true, true, false, D>(L, fs, fd, t, ofused, st);
    return avg ? launch_async_t<true, false, true, D>(L, fs, fd, t, ofused, st)
               : launch_async_t<true, false, false, D>(L, fs, fd, t, ofused, st);
}

int launch_async(const lbm_lattice& L, const float* fs, float* fd, uint32_t mode, const lbm_tile& t, int ofused,
                 cudaStream_t st)
{
    switch (t.stages) {
    case 2: return launch_async_d<2>(L, fs, fd, mode, t, ofused, st);
    case 3: return launch_async_d<3>(L, fs, fd, mode, t, ofused, st);
    case 4: return launch_async_d<4>(L, fs, fd, mode, t, ofused, st);
    default: return fail(LBM_ERR_ARG, "lbm_fused_step: async pipeline takes 2, 3 or 4 stages");
    }
}

template <int V, bool PLAIN, bool OUT, bool UCOL, bool AVG>
int launch_rows_t(const lbm_lattice& L, const uint32_t* list, int n, const float* fs, float* fd, const lbm_tile& t,
                  cudaStream_t st)
{
    if (n <= 0) return LBM_OK;
    auto kern = k_rows<V, PLAIN, OUT, UCOL, AVG>;
    const int threads = 32 * t.warps;
    const int per_sm = occupancy(kern, threads, 0, t.ctas_per_sm);
    long long grid = (long long)sm_count() * per_sm;
    const long long need = ((long long)n + t.warps - 1) / t.warps;
    if (grid > need) grid = need;
    kern<<<(unsigned)grid, threads, 0, st>>>(L, pull_offsets(L), list, n, fs, fd);
    return check_launch(PLAIN ? "k_rows<plain>" : "k_rows<special>");
}

template <int V, int PASSES, bool OUT, bool AVG, typename T>
int launch_edge(const lbm_lattice& L, const T* fs, T* fd, float scale, const lbm_tile& t, cudaStream_t st)
{
    if (L.n_edge <= 0) return LBM_OK;
    auto kern = k_rows_edge<V, PASSES, OUT, AVG, T>;
    const int threads = 32 * t.warps;
    const int per_sm = occupancy(kern, threads, 0, t.ctas_per_sm);
    long long grid = (long long)sm_count() * per_sm;
    const long long need = ((long long)L.n_edge + t.warps - 1) / t.warps;
    if (grid > need) grid = need;
    kern<<<(unsigned)grid, threads, 0, st>>>(L, pull_offsets(L), L.rows_edge, L.n_edge, fs, fd, scale);
    return check_launch("k_rows_edge");
}

template <int V, bool OUT, bool UCOL, bool AVG>
int launch_general_f(const lbm_lattice& L, const float* fs, float* fd, const lbm_tile& t, cudaStream_t st)
{
    if (L.n_special <= 0) return LBM_OK;
    auto kern = k_general<V, 1, OUT, UCOL, AVG, float>;
    const int threads = 32 * t.warps;
    const int per_sm = occupancy(kern, threads, 0, t.ctas_per_sm);
    long long grid = (long long)sm_count() * per_sm;
    const long long need = ((long long)L.n_special + t.warps - 1) / t.warps;
    if (grid > need) grid = need;
    kern<<<(unsigned)grid, threads, 0, st>>>(L, pull_offsets(L), L.rows_special, L.n_special, fs, fd, 1.f);
    return check_launch("k_general");
}

template <int V, bool OUT, bool UCOL, bool AVG>
int launch_split_t(const lbm_lattice& L, const float* fs, float* fd, const lbm_tile& t, uint32_t mode,
                   cudaStream_t st)
{
    // LBM_STEP_OVERLAP: edge and special kernels on the side stream beside the plain kernel, whose
    // CTAs per SM tile.ctas_per_sm then limits alone
    const bool overlap = (mode & LBM_STEP_OVERLAP) && !(mode & (LBM_STEP_SKIP_PLAIN | LBM_STEP_SKIP_SPECIAL));
    cudaStream_t sst = st;
    lbm_tile ts = t;
    std::unique_lock<std::mutex> lk;
    if (overlap) {
        if (int e = overlap_fork(st, &sst, lk)) return e;
        ts.ctas_per_sm = 0;
    }
    int e = LBM_OK;
    if (!(mode & LBM_STEP_SKIP_PLAIN)) e = launch_rows_t<V, true, OUT, false, AVG>(L, L.rows_plain, L.n_plain, fs, fd, t, st);
    if (!e && !(mode & LBM_STEP_SKIP_SPECIAL)) {
        e = launch_edge<V, 1, OUT, AVG, float>(L, fs, fd, 1.f, ts, sst);
        if (!e) e = launch_general_f<V, OUT, UCOL, AVG>(L, fs, fd, ts, sst);
    }
    if (overlap) {
        const int ej = overlap_join(st, sst, lk);
        if (!e) e = ej;
    }
    if (e || (mode & LBM_STEP_SKIP_SPECIAL)) return e;
    if (OUT && L.n_solid > 0) {
        const int threads = 128;
        long long grid = ((long long)L.n_solid * 32 + threads - 1) / threads;
        if (grid > 4LL * sm_count()) grid = 4LL * sm_count();
        k_solid_out<V, AVG><<<(unsigned)grid, threads, 0, st>>>(L, L.rows_solid, L.n_solid);
        if (int e = check_launch("k_solid_out")) return e;
    }
    if (OUT && UCOL) {
        const long long n = (long long)L.ny * L.pitch;
        k_column_mean<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(L);
        if (int e = check_launch("k_column_mean")) return e;
    }
    return LBM_OK;
}

template <int V>
int launch_split_v(const lbm_lattice& L, const float* fs, float* fd, uint32_t mode, const lbm_tile& t, cudaStream_t st)
{
    const bool out = mode & LBM_STEP_OUTPUT, ucol = mode & LBM_STEP_UREF_COLUMN, avg = mode & LBM_STEP_ACCUMULATE;
    if (!out) return ucol ? launch_split_t<V, false, true, false>(L, fs, fd, t, mode, st)
                          : launch_split_t<V, false, false, false>(L, fs, fd, t, mode, st);
    if (ucol) return avg ? launch_split_t<V, true, true, true>(L, fs, fd, t, mode, st)
                         : launch_split_t<V, true, true, false>(L, fs, fd, t, mode, st);
    return avg ? launch_split_t<V, true, false, true>(L, fs, fd, t, mode, st)
               : launch_split_t<V, true, false, false>(L, fs, fd, t, mode, st);
}

int launch_tma(const lbm_lattice& L, const float* fs, float* fd, uint32_t mode, const lbm_tile& t, int ofused,
               cudaStream_t st)
{
    switch (t.warps) {
    case 2: return launch_tma_c<2>(L, fs, fd, mode, t, ofused, st);
    case 4: return launch_tma_c<4>(L, fs, fd, mode, t, ofused, st);
    case 8: return launch_tma_c<8>(L, fs, fd, mode, t, ofused, st);
    default: return fail(LBM_ERR_ARG, "lbm_fused_step: TMA pipeline takes 2, 4 or 8 consumer warps");
    }
}

// ---------------------------------------------------------------------------------------------
// 16-bit storage launchers (fused_half.cuh)
// ---------------------------------------------------------------------------------------------
// warps_needed: warps that have work (default: one list entry per warp)
template <typename K>
int launch_list(K kern, const char* name, const lbm_lattice& L, const uint32_t* list, int n, const __half* hs,
                __half* hd, float scale, const lbm_tile& t, cudaStream_t st, long long warps_needed = -1)
{
    if (n <= 0) return LBM_OK;
    const int threads = 32 * t.warps;
    const int per_sm = occupancy(kern, threads, 0, t.ctas_per_sm);
    long long grid = (long long)sm_count() * per_sm;
    if (warps_needed < 0) warps_needed = n;
    const long long need = (warps_needed + t.warps - 1) / t.warps;
    if (grid > need) grid = need;
    kern<<<(unsigned)grid, threads, 0, st>>>(L, pull_offsets(L), list, n, hs, hd, scale);
    return check_launch(name);
}

// CPL = cells_per_lane of the lists (segments of 32*CPL cells); the plain kernel runs 8 cells
// per lane in groups of 4*CPL lanes, the edge and general paths VG cells per lane in PASSES passes.
template <int CPL, bool OUT, bool UCOL, bool AVG>
int launch_split_h_t(const lbm_lattice& L, const __half* hs, __half* hd, float scale, const lbm_tile& t,
                     uint32_t mode, cudaStream_t st)
{
    constexpr int VG = CPL == 2 ? 2 : 4, PASSES = CPL / VG;
    // LBM_STEP_OVERLAP: edge and special kernels on the side stream beside the plain kernel, whose
    // CTAs per SM tile.ctas_per_sm then limits alone
    const bool overlap = (mode & LBM_STEP_OVERLAP) && !(mode & (LBM_STEP_SKIP_PLAIN | LBM_STEP_SKIP_SPECIAL));
    cudaStream_t sst = st;
    lbm_tile ts = t;
    std::unique_lock<std::mutex> lk;
    if (overlap) {
        if (int e = overlap_fork(st, &sst, lk)) return e;
        ts.ctas_per_sm = 0;
    }
    int err = LBM_OK;
    if (!(mode & LBM_STEP_SKIP_PLAIN) && L.n_plain > 0) {
        // plain kernel: VP cells per lane (tile.stages 4 or 8; 0 = 8), 32*CPL/VP lanes per segment,
        // so a warp takes VP/CPL list entries per pass
        int e = LBM_OK;
        bool done = false;
        if constexpr (CPL <= 4) {
            if (t.stages == 4) {
                const long long warps = (L.n_plain + 4 / CPL - 1) / (4 / CPL);
                e = launch_list(k_rows_h_plain<4, 8 * CPL, OUT, AVG>, "k_rows_h_plain", L, L.rows_plain, L.n_plain,
                                hs, hd, scale, t, st, warps);
                done = true;
            }
        }
        if (!done) {
            const long long warps = (L.n_plain + 8 / CPL - 1) / (8 / CPL);
            e = launch_list(k_rows_h_plain<8, 4 * CPL, OUT, AVG>, "k_rows_h_plain", L, L.rows_plain, L.n_plain, hs,
                            hd, scale, t, st, warps);
        }
        err = e;
    }
    if (!err && !(mode & LBM_STEP_SKIP_SPECIAL)) {
        err = launch_edge<VG, PASSES, OUT, AVG, __half>(L, hs, hd, scale, ts, sst);
        if (!err)
            err = launch_list(k_general<VG, PASSES, OUT, UCOL, AVG, __half>, "k_general", L, L.rows_special,
                              L.n_special, hs, hd, scale, ts, sst);
    }
    if (overlap) {
        const int ej = overlap_join(st, sst, lk);
        if (!err) err = ej;
    }
    if (err || (mode & LBM_STEP_SKIP_SPECIAL)) return err;
    if (OUT && L.n_solid > 0) {
        const int threads = 128;
        long long grid = ((long long)L.n_solid * 32 + threads - 1) / threads;
        if (grid > 4LL * sm_count()) grid = 4LL * sm_count();
        k_solid_out<CPL, AVG><<<(unsigned)grid, threads, 0, st>>>(L, L.rows_solid, L.n_solid);
        if (int e = check_launch("k_solid_out")) return e;
    }
    if (OUT && UCOL) {
        const long long n = (long long)L.ny * L.pitch;
        k_column_mean<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(L);
        if (int e = check_launch("k_column_mean")) return e;
    }
    return LBM_OK;
}

template <int CPL>
int launch_split_h_c(const lbm_lattice& L, const __half* hs, __half* hd, float scale, uint32_t mode,
                     const lbm_tile& t, cudaStream_t st)
{
    const bool out = mode & LBM_STEP_OUTPUT, ucol = mode & LBM_STEP_UREF_COLUMN, avg = mode & LBM_STEP_ACCUMULATE;
    if (!out) return ucol ? launch_split_h_t<CPL, false, true, false>(L, hs, hd, scale, t, mode, st)
                          : launch_split_h_t<CPL, false, false, false>(L, hs, hd, scale, t, mode, st);
    if (ucol) return avg ? launch_split_h_t<CPL, true, true, true>(L, hs, hd, scale, t, mode, st)
                         : launch_split_h_t<CPL, true, true, false>(L, hs, hd, scale, t, mode, st);
    return avg ? launch_split_h_t<CPL, true, false, true>(L, hs, hd, scale, t, mode, st)
               : launch_split_h_t<CPL, true, false, false>(L, hs, hd, scale, t, mode, st);
}

int launch_split_h(const lbm_lattice& L, const __half* hs, __half* hd, float scale, uint32_t mode, const lbm_tile& t,
                   cudaStream_t st)
{
    switch (t.cells_per_lane) {
    case 2: return launch_split_h_c<2>(L, hs, hd, scale, mode, t, st);
    case 4: return launch_split_h_c<4>(L, hs, hd, scale, mode, t, st);
    default: return launch_split_h_c<8>(L, hs, hd, scale, mode, t, st);
    }
}

// A 16-bit storage scale must be a power of two in [2^-8, 2^24] (so that scaling is exact).
int check_scale(float scale, const char* who)
{
    int ex = 0;
    const float m = std::frexp(scale, &ex);
    if (!(scale > 0.f) || m != 0.5f || ex < -7 || ex > 25)
        return fail(LBM_ERR_ARG, "%s: storage scale %g must be a power of two in [2^-8, 2^24]", who, (double)scale);
    return LBM_OK;
}

// ---------------------------------------------------------------------------------------------
// Batch launchers (fused_batch.cuh)
// ---------------------------------------------------------------------------------------------
template <typename K, typename... Args>
int launch_batch_list(K kern, const char* name, int n, long long warps_needed, const lbm_tile& t, cudaStream_t st,
                      Args... args)
{
    if (n <= 0) return LBM_OK;
    const int threads = 32 * t.warps;
    const int per_sm = occupancy(kern, threads, 0, t.ctas_per_sm);
    long long grid = (long long)sm_count() * per_sm;
    const long long need = (warps_needed + t.warps - 1) / t.warps;
    if (grid > need) grid = need;
    kern<<<(unsigned)grid, threads, 0, st>>>(args...);
    return check_launch(name);
}

template <bool OUT, bool UCOL, bool AVG>
int launch_batch_t(const lbm_batch& b, const BatchDesc& B, int parity, uint32_t mode, const lbm_tile& t,
                   cudaStream_t st)
{
    if (!(mode & LBM_STEP_SKIP_PLAIN)) {
        int e;
        if (t.stages == 4)
            e = launch_batch_list(k_batch_plain<4, 16, OUT, AVG>, "k_batch_plain", b.n_plain, (b.n_plain + 1) / 2, t,
                                  st, B, parity, b.rows_plain, b.n_plain);
        else
            e = launch_batch_list(k_batch_plain<8, 8, OUT, AVG>, "k_batch_plain", b.n_plain, (b.n_plain + 3) / 4, t,
                                  st, B, parity, b.rows_plain, b.n_plain);
        if (e) return e;
    }
    if (mode & LBM_STEP_SKIP_SPECIAL) return LBM_OK;
    if (int e = launch_batch_list(k_batch_edge<OUT, AVG>, "k_batch_edge", b.n_edge, b.n_edge, t, st, B, parity,
                                  b.rows_edge, b.n_edge))
        return e;
    if (int e = launch_batch_list(k_batch_general<OUT, UCOL, AVG>, "k_batch_general", b.n_special, b.n_special, t, st,
                                  B, parity, b.rows_special, b.n_special))
        return e;
    if (OUT && b.n_solid > 0) {
        long long grid = ((long long)b.n_solid * 32 + 127) / 128;
        if (grid > 4LL * sm_count()) grid = 4LL * sm_count();
        k_batch_solid_out<AVG><<<(unsigned)grid, 128, 0, st>>>(B, b.rows_solid, b.n_solid);
        if (int e = check_launch("k_batch_solid_out")) return e;
    }
    if (OUT && UCOL) {
        k_batch_column_mean<<<dim3((unsigned)((b.max_columns + 255) / 256), (unsigned)b.count), 256, 0, st>>>(B);
        if (int e = check_launch("k_batch_column_mean")) return e;
    }
    k_batch_bc_rows<<<dim3((unsigned)((b.max_rows + 127) / 128), (unsigned)b.count), 128, 0, st>>>(B, parity);
    return check_launch("k_batch_bc_rows");
}

// Row chunks of the profile reduction (pass 1 runs nx x chunks threads).
int profile_chunks(const lbm_lattice& L) { return L.ny * L.nz < 256 ? L.ny * L.nz : 256; }

// ---------------------------------------------------------------------------------------------
// Static scratch of lbm_build_worklists_noalloc.
//
// For callers that may not allocate device memory at run time: hosts whose own allocator
// reserves the GPU up front and allows no other allocation, and time loops that cannot take
// the device-wide synchronisation of cudaMalloc/cudaFree in mid-run.  The class bytes that
// k_classify writes and k_compact reads live in this file-scope array instead of a caller
// buffer.  Every GPU that loads the library holds it (4 MiB) until exit, and all calls on a
// device share it, so calls whose kernels overlap on the GPU race.  k_classify writes every
// byte that k_compact then reads, so nothing needs clearing between calls.
// ---------------------------------------------------------------------------------------------
constexpr long long kNoAllocMaxSegments = 4LL << 20;  // one class byte per row segment
static __device__ __align__(256) uint8_t g_noalloc_classes[kNoAllocMaxSegments];

// The array's address belongs to a CUDA context, not to a device: the library's module is
// loaded once per context, so a host that runs the call in a context of its own, or one
// that calls after cudaDeviceReset, sees another address than the primary context had.
// Addresses are therefore cached per context, under the context's unique id (cuCtxGetId;
// ids are never reused within a process, so an entry of a destroyed context is never hit).
constexpr int kNoAllocCacheSize = 64;
struct NoAllocEntry {
    unsigned long long ctx_id;
    uint8_t* ptr;
};
std::mutex g_noalloc_mu;
NoAllocEntry g_noalloc_cache[kNoAllocCacheSize] = {};
int g_noalloc_next = 0;

// Device address of g_noalloc_classes in the current context.  The first call in a context
// looks it up (cudaGetSymbolAddress, which may load the module there and, with no context
// current, makes the device's primary context current); later calls in that context reuse
// the cached address.  Without a context id (an old driver) every call looks it up.
int noalloc_scratch(uint8_t** out)
{
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    unsigned long long id = current_context_id();
    if (id != 0)
        for (const NoAllocEntry& en : g_noalloc_cache)
            if (en.ctx_id == id) {
                *out = en.ptr;
                return LBM_OK;
            }
    uint8_t* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress((void**)&p, g_noalloc_classes);
    if (e != cudaSuccess || !p) {
        int dev = -1;
        cudaGetDevice(&dev);
        return fail(LBM_ERR_CUDA, "lbm_build_worklists_noalloc: cudaGetSymbolAddress on device %d: %s", dev,
                    cudaGetErrorString(e));
    }
    id = current_context_id();
    if (id != 0) {
        g_noalloc_cache[g_noalloc_next] = NoAllocEntry{id, p};
        g_noalloc_next = (g_noalloc_next + 1) % kNoAllocCacheSize;
    }
    *out = p;
    return LBM_OK;
}

template <typename T>
int body_forces_t(const lbm_lattice* lat, const T* f, float inv_scale, const uint8_t* body, int nbody, uint32_t mode,
                  double* out, double* scratch, void* stream, const char* who)
{
    g_err[0] = 0;
    if (int e = check_lattice(lat)) return e;
    const lbm_lattice& L = *lat;
    if (nbody < 0 || nbody > kMaxBodies) return fail(LBM_ERR_ARG, "%s: nbody %d outside [0, %d]", who, nbody, kMaxBodies);
    if (!f || !out || !scratch || (nbody > 0 && !body)) return fail(LBM_ERR_ARG, "%s: NULL array", who);
    const bool ucol = mode & LBM_STEP_UREF_COLUMN;
    if (!L.Fx || !L.Fy || !L.Fz || !L.cfw || !L.rho || !L.ux || !L.uy || !L.uz || (ucol ? !L.colU : !L.uref))
        return fail(LBM_ERR_ARG, "%s: NULL field", who);
    static const uint8_t no_body = 0;
    cudaStream_t st = as_stream(stream);
    const int nacc = 3 * nbody + 3;
    k_body_forces<T><<<kBodyBlocks, kBodyThreads, 0, st>>>(L, f, inv_scale, nbody > 0 ? body : &no_body, nbody, ucol,
                                                           scratch);
    if (int e = check_launch("k_body_forces")) return e;
    k_body_forces_sum<<<1, 64, 0, st>>>(scratch, kBodyBlocks, nacc, out);
    return check_launch("k_body_forces_sum");
}
}  // namespace

// =============================================================================================
// C ABI
// =============================================================================================
extern "C" {

const char* lbm_last_error(void) { return g_err; }

int lbm_abi_version(void) { return LBM_ABI_VERSION; }

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

int lbm_build_worklists(const lbm_lattice* lat, int cells_per_lane, uint8_t* scratch, uint32_t* plain,
                        uint32_t* solid, uint32_t* special, uint32_t* edge, int32_t* counts, void* stream)
{
    g_err[0] = 0;
    if (int e = check_lattice(lat)) return e;
    if (cells_per_lane != 2 && cells_per_lane != 4 && cells_per_lane != 8)
        return fail(LBM_ERR_ARG, "lbm_build_worklists: 2, 4 or 8 cells per lane");
    if (!scratch || !plain || !solid || !special || !edge || !counts)
        return fail(LBM_ERR_ARG, "lbm_build_worklists: NULL array");
    const int seg = 32 * cells_per_lane;
    const long long n = (long long)((lat->pitch + seg - 1) / seg) * lat->ny * lat->nz;
    if (n > 0xffffffffLL) return fail(LBM_ERR_ARG, "lbm_build_worklists: too many segments for 32-bit ids");
    cudaStream_t st = as_stream(stream);
    k_classify<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(*lat, cells_per_lane, scratch);
    if (int e = check_launch("k_classify")) return e;
    k_compact<<<1, 1024, 0, st>>>(scratch, n, plain, solid, special, edge, counts);
    return check_launch("k_compact");
}

int lbm_build_worklists_noalloc(const lbm_lattice* lat, int cells_per_lane, uint32_t* plain, uint32_t* solid,
                                uint32_t* special, uint32_t* edge, int32_t* counts, void* stream)
{
    g_err[0] = 0;
    if (int e = check_lattice(lat)) return e;
    if (cells_per_lane != 2 && cells_per_lane != 4 && cells_per_lane != 8)
        return fail(LBM_ERR_ARG, "lbm_build_worklists_noalloc: 2, 4 or 8 cells per lane");
    const int seg = 32 * cells_per_lane;
    const long long n = (long long)((lat->pitch + seg - 1) / seg) * lat->ny * lat->nz;
    if (n > kNoAllocMaxSegments)
        return fail(LBM_ERR_ARG,
                    "lbm_build_worklists_noalloc: %lld row segments exceed the static limit of %lld; "
                    "use lbm_build_worklists with a caller scratch buffer",
                    n, kNoAllocMaxSegments);
    if (!plain || !solid || !special || !edge || !counts)
        return fail(LBM_ERR_ARG, "lbm_build_worklists_noalloc: NULL array");
    uint8_t* scratch = nullptr;
    if (int e = noalloc_scratch(&scratch)) return e;
    cudaStream_t st = as_stream(stream);
    k_classify<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(*lat, cells_per_lane, scratch);
    if (int e = check_launch("k_classify")) return e;
    k_compact<<<1, 1024, 0, st>>>(scratch, n, plain, solid, special, edge, counts);
    return check_launch("k_compact");
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
    lbm_tile t = tile ? *tile : lbm_tile{LBM_PIPE_TMA, 1, 4, 4, 0};
    if (t.warps < 1 || t.warps > 8 || t.ctas_per_sm < 0)
        return fail(LBM_ERR_ARG, "lbm_fused_step: bad tile (%d warps, %d CTAs/SM)", t.warps, t.ctas_per_sm);
    cudaStream_t st = as_stream(stream);
    int e;
    if (L.sponge_cols > 0 && t.pipeline != LBM_PIPE_SPLIT)
        return fail(LBM_ERR_ARG, "lbm_fused_step: the outlet sponge needs the split pipeline");
    if (t.pipeline == LBM_PIPE_REGISTER) {
        if (t.cells_per_lane != 2 && t.cells_per_lane != 4)
            return fail(LBM_ERR_ARG, "lbm_fused_step: register pipeline needs 2 or 4 cells per lane");
        if (t.warps > 4) return fail(LBM_ERR_ARG, "lbm_fused_step: register pipeline takes 1..4 warps per CTA");
        e = t.cells_per_lane == 4 ? launch_reg_v<4>(L, fs, fd, mode, t, st) : launch_reg_v<2>(L, fs, fd, mode, t, st);
    } else if (t.pipeline == LBM_PIPE_TMA) {
        if (t.cells_per_lane != 1 || t.stages < 2 || t.stages > 8)
            return fail(LBM_ERR_ARG, "lbm_fused_step: TMA pipeline needs 1 cell per lane and 2..8 stages");
        e = launch_tma(L, fs, fd, mode, t, (L.nx - 1) % 32 != 0, st);
    } else if (t.pipeline == LBM_PIPE_SPLIT) {
        if (t.cells_per_lane != 2 && t.cells_per_lane != 4)
            return fail(LBM_ERR_ARG, "lbm_fused_step: split pipeline needs 2 or 4 cells per lane");
        if (t.warps > 4) return fail(LBM_ERR_ARG, "lbm_fused_step: split pipeline takes 1..4 warps per CTA");
        if (L.list_cells_per_lane != t.cells_per_lane || (L.n_plain > 0 && !L.rows_plain) ||
            (L.n_special > 0 && !L.rows_special) || (L.n_solid > 0 && !L.rows_solid) ||
            (L.n_edge > 0 && !L.rows_edge))
            return fail(LBM_ERR_ARG, "lbm_fused_step: split pipeline needs work lists built for %d cells per lane",
                        t.cells_per_lane);
        e = t.cells_per_lane == 4 ? launch_split_v<4>(L, fs, fd, mode, t, st) : launch_split_v<2>(L, fs, fd, mode, t, st);
    } else if (t.pipeline == LBM_PIPE_ASYNC) {
        if (t.cells_per_lane != 2)
            return fail(LBM_ERR_ARG, "lbm_fused_step: async pipeline needs 2 cells per lane");
        e = launch_async(L, fs, fd, mode, t, (L.nx - 1) % 32 != 0, st);
    } else {
        return fail(LBM_ERR_ARG, "lbm_fused_step: unknown pipeline %d", t.pipeline);
    }
    if (e) return e;
    if (t.pipeline == LBM_PIPE_SPLIT && (mode & LBM_STEP_SKIP_SPECIAL)) return LBM_OK;
    // x=nx-2 and x=nx-1 in different lanes (register), segments (split) or warps (TMA, async): the
    // outlet gets its own pass
    const bool split = t.pipeline == LBM_PIPE_REGISTER ? (L.nx % t.cells_per_lane == 1)
                     : t.pipeline == LBM_PIPE_SPLIT    ? ((L.nx - 1) % (32 * t.cells_per_lane) == 0)
                                                       : ((L.nx - 1) % 32 == 0);
    if (split) {
        const long long M = (long long)L.ny * L.nz;
        k_bc_rows<float><<<(unsigned)((M + 127) / 128), 128, 0, st>>>(L, fd, 2, 1.f);
        return check_launch("k_bc_rows");
    }
    return LBM_OK;
}

int64_t lbm_profiles_scratch_doubles(const lbm_lattice* lat)
{
    g_err[0] = 0;
    if (int e = check_lattice(lat)) return e;
    return (long long)PROF_NF * lat->nx * profile_chunks(*lat);
}

int lbm_profiles(const lbm_lattice* lat, double inv_navg, double* prof, double* bed_speed2, double* scratch,
                 void* stream)
{
    g_err[0] = 0;
    if (int e = check_lattice(lat)) return e;
    const lbm_lattice& L = *lat;
    if (!prof || !bed_speed2 || !scratch) return fail(LBM_ERR_ARG, "lbm_profiles: NULL output or scratch");
    if (!L.avg && (!L.rho || !L.ux || !L.uy || !L.uz)) return fail(LBM_ERR_ARG, "lbm_profiles: NULL field");
    if (!(inv_navg > 0.0)) return fail(LBM_ERR_ARG, "lbm_profiles: inv_navg must be positive");
    cudaStream_t st = as_stream(stream);
    const int nch = profile_chunks(L);
    const int rows = L.ny * L.nz, per = (rows + nch - 1) / nch;
    k_profile_partials<<<dim3((unsigned)((L.nx + 127) / 128), (unsigned)nch), 128, 0, st>>>(L, inv_navg, per, scratch);
    if (int e = check_launch("k_profile_partials")) return e;
    const long long n = (long long)PROF_NF * L.nx;
    k_profile_sum<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(scratch, nch, L.nx, prof);
    if (int e = check_launch("k_profile_sum")) return e;
    const long long m = (long long)L.nx * L.ny;
    k_bed_speed2<<<(unsigned)((m + 255) / 256), 256, 0, st>>>(L, inv_navg, bed_speed2);
    return check_launch("k_bed_speed2");
}

int64_t lbm_body_forces_scratch_doubles(int nbody)
{
    g_err[0] = 0;
    if (nbody < 0 || nbody > kMaxBodies) return fail(LBM_ERR_ARG, "body forces: nbody %d outside [0, %d]", nbody, kMaxBodies);
    return (int64_t)kBodyBlocks * (3 * nbody + 3);
}


int lbm_body_forces(const lbm_lattice* lat, const float* f, const uint8_t* body, int nbody, uint32_t mode, double* out,
                    double* scratch, void* stream)
{
    return body_forces_t<float>(lat, f, 1.f, body, nbody, mode, out, scratch, stream, "lbm_body_forces");
}

int lbm_body_forces_h(const lbm_lattice* lat, const uint16_t* h, float scale, const uint8_t* body, int nbody,
                      uint32_t mode, double* out, double* scratch, void* stream)
{
    if (int e = check_scale(scale, "lbm_body_forces_h")) return e;
    return body_forces_t<__half>(lat, reinterpret_cast<const __half*>(h), 1.0f / scale, body, nbody, mode, out,
                                 scratch, stream, "lbm_body_forces_h");
}

int lbm_batch_pull_offsets_bytes(void) { return (int)sizeof(PullOffsets); }

namespace {
int check_batch(const lbm_batch* b, const char* who)
{
    if (!b) return fail(LBM_ERR_ARG, "%s: batch is NULL", who);
    if (b->count < 1 || b->count > kBatchMaxCases)
        return fail(LBM_ERR_ARG, "%s: %d lattices (1..%d)", who, b->count, kBatchMaxCases);
    if (!b->lat || !b->pull_offsets || !b->scale || !b->pop0 || !b->pop1)
        return fail(LBM_ERR_ARG, "%s: NULL batch table", who);
    if (b->max_columns < 1 || b->max_rows < 1) return fail(LBM_ERR_ARG, "%s: max_columns/max_rows not set", who);
    if (b->n_plain < 0 || b->n_solid < 0 || b->n_special < 0 || b->n_edge < 0 ||
        (b->n_plain > 0 && !b->rows_plain) || (b->n_solid > 0 && !b->rows_solid) ||
        (b->n_special > 0 && !b->rows_special) || (b->n_edge > 0 && !b->rows_edge))
        return fail(LBM_ERR_ARG, "%s: bad work lists", who);
    return LBM_OK;
}
}  // namespace

int lbm_batch_init(const lbm_batch* b, void* stream)
{
    g_err[0] = 0;
    if (int e = check_batch(b, "lbm_batch_init")) return e;
    const int n = b->count * Q;
    k_batch_pull_offsets<<<(unsigned)((n + 127) / 128), 128, 0, as_stream(stream)>>>(
        b->lat, b->count, static_cast<PullOffsets*>(b->pull_offsets));
    return check_launch("lbm_batch_init");
}

int lbm_batch_step_h(const lbm_batch* b, int parity, uint32_t mode, const lbm_tile* tile, void* stream)
{
    g_err[0] = 0;
    if (int e = check_batch(b, "lbm_batch_step_h")) return e;
    const lbm_tile t = tile ? *tile : lbm_tile{LBM_PIPE_SPLIT, 2, 4, 0, 0};
    if (t.pipeline != LBM_PIPE_SPLIT || t.cells_per_lane != 2 || t.warps < 1 || t.warps > 4 || t.ctas_per_sm < 0 ||
        (t.stages != 0 && t.stages != 4 && t.stages != 8))
        return fail(LBM_ERR_ARG, "lbm_batch_step_h: batches run the split pipeline on 64-cell segments "
                                 "(cells_per_lane 2), 1..4 warps, stages 0/4/8");
    const BatchDesc B{b->lat, static_cast<const PullOffsets*>(b->pull_offsets), b->scale,
                      reinterpret_cast<__half* const*>(b->pop0), reinterpret_cast<__half* const*>(b->pop1)};
    const int par = parity & 1;
    cudaStream_t st = as_stream(stream);
    const bool out = mode & LBM_STEP_OUTPUT, ucol = mode & LBM_STEP_UREF_COLUMN, avg = mode & LBM_STEP_ACCUMULATE;
    if (!out) return ucol ? launch_batch_t<false, true, false>(*b, B, par, mode, t, st)
                          : launch_batch_t<false, false, false>(*b, B, par, mode, t, st);
    if (ucol) return avg ? launch_batch_t<true, true, true>(*b, B, par, mode, t, st)
                         : launch_batch_t<true, true, false>(*b, B, par, mode, t, st);
    return avg ? launch_batch_t<true, false, true>(*b, B, par, mode, t, st)
               : launch_batch_t<true, false, false>(*b, B, par, mode, t, st);
}

int lbm_batch_chunk_h(const lbm_batch* b, int parity0, int nsteps, uint32_t mode, uint32_t last_mode, uint32_t* sync,
                      void* stream)
{
    g_err[0] = 0;
    if (int e = check_batch(b, "lbm_batch_chunk_h")) return e;
    if (nsteps < 1) return fail(LBM_ERR_ARG, "lbm_batch_chunk_h: nsteps %d < 1", nsteps);
    if (!sync) return fail(LBM_ERR_ARG, "lbm_batch_chunk_h: NULL sync words");
    const bool ucol = mode & LBM_STEP_UREF_COLUMN;
    if ((mode & (LBM_STEP_OUTPUT | LBM_STEP_ACCUMULATE | LBM_STEP_SKIP_PLAIN | LBM_STEP_SKIP_SPECIAL)) ||
        !(last_mode & LBM_STEP_OUTPUT) || (bool)(last_mode & LBM_STEP_UREF_COLUMN) != ucol ||
        (last_mode & (LBM_STEP_SKIP_PLAIN | LBM_STEP_SKIP_SPECIAL)))
        return fail(LBM_ERR_ARG, "lbm_batch_chunk_h: mode must be the inner steps' (no OUTPUT/ACCUMULATE/SKIP) and "
                                 "last_mode the output step's, with the same UREF_COLUMN bit");
    const bool avg = last_mode & LBM_STEP_ACCUMULATE;
    const BatchDesc B{b->lat, static_cast<const PullOffsets*>(b->pull_offsets), b->scale,
                      reinterpret_cast<__half* const*>(b->pop0), reinterpret_cast<__half* const*>(b->pop1)};
    cudaStream_t st = as_stream(stream);
    auto kern = ucol ? (avg ? k_batch_chunk<true, true> : k_batch_chunk<true, false>)
                     : (avg ? k_batch_chunk<false, true> : k_batch_chunk<false, false>);
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 128, 0) != cudaSuccess || per_sm < 1)
        return fail(LBM_ERR_CUDA, "lbm_batch_chunk_h: occupancy query failed");
    const unsigned grid = (unsigned)(per_sm * sm_count());
    if (cudaMemsetAsync(sync, 0, 4 * sizeof(uint32_t), st) != cudaSuccess)
        return fail(LBM_ERR_CUDA, "lbm_batch_chunk_h: clearing the sync words: %s", cudaGetErrorString(cudaGetLastError()));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(128);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    const cudaError_t e = cudaLaunchKernelEx(&cfg, kern, B, b->count, parity0 & 1, nsteps, b->rows_special,
                                             b->n_special, b->rows_edge, b->n_edge, b->rows_plain, b->n_plain,
                                             b->rows_solid, b->n_solid, b->max_rows, b->max_columns, sync);
    if (e != cudaSuccess) return fail(LBM_ERR_CUDA, "k_batch_chunk: %s", cudaGetErrorString(e));
    return check_launch("k_batch_chunk");
}

int lbm_lift_coarse(const lbm_lattice* lat, const float* coarse, int stride, int X, int Y, int Z, int factor,
                    float su, float srho, float* f, void* stream)
{
    g_err[0] = 0;
    if (int e = check_lattice(lat)) return e;
    if (!coarse || !f || !lat->rho || !lat->ux || !lat->uy || !lat->uz) return fail(LBM_ERR_ARG, "lbm_lift_coarse: NULL array");
    if (stride < 4 || X < 1 || Y < 1 || Z < 1 || factor < 1) return fail(LBM_ERR_ARG, "lbm_lift_coarse: bad coarse grid");
    k_lift_coarse<<<(unsigned)((lat->cells + 255) / 256), 256, 0, as_stream(stream)>>>(*lat, coarse, stride, X, Y, Z,
                                                                                      factor, su, srho, f);
    return check_launch("lbm_lift_coarse");
}

int lbm_init_equilibrium_h(const lbm_lattice* lat, uint16_t* h, float scale, void* stream)
{
    g_err[0] = 0;
    if (int e = check_lattice(lat)) return e;
    if (int e = check_scale(scale, "lbm_init_equilibrium_h")) return e;
    if (!h) return fail(LBM_ERR_ARG, "lbm_init_equilibrium_h: NULL h");
    k_init_equilibrium_h<<<(unsigned)((lat->cells + 255) / 256), 256, 0, as_stream(stream)>>>(
        *lat, reinterpret_cast<__half*>(h), scale);
    return check_launch("lbm_init_equilibrium_h");
}

int lbm_pack_populations(const lbm_lattice* lat, const float* f, uint16_t* h, float scale, void* stream)
{
    g_err[0] = 0;
    if (int e = check_lattice(lat)) return e;
    if (int e = check_scale(scale, "lbm_pack_populations")) return e;
    if (!f || !h) return fail(LBM_ERR_ARG, "lbm_pack_populations: NULL array");
    const long long n = (long long)Q * lat->cells;
    k_pack_populations<<<(unsigned)((n + 255) / 256), 256, 0, as_stream(stream)>>>(f, reinterpret_cast<__half*>(h),
                                                                                    lat->cells, scale);
    return check_launch("lbm_pack_populations");
}

int lbm_unpack_populations(const lbm_lattice* lat, const uint16_t* h, float* f, float scale, void* stream)
{
    g_err[0] = 0;
    if (int e = check_lattice(lat)) return e;
    if (int e = check_scale(scale, "lbm_unpack_populations")) return e;
    if (!f || !h) return fail(LBM_ERR_ARG, "lbm_unpack_populations: NULL array");
    const long long n = (long long)Q * lat->cells;
    k_unpack_populations<<<(unsigned)((n + 255) / 256), 256, 0, as_stream(stream)>>>(
        reinterpret_cast<const __half*>(h), f, lat->cells, 1.0f / scale);
    return check_launch("lbm_unpack_populations");
}

int lbm_fused_step_h(const lbm_lattice* lat, const uint16_t* hs, uint16_t* hd, float scale, uint32_t mode,
                     const lbm_tile* tile, void* stream)
{
    g_err[0] = 0;
    if (int e = check_lattice(lat)) return e;
    const lbm_lattice& L = *lat;
    if (int e = check_scale(scale, "lbm_fused_step_h")) return e;
    if (L.pitch % 8) return fail(LBM_ERR_ARG, "lbm_fused_step_h: pitch %d must be a multiple of 8", L.pitch);
    if (!hs || !hd || hs == hd) return fail(LBM_ERR_ARG, "lbm_fused_step_h: hs/hd NULL or equal");
    if (!L.Fx || !L.Fy || !L.Fz || !L.cfw || !L.rho || !L.ux || !L.uy || !L.uz || !L.status)
        return fail(LBM_ERR_ARG, "lbm_fused_step_h: NULL field");
    if ((mode & LBM_STEP_UREF_COLUMN) ? !L.colU : !L.uref)
        return fail(LBM_ERR_ARG, "lbm_fused_step_h: NULL uref/colU");
    if ((mode & LBM_STEP_ACCUMULATE) && !L.avg) return fail(LBM_ERR_ARG, "lbm_fused_step_h: NULL avg");
    if (!aligned16(hs) || !aligned16(hd) || !aligned16(L.flags) || !aligned16(L.rho) || !aligned16(L.ux) ||
        !aligned16(L.uy) || !aligned16(L.uz) || (L.avg && !aligned16(L.avg)))
        return fail(LBM_ERR_ARG, "lbm_fused_step_h: arrays must be 16-byte aligned");
    const lbm_tile t = tile ? *tile : lbm_tile{LBM_PIPE_SPLIT, 2, 4, 0, 0};
    const int cpl = t.cells_per_lane;
    if (t.pipeline != LBM_PIPE_SPLIT || (cpl != 2 && cpl != 4 && cpl != 8) || t.warps < 1 || t.warps > 4 ||
        t.ctas_per_sm < 0)
        return fail(LBM_ERR_ARG, "lbm_fused_step_h: 16-bit storage runs the split pipeline with 2, 4 or 8 cells "
                                 "per lane and 1..4 warps per CTA");
    if (t.stages != 0 && t.stages != 8 && !(t.stages == 4 && cpl <= 4))
        return fail(LBM_ERR_ARG, "lbm_fused_step_h: tile.stages (plain-kernel cells per lane) must be 0, 8, or 4 "
                                 "with 2 or 4 cells per lane");
    if (L.list_cells_per_lane != cpl || (L.n_plain > 0 && !L.rows_plain) || (L.n_special > 0 && !L.rows_special) ||
        (L.n_solid > 0 && !L.rows_solid) || (L.n_edge > 0 && !L.rows_edge))
        return fail(LBM_ERR_ARG, "lbm_fused_step_h: needs work lists built for %d cells per lane", cpl);
    cudaStream_t st = as_stream(stream);
    const __half* s16 = reinterpret_cast<const __half*>(hs);
    __half* d16 = reinterpret_cast<__half*>(hd);
    if (int e = launch_split_h(L, s16, d16, scale, mode, t, st)) return e;
    if (mode & LBM_STEP_SKIP_SPECIAL) return LBM_OK;
    const int vg = cpl == 2 ? 2 : 4;
    if ((L.nx - 1) % (32 * vg) == 0) {  // x=nx-2 and x=nx-1 in different segments: the outlet gets its own pass
        const long long M = (long long)L.ny * L.nz;
        k_bc_rows<__half><<<(unsigned)((M + 127) / 128), 128, 0, st>>>(L, d16, 2, scale);
        return check_launch("k_bc_rows");
    }
    return LBM_OK;
}

}  // extern "C"
