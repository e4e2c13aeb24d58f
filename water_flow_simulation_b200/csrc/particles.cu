// particles.cu -- tracer particles advected through the lattice's velocity field on the device
// (Run3D.move_particles, floodsim/reach3d.py:508-536).
//
// One thread per particle, positions in float64 metres (x from the inlet face, y from the
// first lattice row, z from the domain bottom), as the reference keeps them:
//   * the velocity of the cell the particle is in (truncated indices, clipped to the
//     lattice), times vel in float32, non-finite components replaced by 0, times dt in
//     float32, added to the float64 position -- NumPy's promotions of the reference;
//   * a particle that is no longer finite, leaves the domain (x past nx-1 cells, y or z out
//     of range) or lands in a solid cell is put back at the inlet: x uniform in [0, 2 dx),
//     y and z uniform over a random fluid cell of the x = 1 column.
// The reference draws respawn positions from an unseeded NumPy generator; here they come
// from SplitMix64 (Steele, Lea and Flood 2014) of (seed, call counter, particle, draw), so a
// run is reproducible from its seed.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>

#include "d3q19.cuh"
#include "errors.cuh"
#include "../../include/lbm_b200.h"

using namespace wfs;

namespace {

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

__device__ __forceinline__ uint64_t splitmix64(uint64_t z)
{
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// uniform double in [0, 1): the top 53 bits of one SplitMix64 output
__device__ __forceinline__ double uniform(uint64_t seed, uint64_t counter, long long p, int draw)
{
    const uint64_t h = splitmix64(splitmix64(seed ^ splitmix64(counter)) + (uint64_t)p * 4u + (uint64_t)draw);
    return (double)(h >> 11) * 0x1.0p-53;
}

__device__ __forceinline__ int cell_index(double coord, double dx)
{
    const double v = coord / dx;
    if (!(v < 2147483647.0)) return 2147483647;        // +inf / huge: past every bound
    if (!(v > -2147483647.0)) return -2147483647;      // -inf / huge negative
    return (int)v;                                      // truncation toward zero, as astype(int)
}

__device__ __forceinline__ float finite_or_zero(float v) { return isfinite(v) ? v : 0.0f; }

__global__ void __launch_bounds__(256) k_move_particles(const lbm_lattice L, double* __restrict__ P, long long n,
                                                        float vel, float dt, double dx,
                                                        const int32_t* __restrict__ inlet, int n_inlet,
                                                        uint64_t seed, uint64_t counter, int* __restrict__ respawned)
{
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    double x = P[3 * p], y = P[3 * p + 1], z = P[3 * p + 2];
    const int ix = min(max(cell_index(x, dx), 0), L.nx - 1);
    const int iy = min(max(cell_index(y, dx), 0), L.ny - 1);
    const int iz = min(max(cell_index(z, dx), 0), L.nz - 1);
    const long long c = (long long)ix + (long long)L.pitch * (iy + (long long)L.ny * iz);
    const float ux = finite_or_zero(__fmul_rn(L.ux[c], vel));
    const float uy = finite_or_zero(__fmul_rn(L.uy[c], vel));
    const float uz = finite_or_zero(__fmul_rn(L.uz[c], vel));
    x += (double)__fmul_rn(ux, dt);
    y += (double)__fmul_rn(uy, dt);
    z += (double)__fmul_rn(uz, dt);
    const bool fin = isfinite(x) && isfinite(y) && isfinite(z);
    bool bad = !fin;
    if (fin) {
        const int jx = cell_index(x, dx), jy = cell_index(y, dx), jz = cell_index(z, dx);
        bad = jx < 0 || jx >= L.nx - 1 || jy < 0 || jy >= L.ny || jz < 0 || jz >= L.nz;
        if (!bad) bad = (L.flags[(long long)jx + (long long)L.pitch * (jy + (long long)L.ny * jz)] & FLAG_SOLID) != 0;
    }
    if (bad) {
        const int k = min((int)(uniform(seed, counter, p, 0) * n_inlet), n_inlet - 1);
        const int yz = inlet[k];                       // z * ny + y of a fluid cell at x = 1
        x = uniform(seed, counter, p, 1) * 2.0 * dx;
        y = ((double)(yz % L.ny) + uniform(seed, counter, p, 2)) * dx;
        z = ((double)(yz / L.ny) + uniform(seed, counter, p, 3)) * dx;
        if (respawned) atomicAdd(respawned, 1);
    }
    P[3 * p] = x;
    P[3 * p + 1] = y;
    P[3 * p + 2] = z;
}

}  // namespace

extern "C" {

int lbm_move_particles(const lbm_lattice* lat, double* P, int64_t n, float vel, float dt, double dx,
                       const int32_t* inlet, int32_t n_inlet, uint64_t seed, uint64_t counter, int32_t* respawned,
                       void* stream)
{
    g_err[0] = 0;
    if (!lat) return fail(LBM_ERR_ARG, "lbm_move_particles: lattice is NULL");
    if (n < 0) return fail(LBM_ERR_ARG, "lbm_move_particles: negative particle count");
    if (n == 0) return 0;
    if (!P || !inlet || !lat->ux || !lat->uy || !lat->uz || !lat->flags)
        return fail(LBM_ERR_ARG, "lbm_move_particles: NULL array");
    if (n_inlet < 1) return fail(LBM_ERR_ARG, "lbm_move_particles: no fluid inlet cell to respawn at");
    if (!(dx > 0.0)) return fail(LBM_ERR_ARG, "lbm_move_particles: dx must be positive");
    if (lat->nx < 2 || lat->ny < 1 || lat->nz < 1 || lat->pitch < lat->nx)
        return fail(LBM_ERR_ARG, "lbm_move_particles: bad lattice %dx%dx%d", lat->nx, lat->ny, lat->nz);
    const unsigned grid = (unsigned)((n + 255) / 256);
    k_move_particles<<<grid, 256, 0, as_stream(stream)>>>(*lat, P, n, vel, dt, dx, inlet, n_inlet, seed, counter,
                                                          reinterpret_cast<int*>(respawned));
    return check_launch("lbm_move_particles");
}

}  // extern "C"
