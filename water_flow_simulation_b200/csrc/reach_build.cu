// reach_build.cu -- the three-dimensional part of the reach builder on the device
// (build_reach and wall_cf, floodsim/reach3d.py:201-297, 315-343).
//
// Everything in a reach that is a full (nz, ny, nx) array -- the solid and bed masks, the
// wall friction coefficient and the bed/bank wall mask -- is made here from small inputs the
// host computes exactly as the reference does:
//   kb[y, x]   the number of cell centres below the bed of column (y, x) (zc < bed level);
//   outside[y] the columns beyond the top width (solid from bed to lid);
//   hull segments, per x: y index ranges [y0, y1] solid from z index z0 up to the lid
//              (a hull's tapered beam is one y range per x; its keel one z index);
//   cf_col     the Manning cf of each column's bed/bank cells; cf_hull the log-law cf.
// k_reach_masks writes solid = bed | hull and bed; k_reach_walls marks the fluid cells that
// a D3Q19 link (the 18 neighbours) joins to the bed -- with the bed below z = 0 and the two
// y edges of the domain counted as bed -- or to a hull (nothing outside counted), pulling
// x beyond the ends back to the end columns, as the reference's padded binary dilation does.
// Bed/bank cells take cf_col, hull-adjacent cells cf_hull, and the first and last two x
// columns neither.  Pure integer and comparison work: the arrays equal the host builder's
// bit for bit (tests/test_gpu_reach_build.py).
#include <cuda_runtime.h>

#include <cstdint>

#include "errors.cuh"
#include "../../include/lbm_b200.h"

using namespace wfs;

namespace {

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

__global__ void __launch_bounds__(256) k_reach_masks(int nx, int ny, int nz, const int32_t* __restrict__ kb,
                                                     const uint8_t* __restrict__ outside,
                                                     const int32_t* __restrict__ seg_off,
                                                     const int32_t* __restrict__ segs, uint8_t* __restrict__ solid,
                                                     uint8_t* __restrict__ bed)
{
    const long long N = (long long)nx * ny * nz;
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= N) return;
    const int x = (int)(c % nx), y = (int)((c / nx) % ny), z = (int)(c / ((long long)nx * ny));
    const bool b = outside[y] || z < kb[(long long)y * nx + x];
    bool s = b;
    for (int k = seg_off[x]; k < seg_off[x + 1] && !s; ++k)
        s = y >= segs[3 * k] && y <= segs[3 * k + 1] && z >= segs[3 * k + 2];
    solid[c] = s;
    bed[c] = b;
}

// mask value of a neighbour (bit 0 of `m`: the mask itself; out-of-lattice rules per kind)
__device__ __forceinline__ bool neighbour(const uint8_t* __restrict__ m, int x, int y, int z, int nx, int ny, int nz,
                                          bool floor)
{
    x = x < 0 ? 0 : (x >= nx ? nx - 1 : x);               // x: the end columns repeat
    if (y < 0 || y >= ny) return floor;                    // y edges: wall for the bed only
    if (z < 0) return floor;                               // below the bed datum: bed
    if (z >= nz) return false;                             // above the lid: open
    return m[x + (long long)nx * (y + (long long)ny * z)] != 0;
}

__global__ void __launch_bounds__(256) k_reach_walls(int nx, int ny, int nz, const uint8_t* __restrict__ solid,
                                                     const uint8_t* __restrict__ bed, const uint8_t* __restrict__ hull,
                                                     const float* __restrict__ cf_col, float cf_hull,
                                                     float* __restrict__ cf, uint8_t* __restrict__ bedwall)
{
    const long long N = (long long)nx * ny * nz;
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= N) return;
    const int x = (int)(c % nx), y = (int)((c / nx) % ny), z = (int)(c / ((long long)nx * ny));
    bool on_bed = false, on_hull = false;
    if (!solid[c]) {
        for (int dz = -1; dz <= 1; ++dz)
            for (int dy = -1; dy <= 1; ++dy)
                for (int dx = -1; dx <= 1; ++dx) {
                    if (dx != 0 && dy != 0 && dz != 0) continue;       // cube corners are not D3Q19 links
                    on_bed = on_bed || neighbour(bed, x + dx, y + dy, z + dz, nx, ny, nz, true);
                    on_hull = on_hull || neighbour(hull, x + dx, y + dy, z + dz, nx, ny, nz, false);
                }
    }
    const bool ends = x < 2 || x >= nx - 2;
    const bool bw = on_bed && !ends;
    bedwall[c] = bw;
    cf[c] = ends ? 0.0f : (bw ? cf_col[(long long)y * nx + x] : (on_hull ? cf_hull : 0.0f));
}

__global__ void k_hull_mask(long long N, const uint8_t* __restrict__ solid, const uint8_t* __restrict__ bed,
                            uint8_t* __restrict__ hull)
{
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c < N) hull[c] = solid[c] && !bed[c];
}

int check(const char* what, int nx, int ny, int nz)
{
    if (nx < 1 || ny < 1 || nz < 1) return fail(LBM_ERR_ARG, "%s: bad lattice %dx%dx%d", what, nx, ny, nz);
    return 0;
}

}  // namespace

extern "C" {

int lbm_build_reach_masks(int nx, int ny, int nz, const int32_t* kb, const uint8_t* outside, const int32_t* seg_off,
                          const int32_t* segs, uint8_t* solid, uint8_t* bed, void* stream)
{
    g_err[0] = 0;
    if (int e = check("lbm_build_reach_masks", nx, ny, nz)) return e;
    if (!kb || !outside || !seg_off || !segs || !solid || !bed)
        return fail(LBM_ERR_ARG, "lbm_build_reach_masks: NULL array");
    const long long N = (long long)nx * ny * nz;
    k_reach_masks<<<(unsigned)((N + 255) / 256), 256, 0, as_stream(stream)>>>(nx, ny, nz, kb, outside, seg_off, segs,
                                                                            solid, bed);
    return check_launch("lbm_build_reach_masks");
}

int lbm_build_reach_walls(int nx, int ny, int nz, const uint8_t* solid, const uint8_t* bed, uint8_t* hull_scratch,
                          const float* cf_col, float cf_hull, float* cf, uint8_t* bedwall, void* stream)
{
    g_err[0] = 0;
    if (int e = check("lbm_build_reach_walls", nx, ny, nz)) return e;
    if (!solid || !bed || !hull_scratch || !cf_col || !cf || !bedwall)
        return fail(LBM_ERR_ARG, "lbm_build_reach_walls: NULL array");
    const long long N = (long long)nx * ny * nz;
    const unsigned grid = (unsigned)((N + 255) / 256);
    k_hull_mask<<<grid, 256, 0, as_stream(stream)>>>(N, solid, bed, hull_scratch);
    if (int e = check_launch("lbm_build_reach_walls (hull)")) return e;
    k_reach_walls<<<grid, 256, 0, as_stream(stream)>>>(nx, ny, nz, solid, bed, hull_scratch, cf_col, cf_hull, cf,
                                                      bedwall);
    return check_launch("lbm_build_reach_walls");
}

}  // extern "C"
