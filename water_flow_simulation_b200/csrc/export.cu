// export.cu -- the web viewer's velocity export on the device (floodsim/web3d.py:35-56).
//
// The viewer stores the time-averaged velocity of a case pooled over 2 x 2 horizontal blocks
// (the fluid-cell mean of each block) and quantised to int8 with one scale for the case.  On
// the host that reads three float32 fields of the whole lattice back from the GPU and makes
// several full-size NumPy temporaries; here two launches read the float32 time-average sums
// where they already are and return only the int8 blocks (3 bytes per 4 cells) and the
// block speeds the percentile needs.
//
//   pass 1 (k_export_pool): one thread per block, writing (vx, vy, vz, fluid count).
//     mean = sum / navg, x vel (float32, as Run3D.field rounds it); the block sum in NumPy's order for the reference's two-axis
//     reduction, (a00 + a01) + (a10 + a11) with a_row,col, solids multiplied by 0 as `a * fl`
//     does; divided by the fluid count.  The largest |component| goes to one word by
//     atomicMax on its bits (non-negative floats order like their bit patterns).
//   pass 2 (k_export_quantize): scale = float32(umax / 126) in float64 (NumPy converts the
//     Python float scale to float32 for `a / scale`), q = clip(rint(a / scale), +-126), -128
//     where the block has no fluid; the block speed sqrt(a0^2 + a1^2 + a2^2) in float32.
// Every float operation is an explicitly rounded intrinsic, so --use_fast_math changes
// nothing and the output equals the reference's bit for bit.
#include <cuda_runtime.h>

#include <cstdint>

#include "d3q19.cuh"
#include "errors.cuh"
#include "../../include/lbm_b200.h"

using namespace wfs;

namespace {

constexpr int kExportStride = 2;

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

__device__ __forceinline__ float cell_value(const float* __restrict__ sum, const uint32_t* __restrict__ flags,
                                            long long c, float navg, float vel, float& fl)
{
    fl = (flags[c] & FLAG_SOLID) ? 0.0f : 1.0f;
    return __fmul_rn(__fmul_rn(__fdiv_rn(sum[c], navg), vel), fl);
}

__global__ void __launch_bounds__(256) k_export_pool(const lbm_lattice L, float navg, float vel,
                                                     float* __restrict__ pooled, uint32_t* __restrict__ umax_bits)
{
    const int nx2 = L.nx / kExportStride, ny2 = L.ny / kExportStride;
    const long long nb = (long long)nx2 * ny2 * L.nz;
    const long long b = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    float local = 0.0f;
    if (b < nb) {
        const int i = (int)(b % nx2), j = (int)((b / nx2) % ny2), z = (int)(b / ((long long)nx2 * ny2));
        const long long r0 = (long long)L.pitch * ((long long)2 * j + (long long)L.ny * z) + 2 * i;
        const long long r1 = r0 + L.pitch;
        float n = 0.0f;
        for (int k = 0; k < 3; ++k) {
            const float* sum = L.avg + (long long)k * L.cells;
            float f00, f01, f10, f11;
            const float a00 = cell_value(sum, L.flags, r0, navg, vel, f00);
            const float a01 = cell_value(sum, L.flags, r0 + 1, navg, vel, f01);
            const float a10 = cell_value(sum, L.flags, r1, navg, vel, f10);
            const float a11 = cell_value(sum, L.flags, r1 + 1, navg, vel, f11);
            if (k == 0) n = (f00 + f01) + (f10 + f11);            // small integers: exact
            const float tot = __fadd_rn(__fadd_rn(a00, a01), __fadd_rn(a10, a11));
            const float v = n > 0.0f ? __fdiv_rn(tot, n) : 0.0f;
            pooled[b * 4 + k] = v;
            local = fmaxf(local, fabsf(v));
        }
        pooled[b * 4 + 3] = n;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) local = fmaxf(local, __shfl_xor_sync(0xffffffffu, local, o));
    if ((threadIdx.x & 31) == 0 && local > 0.0f) atomicMax(umax_bits, __float_as_uint(local));
}

__global__ void __launch_bounds__(256) k_export_quantize(const float* __restrict__ pooled, long long nb,
                                                         const uint32_t* __restrict__ umax_bits,
                                                         int8_t* __restrict__ q, float* __restrict__ sp)
{
    const long long b = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nb) return;
    float umax = __uint_as_float(*umax_bits);
    if (umax == 0.0f) umax = 1.0f;                                // `max(...) or 1.0`
    const float scale = (float)((double)umax / 126.0);
    const float4 p = reinterpret_cast<const float4*>(pooled)[b];
    if (p.w == 0.0f) {                                            // no fluid in the block
        q[b * 3] = q[b * 3 + 1] = q[b * 3 + 2] = (int8_t)-128;
        sp[b] = 0.0f;
        return;
    }
    const float a[3] = {p.x, p.y, p.z};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float r = fminf(fmaxf(rintf(__fdiv_rn(a[k], scale)), -126.0f), 126.0f);
        q[b * 3 + k] = (int8_t)(int)r;
    }
    sp[b] = __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(a[0], a[0]), __fmul_rn(a[1], a[1])), __fmul_rn(a[2], a[2])));
}

}  // namespace

extern "C" {

int64_t lbm_export_blocks(const lbm_lattice* lat)
{
    g_err[0] = 0;
    if (!lat) return fail(LBM_ERR_ARG, "lbm_export_blocks: lattice is NULL");
    if (lat->nx < kExportStride || lat->ny < kExportStride || lat->nz < 1)
        return fail(LBM_ERR_ARG, "lbm_export_blocks: lattice %dx%dx%d smaller than one block", lat->nx, lat->ny,
                    lat->nz);
    return (int64_t)(lat->nx / kExportStride) * (lat->ny / kExportStride) * lat->nz;
}

int lbm_export_velocity(const lbm_lattice* lat, int navg, float vel, float* pooled, uint32_t* umax_bits, int8_t* q,
                        float* sp, void* stream)
{
    const int64_t nb = lbm_export_blocks(lat);
    if (nb < 0) return (int)nb;
    if (!lat->avg || !lat->flags) return fail(LBM_ERR_ARG, "lbm_export_velocity: no time averages or flags");
    if (!pooled || !umax_bits || !q || !sp) return fail(LBM_ERR_ARG, "lbm_export_velocity: NULL output");
    if (reinterpret_cast<uintptr_t>(pooled) & 15)
        return fail(LBM_ERR_ARG, "lbm_export_velocity: pooled must be 16-byte aligned");
    if (navg < 1 || navg > (1 << 24)) return fail(LBM_ERR_ARG, "lbm_export_velocity: navg %d out of range", navg);
    if (lat->pitch < lat->nx || lat->cells != (int64_t)lat->pitch * lat->ny * lat->nz)
        return fail(LBM_ERR_ARG, "lbm_export_velocity: pitch/cells inconsistent");
    cudaStream_t st = as_stream(stream);
    if (cudaMemsetAsync(umax_bits, 0, sizeof(uint32_t), st) != cudaSuccess) return check_launch("lbm_export_velocity");
    const unsigned grid = (unsigned)((nb + 255) / 256);
    k_export_pool<<<grid, 256, 0, st>>>(*lat, (float)navg, vel, pooled, umax_bits);
    if (int e = check_launch("lbm_export_velocity (pool)")) return e;
    k_export_quantize<<<grid, 256, 0, st>>>(pooled, nb, umax_bits, q, sp);
    return check_launch("lbm_export_velocity (quantize)");
}

}  // extern "C"
