// fused_async.cuh -- per-warp asynchronous-copy pipeline of the fused step (lbm_tile.pipeline = 2).
// Included inside the anonymous namespace of lbm_kernels.cu, after fused_tma.cuh.
//
// Every warp is independent.  It owns work items (64-cell x segment, y) -- global warp
// g takes items g, g + W_total, ... -- and walks the nz rows of each item in turn, so the
// depth-mean column sums of the wall model accumulate in registers.
//
// All bulk global traffic moves in 16-byte pieces (on B200 this 38-stream pattern reaches
// ~6 TB/s with 16-byte accesses but only ~4 TB/s with 4- or 8-byte ones):
//   * loads: cp.async 16-byte copies stage the next D-1 rows -- the 19 pulled source rows
//     of the 64 cells (one copy instruction covers two directions: 16 lanes x 16 bytes
//     each), the 16-byte halo chunks that the 10 x-moving directions need, and the 64 flag
//     words -- into a private ring of D shared-memory slots, while the warp collides the
//     current row; no registers hold data in flight;
//   * stores: each cell writes its 19 outputs to a shared-memory row buffer, and the warp
//     writes the buffer back with 16-byte streaming stores (two directions per instruction).
// A lane collides cells x0+lane and x0+32+lane, so all shared-memory accesses of the
// collision are conflict-free.  Inlet/outlet extrapolation uses warp shuffles.
#pragma once

constexpr int kSegA = 64;          // cells of a row per warp
constexpr int kRowA = kSegA + 8;   // staged floats per direction row: x0-4 .. x0+67

struct AsyncLayout {
    int warps, D;
    size_t slot_bytes, out_bytes, warp_bytes, bytes;
    __host__ __device__ AsyncLayout(int w, int d) : warps(w), D(d)
    {
        slot_bytes = (size_t)Q * kRowA * sizeof(float) + (size_t)kSegA * sizeof(uint32_t);
        out_bytes = (size_t)Q * kSegA * sizeof(float);
        warp_bytes = (size_t)D * slot_bytes + out_bytes;
        warp_bytes = (warp_bytes + 127) / 128 * 128;   // every warp's region starts 128-byte aligned
        bytes = (size_t)warps * warp_bytes;
    }
};

__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gsrc)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(static_cast<uint32_t>(__cvta_generic_to_shared(smem_dst))),
                 "l"(gsrc)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// x-moving directions and the halo chunk each needs: lanes 0..4 copy the chunk left of the
// segment for c_x = +1, lanes 5..9 the chunk right of it for c_x = -1.
__host__ __device__ constexpr int halo_dir(int k)
{
    return k == 0 ? 1 : k == 1 ? 7 : k == 2 ? 9 : k == 3 ? 11 : k == 4 ? 13
         : k == 5 ? 2 : k == 6 ? 8 : k == 7 ? 10 : k == 8 ? 12 : 14;
}

// Stage row (y, z) of the segment starting at x0 into `slot` (index in a direction row:
// x - x0 + 4).  Copies outside [0, pitch) are skipped: only x edges and padding read them.
template <bool INTERIOR>
__device__ __forceinline__ void stage_row16(float* slot, const lbm_lattice& L, const float* fs, const PullOffsets& po,
                                            int x0, int y, int z, int lane)
{
    const long long rowc = ((long long)z * L.ny + y) * L.pitch;
    const int half = lane >> 4, chunk = lane & 15;
    const int xc = x0 + 4 * chunk;
    const bool okc = xc < L.pitch;
#pragma unroll
    for (int j = 0; j < (Q + 1) / 2; ++j) {
        const int i = 2 * j + half;
        if (i < Q && okc) {
            const float* row = INTERIOR ? fs + rowc + po.d[i] : source_row(L, fs, i, y, z);
            cp_async16(slot + i * kRowA + 4 + 4 * chunk, row + xc);
        }
    }
    if (lane < 10) {
        const int i = halo_dir(lane);
        const int xh = lane < 5 ? x0 - 4 : x0 + kSegA;
        if (xh >= 0 && xh + 4 <= L.pitch) {
            const float* row = INTERIOR ? fs + rowc + po.d[i] : source_row(L, fs, i, y, z);
            cp_async16(slot + i * kRowA + (lane < 5 ? 0 : kSegA + 4), row + xh);
        }
    }
    if (lane < 16 && okc) cp_async16(slot + Q * kRowA + 4 * chunk, L.flags + rowc + xc);
}

template <int I>
__device__ __forceinline__ void read_dir(float (&f)[Q], const float* s, uint32_t rwm)
{
    if constexpr (I == 0) f[0] = s[0];
    else f[I] = s[I * kRowA - ((rwm >> I) & 1u ? 0 : cx(I))];
}
template <int... Is>
__device__ __forceinline__ void read_all(std::integer_sequence<int, Is...>, float (&f)[Q], const float* s, uint32_t rwm)
{
    (read_dir<Is>(f, s, rwm), ...);
}

template <int I>
__device__ __forceinline__ void read_dir_interior(float (&f)[Q], const float* s)
{
    f[I] = s[I * kRowA - cx(I)];
}
template <int... Is>
__device__ __forceinline__ void read_all_interior(std::integer_sequence<int, Is...>, float (&f)[Q], const float* s)
{
    (read_dir_interior<Is>(f, s), ...);
}

template <bool OUT, bool UCOL, bool AVG, int D>
__global__ void __launch_bounds__(256, 2) k_fused_async(const lbm_lattice L, const PullOffsets po,
                                                        const float* __restrict__ fs, float* __restrict__ fd,
                                                        int outlet_fused)
{
    extern __shared__ __align__(128) unsigned char smem[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const AsyncLayout lay(nw, D);
    unsigned char* wbase = smem + warp * lay.warp_bytes;
    float* ring = reinterpret_cast<float*>(wbase);
    float* outb = reinterpret_cast<float*>(wbase + (size_t)D * lay.slot_bytes);
    const size_t slotf = lay.slot_bytes / sizeof(float);

    const int nseg = (L.pitch + kSegA - 1) / kSegA;
    const int nitems = nseg * L.ny;
    const int gw = blockIdx.x * nw + warp, W = gridDim.x * nw;
    if (gw >= nitems) return;                                   // whole warp; no CTA-wide barrier follows
    const int nrows = ((nitems - 1 - gw) / W + 1) * L.nz;
    const long long S = L.cells;

    int it_item = gw, it_z = 0;                                 // next row to stage
    auto stage_next = [&](int slot_idx) {
        const int seg = it_item % nseg, y = it_item / nseg;
        float* slot = ring + slot_idx * slotf;
        const bool interior = y >= 1 && y <= L.ny - 2 && it_z >= 1 && it_z <= L.nz - 2;
        if (interior) stage_row16<true>(slot, L, fs, po, seg * kSegA, y, it_z, lane);
        else stage_row16<false>(slot, L, fs, po, seg * kSegA, y, it_z, lane);
        if (++it_z == L.nz) { it_z = 0; it_item += W; }
    };
#pragma unroll
    for (int q = 0; q < D - 1; ++q) {
        if (q < nrows) stage_next(q);
        cp_async_commit();
    }

    int item = gw, z = 0;                                       // row being computed
    int slot_idx = 0;
    float csx0 = 0.f, csy0 = 0.f, ccn0 = 0.f, csx1 = 0.f, csy1 = 0.f, ccn1 = 0.f;   // column sums, cells 0/1
    for (int r = 0; r < nrows; ++r) {
        const int ahead = r + D - 1;
        if (ahead < nrows) stage_next(ahead % D);
        cp_async_commit();
        cp_async_wait<D - 1>();                                 // this lane's copies of row r have landed
        __syncwarp();                                           // ... and every other lane's

        const int seg = item % nseg, y = item / nseg;
        const int x0 = seg * kSegA;
        const float* slot = ring + slot_idx * slotf;
        const uint32_t* sfl = reinterpret_cast<const uint32_t*>(slot + Q * kRowA);
        const long long rowc = ((long long)z * L.ny + y) * L.pitch;
        uint32_t rwm = 0;                                       // directions whose source row is outside
#pragma unroll
        for (int i = 1; i < Q; ++i) {
            const int ys = y - cy(i), zs = z - cz(i);
            if (ys < 0 || ys >= L.ny || zs < 0) rwm |= 1u << i;
        }
        // rows with no edge, wall, solid or forced cell take the fast path: compile-time
        // shared-memory offsets, no per-cell tests (warp-uniform decision per 32-cell group)
        const bool edge_seg = x0 == 0 || (x0 <= L.nx - 1 && L.nx - 1 < x0 + kSegA) || x0 + kSegA > L.nx;
        constexpr uint32_t kSpecial = FLAG_SOLID | FLAG_WALLS | FLAG_WALLFN | FLAG_FORCE;
#pragma unroll 1
        for (int k = 0; k < 2; ++k) {
            const int xi = 32 * k + lane;                       // cell's index within the segment
            const int x = x0 + xi;
            const bool inrow = x < L.pitch;
            const long long c = rowc + x;
            const uint32_t fk = inrow ? sfl[xi] : (FLAG_GHOST | FLAG_SOLID);
            float f[Q];
            float R, UX, UY, UZ;
            const bool fast = rwm == 0 && !edge_seg && __all_sync(0xffffffffu, (fk & kSpecial) == 0);
            if (fast) {
                read_all_interior(std::make_integer_sequence<int, Q>{}, f, slot + xi + 4);
                collide(f, 0.f, 0.f, 0.f, L.tau0, L.csmag2, R, UX, UY, UZ);
            } else if (fk & FLAG_SOLID) {
                R = 1.f; UX = 0.f; UY = 0.f; UZ = 0.f;
#pragma unroll
                for (int i = 0; i < Q; ++i) f[i] = wgt(i);
            } else {
                read_all(std::make_integer_sequence<int, Q>{}, f, slot + xi + 4, rwm);
                const uint32_t bb = fk & FLAG_WALLS & ~rwm;
                if (bb) {
#pragma unroll
                    for (int i = 1; i < Q; ++i)
                        if (bb & (1u << i)) f[i] = __ldg(fs + (long long)opp(i) * S + c);
                }
                if (x == 0 || x == L.nx - 1) {
#pragma unroll
                    for (int i = 1; i < Q; ++i)
                        if ((x == 0 && cx(i) == 1) || (x == L.nx - 1 && cx(i) == -1))
                            f[i] = __ldg(fs + (long long)i * S + c);
                }
                if (fk & FLAG_WALLFN) {
                    float U;
                    if constexpr (UCOL) U = (fk & FLAG_BEDWALL) ? L.colU[(long long)y * L.pitch + x] : 0.f;
                    else U = L.uref[c];
                    wall_function(f, fk & FLAG_WALLS, L.cfw[c], L.ux[c], L.uy[c], L.uz[c], L.rho[c], U);
                }
                float fx = 0.f, fy = 0.f, fz = 0.f;
                if (fk & FLAG_FORCE) {
                    fx = L.Fx[c] * L.force_scale;
                    fy = L.Fy[c] * L.force_scale;
                    fz = L.Fz[c] * L.force_scale;
                }
                collide(f, fx, fy, fz, L.tau0, L.csmag2, R, UX, UY, UZ);
            }
            // inlet: x=0 (lane 0 of the first group of segment 0) from x=1 (lane 1)
            if (x0 == 0 && k == 0) {
                float g[Q];
#pragma unroll
                for (int i = 0; i < Q; ++i) g[i] = __shfl_down_sync(0xffffffffu, f[i], 1);
                const uint32_t f1 = __shfl_down_sync(0xffffffffu, fk, 1);
                if (lane == 0 && !(fk & FLAG_SOLID) && !(f1 & FLAG_SOLID))
                    nebb<true>(g, f, L.uin[y + (long long)L.ny * z], L.rho_out);
            }
            // outlet: x=nx-1 from x=nx-2, one lane lower in the same 32-cell group
            if (outlet_fused && x0 + 32 * k <= L.nx - 1 && L.nx - 1 < x0 + 32 * k + 32) {
                float g[Q];
#pragma unroll
                for (int i = 0; i < Q; ++i) g[i] = __shfl_up_sync(0xffffffffu, f[i], 1);
                const uint32_t fm = __shfl_up_sync(0xffffffffu, fk, 1);
                if (x == L.nx - 1 && !(fk & FLAG_SOLID) && !(fm & FLAG_SOLID)) nebb<false>(g, f, 0.f, L.rho_out);
            }
#pragma unroll
            for (int i = 0; i < Q; ++i) outb[i * kSegA + xi] = f[i];
            if (inrow) {
                if constexpr (OUT) {
                    L.rho[c] = R; L.ux[c] = UX; L.uy[c] = UY; L.uz[c] = UZ;
                    if (!(R > 0.f && R < 3.4e38f)) atomicOr(L.status, 1);
                    if constexpr (AVG) {
                        L.avg[c] += UX;
                        L.avg[S + c] += UY;
                        L.avg[2 * S + c] += UZ;
                        L.avg[3 * S + c] += R;
                        L.avg[4 * S + c] += sqrtf(UX * UX + UY * UY + UZ * UZ);
                        L.avg[5 * S + c] += UX * UX;
                    }
                    if constexpr (UCOL) {
                        float sx = k ? csx1 : csx0, sy = k ? csy1 : csy0, sn = k ? ccn1 : ccn0;
                        if (z == 0) { sx = 0.f; sy = 0.f; sn = 0.f; }
                        if (!(fk & FLAG_SOLID)) { sx += UX; sy += UY; sn += 1.f; }
                        if (z == L.nz - 1 && x < L.nx)
                            L.colU[(long long)y * L.pitch + x] = sqrtf(sx * sx + sy * sy) / fmaxf(sn, 1.f);
                        if (k) { csx1 = sx; csy1 = sy; ccn1 = sn; } else { csx0 = sx; csy0 = sy; ccn0 = sn; }
                    }
                } else if (fk & FLAG_WALLFN) {
                    L.rho[c] = R; L.ux[c] = UX; L.uy[c] = UY; L.uz[c] = UZ;
                }
            }
        }
        __syncwarp();                                           // row buffer complete; slot fully read
        {   // write the 19 output rows back, two directions per instruction, 16 bytes per lane
            const int half = lane >> 4, chunk = lane & 15;
            const int xc = x0 + 4 * chunk;
            if (xc < L.pitch) {
                float* dst = fd + (long long)half * S + rowc + xc;
                const float* src = outb + half * kSegA + 4 * chunk;
#pragma unroll
                for (int j = 0; j < (Q + 1) / 2; ++j) {
                    if (2 * j + half < Q)
                        __stcs(reinterpret_cast<float4*>(dst), *reinterpret_cast<const float4*>(src));
                    dst += 2 * S;
                    src += 2 * kSegA;
                }
            }
        }
        __syncwarp();                                           // row buffer read before the next row writes it
        if (++slot_idx == D) slot_idx = 0;
        if (++z == L.nz) { z = 0; item += W; }
    }
    cp_async_wait<0>();
}
