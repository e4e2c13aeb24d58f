// fused_tma.cuh -- TMA-staged, warp-specialized pipeline of the fused step (lbm_tile.pipeline = 1).
// Included inside the anonymous namespace of lbm_kernels.cu.
//
// CTA = C consumer warps + 1 producer warp; a CTA row is T = 32*C consecutive x cells of
// one (y, z) row.  Persistent CTAs take work items (x segment, y) and walk all nz rows of
// each item in turn.
//
// Producer warp (bulk asynchronous copies on the TMA engine, no multicast):
//   * loads: for every row, lane i < 19 copies the T-cell source row of direction i
//     (the row at (y-cy, z-cz), mirrored at the lid; the cell's own opposite direction
//     for rows outside the domain) plus a 16-byte halo each side, and lane 19 the row's
//     T flag words, into slot r % S of a load ring, completing on mbarrier full[slot];
//   * stores: once the consumers have written row r into slot r % SO of an output ring
//     (mbarrier ofull), lane i < 19 copies output row i to global memory; when those
//     copies have read shared memory the slot is handed back (mbarrier oempty).
// Consumer warps: one cell per thread; the 19 pulled populations are read from the load
// slot at x - c_x (compile-time offsets), collided, and written to the output slot.
// Consumers and producer meet only at mbarriers -- there is no CTA-wide barrier in the
// loop.  The inlet/outlet extrapolation uses warp shuffles (x=1 -> x=0, x=nx-2 -> x=nx-1).
//
// Every mbarrier wait is bounded (about one second of clock cycles); a wait that runs
// out sets bit 1 of the status word and the kernel carries on to its end instead of
// hanging the GPU; the producer drains its outstanding bulk stores before exiting.
#pragma once

constexpr long long kWaitCycles = 2000000000LL;   // ~1 s at 1.9 GHz
constexpr int kOutSlots = 2;                      // output ring depth

__device__ __forceinline__ uint32_t smem_addr(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* b, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* b)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(b)) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* b, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(b)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_test(uint64_t* b, uint32_t parity)
{
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(smem_addr(b)), "r"(parity)
        : "memory");
    return done != 0;
}
// Wait for the phase with the given parity to complete; false after `limit` cycles.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* b, uint32_t parity, long long limit)
{
    if (mbar_test(b, parity)) return true;
    const long long t0 = clock64();
    while (!mbar_test(b, parity))
        if (clock64() - t0 > limit) return false;
    return true;
}
// global -> shared bulk copy; both addresses 16-byte aligned, bytes a multiple of 16
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(smem_addr(dst)), "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}
// shared -> global bulk copy (same alignment rules), tracked by the issuing thread's bulk groups
__device__ __forceinline__ void bulk_store(void* dst, const void* src, uint32_t bytes)
{
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;"
                 ::"l"(dst), "r"(smem_addr(src)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void bulk_wait_read() { asm volatile("cp.async.bulk.wait_group.read %0;" ::"n"(N) : "memory"); }
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void fence_mbarrier_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// Shared-memory layout (bytes) for T cells per row, S load slots.
struct TmaLayout {
    int T, S, rowf;           // rowf = floats per staged input row = T + 8
    size_t in_f, in_fl, out_f, bars, bytes;
    __host__ __device__ TmaLayout(int cells, int stages) : T(cells), S(stages), rowf(cells + 8)
    {
        in_f = 0;
        in_fl = in_f + (size_t)S * Q * rowf * sizeof(float);
        out_f = in_fl + (size_t)S * T * sizeof(uint32_t);
        bars = out_f + (size_t)kOutSlots * Q * T * sizeof(float);
        bytes = bars + (size_t)(2 * S + 2 * kOutSlots) * sizeof(uint64_t);
    }
};

// Walks this CTA's rows in order: for each of its work items (x segment, y) -- items
// blockIdx.x, blockIdx.x + gridDim.x, ... -- the rows z = 0 .. nz-1.  32-bit arithmetic,
// one division per item.
struct RowIter {
    int item, seg, y, z;
    __device__ __forceinline__ void start(int nseg)
    {
        item = blockIdx.x; z = 0;
        seg = item % nseg; y = item / nseg;
    }
    __device__ __forceinline__ void next(int nz, int nseg)
    {
        if (++z == nz) {
            z = 0;
            item += gridDim.x;
            seg = item % nseg; y = item / nseg;
        }
    }
};

// Ring position: slot index and the parity of the slot's current fill.
struct Ring {
    int slot, n;
    uint32_t parity;
    __device__ __forceinline__ void start(int slots) { slot = 0; n = slots; parity = 0; }
    __device__ __forceinline__ void next()
    {
        if (++slot == n) { slot = 0; parity ^= 1u; }
    }
};

// Source row (start of the row in fs) of direction i for destination row (y, z).
__device__ __forceinline__ const float* source_row(const lbm_lattice& L, const float* fs, int i, int y, int z)
{
    const int cyi = cy(i), czi = cz(i);
    int ys = y - cyi, zs = z - czi, di = i;
    if (czi == -1 && z == L.nz - 1) { zs = z; di = mirz(i); }     // rigid lid: mirrored population
    if (ys < 0 || ys >= L.ny || zs < 0)                            // outside the domain: own opposite
        return fs + (long long)opp(i) * L.cells + ((long long)z * L.ny + y) * L.pitch;
    return fs + (long long)di * L.cells + ((long long)zs * L.ny + ys) * L.pitch;
}

template <int I, int ROWF>
__device__ __forceinline__ void take_dir(float (&f)[Q], const float* sf, uint32_t rwm)
{
    if constexpr (I == 0) f[0] = sf[0];
    else f[I] = sf[I * ROWF - ((rwm >> I) & 1u ? 0 : cx(I))];
}
template <int ROWF, int... Is>
__device__ __forceinline__ void take_all(std::integer_sequence<int, Is...>, float (&f)[Q], const float* sf, uint32_t rwm)
{
    (take_dir<Is, ROWF>(f, sf, rwm), ...);
}
template <int I, int ROWF>
__device__ __forceinline__ void take_dir_interior(float (&f)[Q], const float* sf)
{
    f[I] = sf[I * ROWF - cx(I)];
}
template <int ROWF, int... Is>
__device__ __forceinline__ void take_all_interior(std::integer_sequence<int, Is...>, float (&f)[Q], const float* sf)
{
    (take_dir_interior<Is, ROWF>(f, sf), ...);
}

template <int C, bool OUT, bool UCOL, bool AVG>
__global__ void __launch_bounds__(32 * (C + 1), C == 8 ? 2 : 1) k_fused_tma(const lbm_lattice L, const float* __restrict__ fs,
                                                            float* __restrict__ fd, int stages, int outlet_fused)
{
    constexpr int T = 32 * C;
    constexpr int ROWF = T + 8;
    extern __shared__ __align__(128) unsigned char smem[];
    const TmaLayout lay(T, stages);
    float* in_f = reinterpret_cast<float*>(smem + lay.in_f);
    uint32_t* in_fl = reinterpret_cast<uint32_t*>(smem + lay.in_fl);
    float* out_f = reinterpret_cast<float*>(smem + lay.out_f);
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + lay.bars);
    uint64_t* ofull = full + stages;
    uint64_t* oempty = ofull + kOutSlots;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nseg = (L.pitch + T - 1) / T;
    const int nitems = nseg * L.ny;
    if ((int)blockIdx.x >= nitems) return;
    const int nrows = ((nitems - 1 - (int)blockIdx.x) / (int)gridDim.x + 1) * L.nz;
    const long long S = L.cells;

    if (threadIdx.x == 0) {
        for (int s = 0; s < stages; ++s) mbar_init(&full[s], 1);
        for (int o = 0; o < kOutSlots; ++o) { mbar_init(&ofull[o], C); mbar_init(&oempty[o], 1); }
        fence_mbarrier_init();
    }
    __syncthreads();

    if (warp == C) {
        // ------------------------------------------------------------------ producer warp
        long long limit = kWaitCycles;
        auto issue_load = [&](const RowIter& id, const Ring& ld) {
            const int x0 = id.seg * T;
            const int lo = x0 >= 4 ? x0 - 4 : 0;
            const int hi = min(x0 + T + 4, L.pitch);
            const uint32_t bytes = (uint32_t)(hi - lo) * 4u;
            const uint32_t fl_bytes = (uint32_t)(min(x0 + T, L.pitch) - x0) * 4u;
            if (lane == 0) mbar_arrive_expect_tx(&full[ld.slot], (uint32_t)Q * bytes + fl_bytes);
            __syncwarp();
            if (lane < Q) {
                float* dst = in_f + ((size_t)ld.slot * Q + lane) * ROWF + (lo - (x0 - 4));
                bulk_load(dst, source_row(L, fs, lane, id.y, id.z) + lo, bytes, &full[ld.slot]);
            } else if (lane == Q) {
                const long long rowc = ((long long)id.z * L.ny + id.y) * L.pitch;
                bulk_load(in_fl + (size_t)ld.slot * T, L.flags + rowc + x0, fl_bytes, &full[ld.slot]);
            }
        };
        RowIter ahead;            // next row to load
        Ring ld;
        ahead.start(nseg);
        ld.start(stages);
        int loaded = 0;
        for (; loaded < stages && loaded < nrows; ++loaded) {
            issue_load(ahead, ld);
            ahead.next(L.nz, nseg);
            ld.next();
        }
        RowIter cur;              // row being stored
        Ring out;
        cur.start(nseg);
        out.start(kOutSlots);
        int prev_slot = -1;
        for (int r = 0; r < nrows; ++r) {
            if (!mbar_wait_bounded(&ofull[out.slot], out.parity, limit)) {
                if (lane == 0) atomicOr(L.status, 2);
                limit = 1000;
            }
            // consumers are done with row r: its load slot takes the next row ahead
            if (loaded < nrows) {
                issue_load(ahead, ld);
                ahead.next(L.nz, nseg);
                ld.next();
                ++loaded;
            }
            const int x0 = cur.seg * T;
            const uint32_t bytes = (uint32_t)(min(x0 + T, L.pitch) - x0) * 4u;
            if (lane < Q) {
                const long long rowc = ((long long)cur.z * L.ny + cur.y) * L.pitch;
                bulk_store(fd + (long long)lane * S + rowc + x0, out_f + ((size_t)out.slot * Q + lane) * T, bytes);
                bulk_commit();
                bulk_wait_read<1>();     // the previous row's stores have read their slot
            }
            __syncwarp();
            if (lane == 0 && prev_slot >= 0) mbar_arrive(&oempty[prev_slot]);
            prev_slot = out.slot;
            cur.next(L.nz, nseg);
            out.next();
        }
        if (lane < Q) bulk_wait_all();
        return;
    }

    // ---------------------------------------------------------------------- consumer warps
    const int tid = threadIdx.x;            // 0 .. T-1
    float csx = 0.f, csy = 0.f, ccn = 0.f;
    long long limit = kWaitCycles;
    RowIter id;
    Ring ld, out;
    id.start(nseg);
    ld.start(stages);
    out.start(kOutSlots);
    for (int r = 0; r < nrows; ++r, id.next(L.nz, nseg), ld.next(), out.next()) {
        const int s = ld.slot, o = out.slot;
        if (!mbar_wait_bounded(&full[s], ld.parity, limit)) {
            atomicOr(L.status, 2);
            limit = 1000;
        }
        const int x0 = id.seg * T;
        const int x = x0 + tid;
        const bool inrow = x < L.pitch;
        const long long rowc = ((long long)id.z * L.ny + id.y) * L.pitch;
        const long long c = rowc + x;
        const uint32_t fk = inrow ? in_fl[(size_t)s * T + tid] : (FLAG_GHOST | FLAG_SOLID);
        const float* sf = in_f + (size_t)s * Q * ROWF + tid + 4;    // this cell's x in every staged row

        float f[Q];
        float R = 1.f, UX = 0.f, UY = 0.f, UZ = 0.f;
        // rows whose pulls all come from inside the domain read every direction shifted by -c_x
        const bool interior = id.y >= 1 && id.y <= L.ny - 2 && id.z >= 1;
        if (interior) {
            take_all_interior<ROWF>(std::make_integer_sequence<int, Q>{}, f, sf);
        } else {
            uint32_t rwm = 0;
#pragma unroll
            for (int i = 1; i < Q; ++i) {
                const int ys = id.y - cy(i), zs = id.z - cz(i);
                if (ys < 0 || ys >= L.ny || (zs < 0)) rwm |= 1u << i;
            }
            take_all<ROWF>(std::make_integer_sequence<int, Q>{}, f, sf, rwm);
        }
        if (fk & FLAG_SOLID) {
#pragma unroll
            for (int i = 0; i < Q; ++i) f[i] = wgt(i);
        } else {
            // solid neighbours inside the domain: bounce back the cell's own opposite population
            uint32_t bb = fk & FLAG_WALLS;
            if (!interior) {
#pragma unroll
                for (int i = 1; i < Q; ++i) {
                    const int ys = id.y - cy(i), zs = id.z - cz(i);
                    if (ys < 0 || ys >= L.ny || zs < 0) bb &= ~(1u << i);
                }
            }
            if (bb) {
#pragma unroll
                for (int i = 1; i < Q; ++i)
                    if (bb & (1u << i)) f[i] = __ldg(fs + (long long)opp(i) * S + c);
            }
            if (x == 0 || x == L.nx - 1) {                  // x edges keep their own population
#pragma unroll
                for (int i = 1; i < Q; ++i)
                    if ((x == 0 && cx(i) == 1) || (x == L.nx - 1 && cx(i) == -1))
                        f[i] = __ldg(fs + (long long)i * S + c);
            }
            if (fk & FLAG_WALLFN) {
                float U;
                if constexpr (UCOL) U = (fk & FLAG_BEDWALL) ? L.colU[(long long)id.y * L.pitch + x] : 0.f;
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

        // inlet: x=0 (lane 0 of warp 0, segment 0) from x=1 (lane 1)
        if (id.seg == 0 && warp == 0) {
            float g[Q];
#pragma unroll
            for (int i = 0; i < Q; ++i) g[i] = __shfl_down_sync(0xffffffffu, f[i], 1);
            const uint32_t f1 = __shfl_down_sync(0xffffffffu, fk, 1);
            if (lane == 0 && !(fk & FLAG_SOLID) && !(f1 & FLAG_SOLID))
                nebb<true>(g, f, L.uin[id.y + (long long)L.ny * id.z], L.rho_out);
        }
        // outlet: x=nx-1 from x=nx-2 (one lane lower, same warp when outlet_fused)
        if (outlet_fused && x0 + 32 * warp <= L.nx - 1 && L.nx - 1 < x0 + 32 * warp + 32) {
            float g[Q];
#pragma unroll
            for (int i = 0; i < Q; ++i) g[i] = __shfl_up_sync(0xffffffffu, f[i], 1);
            const uint32_t fm = __shfl_up_sync(0xffffffffu, fk, 1);
            if (x == L.nx - 1 && !(fk & FLAG_SOLID) && !(fm & FLAG_SOLID)) nebb<false>(g, f, 0.f, L.rho_out);
        }

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
                    if (id.z == 0) { csx = 0.f; csy = 0.f; ccn = 0.f; }
                    if (!(fk & FLAG_SOLID)) { csx += UX; csy += UY; ccn += 1.f; }
                    if (id.z == L.nz - 1 && x < L.nx)
                        L.colU[(long long)id.y * L.pitch + x] = sqrtf(csx * csx + csy * csy) / fmaxf(ccn, 1.f);
                }
            } else if (fk & FLAG_WALLFN) {
                L.rho[c] = R; L.ux[c] = UX; L.uy[c] = UY; L.uz[c] = UZ;
            }
        }

        // output slot o is free once the producer's stores of row r - kOutSlots have read it
        if (r >= kOutSlots && !mbar_wait_bounded(&oempty[o], out.parity ^ 1u, limit)) {
            atomicOr(L.status, 2);
            limit = 1000;
        }
        float* so = out_f + (size_t)o * Q * T + tid;
#pragma unroll
        for (int i = 0; i < Q; ++i) so[i * T] = f[i];
        fence_proxy_async_smem();           // these shared stores are read next by the async proxy
        __syncwarp();
        if (lane == 0) mbar_arrive(&ofull[o]);
    }
}
