// fused_tma.cuh -- TMA-staged pipeline of the fused step (lbm_tile.pipeline = 1).
// Included inside the anonymous namespace of lbm_kernels.cu.
//
// A CTA of T = 32*warps threads owns a run of rows: for each work item (x segment of
// T cells, y) all nz rows in turn.  For every row, one thread issues 20 bulk
// asynchronous copies (cp.async.bulk, the TMA engine; no multicast) into a ring of
// `stages` shared-memory slots:
//   * for each direction i, the T-cell source row of the pull (the row at (y-cy, z-cz),
//     mirrored at the lid; the cell's own opposite direction for rows outside the
//     domain), widened by a 16-byte halo on each side;
//   * the row's T flag words.
// Completion is tracked by one mbarrier per slot (expect_tx = total bytes), so the
// copies for `stages-1` rows ahead are in flight while the threads collide the
// current one.  Each thread owns one cell: it reads its 19 pulled populations from
// shared memory at offset x - c_x (no shuffles, no alignment constraint), collides,
// and writes 19 coalesced 4-byte stores.  Inlet/outlet extrapolation exchanges the
// x=1 / x=nx-2 post-collision populations through shared memory.
//
// Every mbarrier wait is bounded (about one second of clock cycles); a wait that runs
// out sets bit 1 of the status word and the kernel carries on and returns, instead of
// hanging the GPU.
#pragma once

constexpr long long kWaitCycles = 2000000000LL;   // ~1 s at 1.9 GHz

__device__ __forceinline__ uint32_t smem_addr(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* b, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(b)), "r"(count) : "memory");
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
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* b, uint32_t parity, long long limit)
{
    if (mbar_test(b, parity)) return true;
    const long long t0 = clock64();
    while (!mbar_test(b, parity))
        if (clock64() - t0 > limit) return false;
    return true;
}
// global -> shared bulk copy; dst, src 16-byte aligned, bytes a multiple of 16
__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(smem_addr(dst)), "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void fence_mbarrier_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// Shared-memory layout of k_fused_tma (bytes), for T threads and S stages.
struct TmaLayout {
    int T, S, rowf;           // rowf = floats per staged row = T + 8
    size_t f_off, fl_off, bc_off, bar_off, bytes;
    __host__ __device__ TmaLayout(int threads, int stages) : T(threads), S(stages), rowf(threads + 8)
    {
        f_off = 0;
        fl_off = f_off + (size_t)S * Q * rowf * sizeof(float);
        bc_off = fl_off + (size_t)S * T * sizeof(uint32_t);
        bar_off = bc_off + (size_t)2 * 2 * Q * sizeof(float);
        bytes = bar_off + (size_t)S * sizeof(uint64_t);
    }
};

struct RowId {
    int seg, y, z;
};

__device__ __forceinline__ RowId row_of(long long r, int nz, int nseg)
{
    const long long item = blockIdx.x + (r / nz) * (long long)gridDim.x;
    return RowId{(int)(item % nseg), (int)(item / nseg), (int)(r % nz)};
}

template <int I>
__device__ __forceinline__ void issue_dir(const lbm_lattice& L, const float* fs, float* sf_row, long long rowc,
                                          int y, int z, int lo, uint32_t bytes, uint64_t* bar)
{
    constexpr int CYI = cy(I), CZI = cz(I);
    int ys = y - CYI, zs = z - CZI, di = I;
    if (CZI == -1 && z == L.nz - 1) { zs = z; di = mirz(I); }
    const bool rowwall = (ys < 0) || (ys >= L.ny) || (zs < 0);
    const float* row = rowwall ? fs + (long long)opp(I) * L.cells + rowc
                               : fs + (long long)di * L.cells + ((long long)zs * L.ny + ys) * L.pitch;
    bulk_copy_g2s(sf_row, row + lo, bytes, bar);
}
template <int... Is>
__device__ __forceinline__ void issue_all(std::integer_sequence<int, Is...>, const lbm_lattice& L, const float* fs,
                                          float* sf, int rowf, int dst_off, long long rowc, int y, int z, int lo,
                                          uint32_t bytes, uint64_t* bar)
{
    (issue_dir<Is>(L, fs, sf + Is * rowf + dst_off, rowc, y, z, lo, bytes, bar), ...);
}

template <int I>
__device__ __forceinline__ void take_dir(float (&f)[Q], uint32_t& rwm, const lbm_lattice& L, const float* sf,
                                         int rowf, int sx, int y, int z)
{
    constexpr int CXI = cx(I), CYI = cy(I), CZI = cz(I);
    if constexpr (I == 0) {
        f[0] = sf[sx];
    } else {
        int ys = y - CYI, zs = z - CZI;
        if (CZI == -1 && z == L.nz - 1) zs = z;
        const bool rowwall = (ys < 0) || (ys >= L.ny) || (zs < 0);
        f[I] = sf[I * rowf + sx - (rowwall ? 0 : CXI)];
        rwm |= rowwall ? (1u << I) : 0u;
    }
}
template <int... Is>
__device__ __forceinline__ void take_all(std::integer_sequence<int, Is...>, float (&f)[Q], uint32_t& rwm,
                                         const lbm_lattice& L, const float* sf, int rowf, int sx, int y, int z)
{
    (take_dir<Is>(f, rwm, L, sf, rowf, sx, y, z), ...);
}

template <bool OUT, bool UCOL, bool AVG>
__global__ void __launch_bounds__(256, 2) k_fused_tma(const lbm_lattice L, const float* __restrict__ fs,
                                                      float* __restrict__ fd, int stages, int outlet_fused)
{
    extern __shared__ __align__(128) unsigned char smem[];
    const int T = blockDim.x, tid = threadIdx.x;
    const TmaLayout lay(T, stages);
    float* stage_f = reinterpret_cast<float*>(smem + lay.f_off);
    uint32_t* stage_fl = reinterpret_cast<uint32_t*>(smem + lay.fl_off);
    float* bcx = reinterpret_cast<float*>(smem + lay.bc_off);        // [row parity][inlet/outlet][Q]
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + lay.bar_off);
    const int rowf = lay.rowf;

    const int nseg = (L.pitch + T - 1) / T;
    const long long nitems = (long long)nseg * L.ny;
    if ((long long)blockIdx.x >= nitems) return;
    const long long my_items = (nitems - 1 - blockIdx.x) / gridDim.x + 1;
    const long long nrows = my_items * L.nz;
    const long long S = L.cells;

    if (tid == 0) {
        for (int s = 0; s < stages; ++s) mbar_init(&bars[s], 1);
        fence_mbarrier_init();
    }
    __syncthreads();

    auto issue = [&](long long r) {   // one thread: stage row r into slot r % stages
        const RowId id = row_of(r, L.nz, nseg);
        const int s = (int)(r % stages);
        const int x0 = id.seg * T;
        const int lo = x0 >= 4 ? x0 - 4 : 0;
        const int hi = min(x0 + T + 4, L.pitch);
        const uint32_t bytes = (uint32_t)(hi - lo) * 4u;
        const uint32_t fl_bytes = (uint32_t)(min(x0 + T, L.pitch) - x0) * 4u;
        const long long rowc = ((long long)id.z * L.ny + id.y) * L.pitch;
        mbar_arrive_expect_tx(&bars[s], (uint32_t)Q * bytes + fl_bytes);
        issue_all(std::make_integer_sequence<int, Q>{}, L, fs, stage_f + (size_t)s * Q * rowf, rowf,
                  lo - (x0 - 4), rowc, id.y, id.z, lo, bytes, &bars[s]);
        bulk_copy_g2s(stage_fl + (size_t)s * T, L.flags + rowc + x0, fl_bytes, &bars[s]);
    };

    if (tid == 0)
        for (long long q = 0; q < stages - 1 && q < nrows; ++q) issue(q);

    float csx = 0.f, csy = 0.f, ccn = 0.f;
    long long limit = kWaitCycles;
    for (long long r = 0; r < nrows; ++r) {
        if (tid == 0 && r + stages - 1 < nrows) {
            fence_proxy_async_smem();        // earlier generic reads of the slot before the async refill
            issue(r + stages - 1);
        }
        const RowId id = row_of(r, L.nz, nseg);
        const int s = (int)(r % stages);
        if (!mbar_wait_bounded(&bars[s], (uint32_t)((r / stages) & 1), limit)) {
            atomicOr(L.status, 2);
            limit = 1000;                    // after one timeout, do not wait long again
        }
        const int x = id.seg * T + tid;
        const bool inrow = x < L.pitch;
        const long long rowc = ((long long)id.z * L.ny + id.y) * L.pitch;
        const long long c = rowc + x;
        const float* sf = stage_f + (size_t)s * Q * rowf;
        const uint32_t fk = inrow ? stage_fl[(size_t)s * T + tid] : (FLAG_GHOST | FLAG_SOLID);
        const int par = (int)(r & 1);
        // flags of x=1 and x=nx-2, needed by the boundary threads after the slot is released
        const bool in_bc = (x == 0) && !(fk & FLAG_SOLID) && !(stage_fl[(size_t)s * T + 1] & FLAG_SOLID);
        const bool out_bc = outlet_fused && (x == L.nx - 1) && !(fk & FLAG_SOLID) &&
                            !(stage_fl[(size_t)s * T + tid - 1] & FLAG_SOLID);

        float f[Q];
        float R = 1.f, UX = 0.f, UY = 0.f, UZ = 0.f;
        if (fk & FLAG_SOLID) {
#pragma unroll
            for (int i = 0; i < Q; ++i) f[i] = wgt(i);
        } else {
            uint32_t rwm = 0;
            take_all(std::make_integer_sequence<int, Q>{}, f, rwm, L, sf, rowf, tid + 4, id.y, id.z);
            const uint32_t bb = fk & FLAG_WALLS & ~rwm;
            if (bb) {                                                   // solid neighbours: bounce back
#pragma unroll
                for (int i = 1; i < Q; ++i)
                    if (bb & (1u << i)) f[i] = __ldg(fs + (long long)opp(i) * S + c);
            }
            if (x == 0) {                                               // x edges keep their own population
#pragma unroll
                for (int i = 1; i < Q; ++i)
                    if (cx(i) == 1) f[i] = __ldg(fs + (long long)i * S + c);
            }
            if (x == L.nx - 1) {
#pragma unroll
                for (int i = 1; i < Q; ++i)
                    if (cx(i) == -1) f[i] = __ldg(fs + (long long)i * S + c);
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

        // boundary exchange: x=1 and x=nx-2 publish their post-collision populations
        if (x == 1) {
#pragma unroll
            for (int i = 0; i < Q; ++i) bcx[(par * 2 + 0) * Q + i] = f[i];
        }
        if (outlet_fused && x == L.nx - 2) {
#pragma unroll
            for (int i = 0; i < Q; ++i) bcx[(par * 2 + 1) * Q + i] = f[i];
        }
        if (inrow && !in_bc && !out_bc) {
#pragma unroll
            for (int i = 0; i < Q; ++i) __stcs(fd + (long long)i * S + c, f[i]);
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
        __syncthreads();                    // slot s and this row's exchange buffer are complete
        if (in_bc) {
            float g[Q];
#pragma unroll
            for (int i = 0; i < Q; ++i) g[i] = bcx[(par * 2 + 0) * Q + i];
            nebb<true>(g, f, L.uin[id.y + (long long)L.ny * id.z], L.rho_out);
#pragma unroll
            for (int i = 0; i < Q; ++i) __stcs(fd + (long long)i * S + c, f[i]);
        }
        if (out_bc) {
            float g[Q];
#pragma unroll
            for (int i = 0; i < Q; ++i) g[i] = bcx[(par * 2 + 1) * Q + i];
            nebb<false>(g, f, 0.f, L.rho_out);
#pragma unroll
            for (int i = 0; i < Q; ++i) __stcs(fd + (long long)i * S + c, f[i]);
        }
    }
}
