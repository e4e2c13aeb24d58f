// fused_split.cuh -- work-list pipeline of the fused step (lbm_tile.pipeline = 3).
// Included inside the anonymous namespace of lbm_kernels.cu, after fused_reg.cuh.
//
// The lattice is cut into row segments of 32*V cells (V = 4: 128 cells).  Once per
// geometry (lbm_build_worklists) every segment is classified and compacted, in order,
// into one of three lists:
//   plain   -- interior row (1 <= y <= ny-2, 1 <= z <= nz-2), clear of the x edges and of
//              padding, no cell solid, walled, forced or under the wall function;
//   solid   -- every cell solid (or padding);
//   special -- everything else (walls, bed, lid, banks, hulls, forcing, inlet, outlet).
// A step then runs
//   k_rows<PLAIN>   over the plain list: 19 V-wide pulls at constant offsets (the +-1 x
//                   neighbours by warp shuffle), collision with no force, 19 V-wide
//                   streaming stores -- no flag word is read; this is where the cells are;
//   k_rows<SPECIAL> over the special list: the general path of fused_reg.cuh (flag words,
//                   y-wall/bed/lid rows, bounce-back, x edges, wall function, forcing,
//                   inlet/outlet), compiled separately so its register needs do not
//                   throttle the plain kernel;
//   k_solid_out     on output steps only: the fields of solid segments;
//   k_column_mean   on output steps with the column-mean wall model: the depth-mean speed
//                   of every (y, x) column, summed over z in order.
// Solid segments move no populations: solid cells are never read and both population
// buffers hold their rest state from the start.
#pragma once

// Row-segment id: (z * ny + y) * nseg + seg.
__device__ __forceinline__ void decode_row(uint32_t id, int nseg, int ny, int& seg, int& y, int& z)
{
    seg = (int)(id % (uint32_t)nseg);
    const uint32_t yz = id / (uint32_t)nseg;
    y = (int)(yz % (uint32_t)ny);
    z = (int)(yz / (uint32_t)ny);
}

// 0 plain, 1 solid, 2 special (see the file comment); one thread per segment.
__global__ void k_classify(const lbm_lattice L, int V, uint8_t* __restrict__ cls)
{
    const int SEG = 32 * V;
    const int nseg = (L.pitch + SEG - 1) / SEG;
    const long long n = (long long)nseg * L.ny * L.nz;
    const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= n) return;
    const int seg = (int)(id % nseg);
    const long long yz = id / nseg;
    const int y = (int)(yz % L.ny), z = (int)(yz / L.ny);
    const long long rowc = ((long long)z * L.ny + y) * L.pitch;
    const int xa = seg * SEG, xb = min(xa + SEG, L.pitch);
    bool all_solid = true, any_special = false;
    for (int x = xa; x < xb; ++x) {
        const uint32_t fk = L.flags[rowc + x];
        all_solid &= (fk & FLAG_SOLID) != 0;
        any_special |= (fk & (FLAG_SOLID | FLAG_WALLS | FLAG_WALLFN | FLAG_FORCE)) != 0;
    }
    const bool interior = y >= 1 && y <= L.ny - 2 && z >= 1 && z <= L.nz - 2 && seg > 0 && xa + SEG < L.nx;
    cls[id] = all_solid ? 1 : (interior && !any_special ? 0 : 2);
}

// Ordered stream compaction of the three classes by one CTA (one-time set-up work).
// counts[c] receives the number of segments of class c; lists[c] their ids in order.
__global__ void __launch_bounds__(1024) k_compact(const uint8_t* __restrict__ cls, long long n,
                                                  uint32_t* __restrict__ plain, uint32_t* __restrict__ solid,
                                                  uint32_t* __restrict__ special, int* __restrict__ counts)
{
    __shared__ int warp_tot[3][32];
    __shared__ int base[3];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid < 3) base[tid] = 0;
    __syncthreads();
    for (long long start = 0; start < n; start += blockDim.x) {
        const long long i = start + tid;
        const int c = i < n ? cls[i] : 3;
        int rank[3], tot_before[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const unsigned m = __ballot_sync(0xffffffffu, c == k);
            rank[k] = __popc(m & ((1u << lane) - 1u));
            if (lane == 0) warp_tot[k][warp] = __popc(m);
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            int acc = 0;
            for (int w = 0; w < warp; ++w) acc += warp_tot[k][w];
            tot_before[k] = acc;
        }
        if (c < 3) {
            uint32_t* dst = c == 0 ? plain : (c == 1 ? solid : special);
            dst[base[c] + tot_before[c] + rank[c]] = (uint32_t)i;
        }
        __syncthreads();
        if (tid < 3) {
            int sum = 0;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) sum += warp_tot[tid][w];
            base[tid] += sum;
        }
        __syncthreads();
    }
    if (tid < 3) counts[tid] = base[tid];
}

template <int V, bool PLAIN, bool OUT, bool UCOL, bool AVG>
__global__ void __launch_bounds__(128, PLAIN ? 3 : 2) k_rows(const lbm_lattice L, const PullOffsets po,
                                                             const uint32_t* __restrict__ list, int nlist,
                                                             const float* __restrict__ fs, float* __restrict__ fd)
{
    constexpr int SEG = 32 * V;
    const int lane = threadIdx.x & 31;
    const int gw = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), W = (int)((gridDim.x * blockDim.x) >> 5);
    const int nseg = (L.pitch + SEG - 1) / SEG;
    const long long S = L.cells;
    uint32_t next = gw < nlist ? __ldg(list + gw) : 0u;          // list entries are fetched one ahead
    for (int w = gw; w < nlist; w += W) {
        const uint32_t id = next;
        if (w + W < nlist) next = __ldg(list + w + W);
        int seg, y, z;
        decode_row(id, nseg, L.ny, seg, y, z);
        const int x0 = seg * SEG + lane * V;
        const long long rowc = ((long long)z * L.ny + y) * L.pitch;
        const long long own = rowc + x0;
        float f[V][Q];
        float R[V], UX[V], UY[V], UZ[V];
        bool active = true;
        if constexpr (PLAIN) {
            pull_fast_all<V>(std::make_integer_sequence<int, Q>{}, f, fs + own, po, lane);
#pragma unroll
            for (int k = 0; k < V; ++k) collide(f[k], 0.f, 0.f, 0.f, L.tau0, L.csmag2, R[k], UX[k], UY[k], UZ[k]);
        } else {
            active = x0 < L.pitch;
            const int x0c = active ? x0 : L.pitch - V;
            PullCtx pc{fs, S, rowc, rowc + x0c, x0, x0c, y, z, lane};
            uint32_t fl[V];
            Vec<V>::loadu(fl, L.flags + pc.own);
            const bool interior = y >= 1 && y <= L.ny - 2 && z >= 1 && z <= L.nz - 2;
            uint32_t rwm = 0;
            if (interior) pull_fast_all<V>(std::make_integer_sequence<int, Q>{}, f, fs + pc.own, po, lane);
            else rwm = pull_rows<V>(std::make_integer_sequence<int, Q>{}, f, L, pc);
            uint32_t flany = 0;
#pragma unroll
            for (int k = 0; k < V; ++k) {
                if (!active) fl[k] = FLAG_GHOST | FLAG_SOLID;
                flany |= fl[k];
            }
            pull_fixups<V>(std::make_integer_sequence<int, Q>{}, f, L, pc, fl, flany & FLAG_WALLS & ~rwm);
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
            if (!OUT && active) {                                // the wall function reads these next step
#pragma unroll
                for (int k = 0; k < V; ++k)
                    if (fl[k] & FLAG_WALLFN) {
                        L.rho[own + k] = R[k]; L.ux[own + k] = UX[k]; L.uy[own + k] = UY[k]; L.uz[own + k] = UZ[k];
                    }
            }
            if (OUT && active) {
                bool bad = false;
#pragma unroll
                for (int k = 0; k < V; ++k) bad |= !(fl[k] & FLAG_SOLID) && !(R[k] > 0.f && R[k] < 3.4e38f);
                if (bad) atomicOr(L.status, 1);
            }
        }
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
                if constexpr (PLAIN) {
                    bool bad = false;
#pragma unroll
                    for (int k = 0; k < V; ++k) bad |= !(R[k] > 0.f && R[k] < 3.4e38f);
                    if (bad) atomicOr(L.status, 1);
                }
                if constexpr (AVG) {
                    float a[V], s[V];
#define WFS_ACC(M, EXPR)                                                   \
                    vload_plain<V>(a, L.avg + (long long)(M) * S + own);     \
                    _Pragma("unroll") for (int k = 0; k < V; ++k) {         \
                        s[k] = a[k] + (EXPR);                               \
                    }                                                       \
                    vstore_plain<V>(L.avg + (long long)(M) * S + own, s);
                    WFS_ACC(0, UX[k])
                    WFS_ACC(1, UY[k])
                    WFS_ACC(2, UZ[k])
                    WFS_ACC(3, R[k])
                    WFS_ACC(4, sqrtf(UX[k] * UX[k] + UY[k] * UY[k] + UZ[k] * UZ[k]))
                    WFS_ACC(5, UX[k] * UX[k])
#undef WFS_ACC
                }
            }
        }
    }
}

// Output step: fields of solid segments (rho = 1, u = 0) and their time-average sums.
template <int V, bool AVG>
__global__ void k_solid_out(const lbm_lattice L, const uint32_t* __restrict__ list, int nlist)
{
    constexpr int SEG = 32 * V;
    const int lane = threadIdx.x & 31;
    const int gw = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), W = (int)((gridDim.x * blockDim.x) >> 5);
    const int nseg = (L.pitch + SEG - 1) / SEG;
    const long long S = L.cells;
    for (int w = gw; w < nlist; w += W) {
        int seg, y, z;
        decode_row(__ldg(list + w), nseg, L.ny, seg, y, z);
        const int x0 = seg * SEG + lane * V;
        if (x0 >= L.pitch) continue;
        const long long own = ((long long)z * L.ny + y) * L.pitch + x0;
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

// Depth-mean speed of every (y, x) column (floodsim/reach3d.py:412-417): the sums of ux and
// uy over the column's fluid cells, taken in z order, then sqrt(sx^2 + sy^2) / n.
__global__ void k_column_mean(const lbm_lattice L)
{
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;   // x + pitch * y
    if (q >= (long long)L.ny * L.pitch) return;
    const int x = (int)(q % L.pitch);
    if (x >= L.nx) return;
    const long long plane = (long long)L.ny * L.pitch;
    float sx = 0.f, sy = 0.f, n = 0.f;
    for (int z = 0; z < L.nz; ++z) {
        const long long c = q + plane * z;
        if (!(L.flags[c] & FLAG_SOLID)) { sx += L.ux[c]; sy += L.uy[c]; n += 1.f; }
    }
    L.colU[q] = sqrtf(sx * sx + sy * sy) / fmaxf(n, 1.f);
}
