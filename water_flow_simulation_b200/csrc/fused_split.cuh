// fused_split.cuh -- work-list pipeline of the fused step (lbm_tile.pipeline = 3).
// Included inside the anonymous namespace of lbm_kernels.cu, after fused_reg.cuh.
//
// The lattice is cut into row segments of 32*V cells (V = 4: 128 cells).  Once per
// geometry (lbm_build_worklists) every segment is classified and compacted, in order,
// into one of four lists:
//   plain   -- open row (1 <= y <= ny-2, 1 <= z <= nz-1: the row under the lid included),
//              clear of the x edges and of padding, no cell solid, walled, forced or under
//              the wall function;
//   edge    -- the same, except that the segment holds x = 0 (inlet) or x = nx-1 (outlet)
//              and possibly padding: the first and last segment of an open row;
//   solid   -- every cell solid (or padding);
//   special -- everything else (walls, bed, lid, banks, hulls, forcing).
// A step then runs
//   k_rows<PLAIN>   over the plain list: 19 V-wide pulls at constant offsets (the +-1 x
//                   neighbours by warp shuffle), collision with no force, 19 V-wide
//                   streaming stores -- no flag word is read; this is where the cells are;
//   k_rows_edge     over the edge list: the plain pull, the x-edge copies, the inlet and
//                   outlet extrapolation and rest-state padding, still without flag words;
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

// 0 plain, 1 solid, 2 special, 3 edge (see the file comment); one thread per segment.
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
        if (x < L.nx) any_special |= (fk & (FLAG_SOLID | FLAG_WALLS | FLAG_WALLFN | FLAG_FORCE)) != 0;
    }
    // open rows: clear of the y walls and the bed; the row under the lid counts (its -z movers
    // read the own row's mirrored populations at constant offsets)
    if (L.sponge_cols > 0 && xb > L.nx - L.sponge_cols) any_special = true;   // per-cell relaxation time
    const bool interior_row = y >= 1 && y <= L.ny - 2 && z >= 1 && z <= L.nz - 1;
    const bool clear_of_edges = seg > 0 && xa + SEG < L.nx;
    int c = 2;
    if (all_solid) c = 1;
    else if (interior_row && !any_special) c = clear_of_edges ? 0 : 3;
    cls[id] = (uint8_t)c;
}

// Ordered stream compaction of the four classes by one CTA (one-time set-up work).
// counts[c] receives the number of segments of class c; lists[c] their ids in order.
__global__ void __launch_bounds__(1024) k_compact(const uint8_t* __restrict__ cls, long long n,
                                                  uint32_t* __restrict__ plain, uint32_t* __restrict__ solid,
                                                  uint32_t* __restrict__ special, uint32_t* __restrict__ edge,
                                                  int* __restrict__ counts)
{
    constexpr int NC = 4;
    __shared__ int warp_tot[NC][32];
    __shared__ int base[NC];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid < NC) base[tid] = 0;
    __syncthreads();
    uint32_t* const lists[NC] = {plain, solid, special, edge};
    for (long long start = 0; start < n; start += blockDim.x) {
        const long long i = start + tid;
        const int c = i < n ? cls[i] : NC;
        int rank[NC], tot_before[NC];
#pragma unroll
        for (int k = 0; k < NC; ++k) {
            const unsigned m = __ballot_sync(0xffffffffu, c == k);
            rank[k] = __popc(m & ((1u << lane) - 1u));
            if (lane == 0) warp_tot[k][warp] = __popc(m);
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < NC; ++k) {
            int acc = 0;
            for (int w = 0; w < warp; ++w) acc += warp_tot[k][w];
            tot_before[k] = acc;
        }
#pragma unroll
        for (int k = 0; k < NC; ++k)
            if (c == k) lists[k][base[k] + tot_before[k] + rank[k]] = (uint32_t)i;
        __syncthreads();
        if (tid < NC) {
            int sum = 0;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) sum += warp_tot[tid][w];
            base[tid] += sum;
        }
        __syncthreads();
    }
    if (tid < NC) counts[tid] = base[tid];
}

// Streaming stores of the V cells' 19 populations (T = float or 16-bit storage).
template <int I, int V, typename T>
__device__ __forceinline__ void store_pop(T* p, const float (&f)[V][Q], float scale)
{
    float v[V];
#pragma unroll
    for (int k = 0; k < V; ++k) v[k] = f[k][I];
    stv<I, V>(p, v, scale);
}
template <int V, typename T, int... Is>
__device__ __forceinline__ void store_pops(std::integer_sequence<int, Is...>, T* fd, long long S, long long own,
                                           const float (&f)[V][Q], float scale)
{
    (store_pop<Is, V>(fd + (long long)Is * S + own, f, scale), ...);
}

// Output-step fields of V cells and, with AVG, their time-average sums
// (floodsim/reach3d.py:443-451: ux, uy, uz, rho, speed, ux^2).
template <int V, bool AVG>
__device__ __forceinline__ void store_fields(const lbm_lattice& L, long long own, const float (&R)[V],
                                             const float (&UX)[V], const float (&UY)[V], const float (&UZ)[V])
{
    const long long S = L.cells;
    vstore_plain<V>(L.rho + own, R);
    vstore_plain<V>(L.ux + own, UX);
    vstore_plain<V>(L.uy + own, UY);
    vstore_plain<V>(L.uz + own, UZ);
    if constexpr (AVG) {
        if (!L.avg) return;                // a batched lattice outside its averaging window
        float a[V], s[V];
#define WFS_ACC(M, EXPR)                                                   \
        vload_plain<V>(a, L.avg + (long long)(M) * S + own);               \
        _Pragma("unroll") for (int k = 0; k < V; ++k) {                   \
            s[k] = a[k] + (EXPR);                                         \
        }                                                                 \
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

// Outlet cell x = nx-1 as the first cell of a lane whose left neighbour lane holds x = nx-2:
// that lane's post-collision populations arrive by shuffle, so the extrapolation uses the
// same unrounded values as when both cells share a lane.  (When x = nx-2 is in the previous
// segment -- nx-1 a multiple of the segment length -- a separate pass does it.)  Called by
// all lanes of the warp.
template <int V>
__device__ __forceinline__ void outlet_from_left_lane(float (&f)[V][Q], const lbm_lattice& L, int x0, int lane,
                                                      bool own_solid, bool last_solid)
{
    const bool here = x0 == L.nx - 1 && lane > 0;
    if (!__any_sync(0xffffffffu, here)) return;
    float g[Q];
#pragma unroll
    for (int i = 0; i < Q; ++i) g[i] = __shfl_up_sync(0xffffffffu, f[V - 1][i], 1);
    const bool left_solid = __shfl_up_sync(0xffffffffu, last_solid, 1);
    if (here && !own_solid && !left_solid) nebb<false>(g, f[0], 0.f, L.rho_out);
}

// Relaxation time at zero strain of column x: tau0, or inside the optional outlet sponge
// tau0 + (sponge_tau - tau0) s^2 (explicitly rounded, so every kernel computes the same value).
__device__ __forceinline__ float sponge_tau0(const lbm_lattice& L, int x)
{
    const int x0 = L.nx - L.sponge_cols;
    if (L.sponge_cols <= 0 || x < x0) return L.tau0;
    const float s = __fdiv_rn((float)(x - x0 + 1), (float)L.sponge_cols);
    return __fadd_rn(L.tau0, __fmul_rn(__fsub_rn(L.sponge_tau, L.tau0), __fmul_rn(s, s)));
}

// The general path for the V cells from x0 of row (y, z): flag words, y-wall/bed/lid rows,
// bounce-back, x edges, wall function, forcing, inlet/outlet, then the stores.  T is the
// population element type; `scale` / `inv_scale` are the 16-bit storage scale and its inverse.
template <int V, bool OUT, bool UCOL, bool AVG, typename T>
__device__ __forceinline__ void general_segment(const lbm_lattice& L, const PullOffsets& po, const T* __restrict__ fs,
                                                T* __restrict__ fd, float scale, float inv_scale, int x0, int y, int z,
                                                int lane)
{
    const long long S = L.cells;
    const long long rowc = ((long long)z * L.ny + y) * L.pitch;
    const long long own = rowc + x0;
    float f[V][Q];
    float R[V], UX[V], UY[V], UZ[V];
    const bool active = x0 < L.pitch;
    const int x0c = active ? x0 : L.pitch - V;
    PullCtxT<T> pc{fs, S, rowc, rowc + x0c, x0, x0c, y, z, lane};
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
    raw_to_pop<T, V>(f, inv_scale);
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
            collide(f[k], fx, fy, fz, sponge_tau0(L, x0 + k), L.csmag2, R[k], UX[k], UY[k], UZ[k]);
        }
    }
    // inlet (x=0 from x=1) and outlet (x=nx-1 from x=nx-2), both inside this lane
    if (x0 == 0 && !(fl[0] & FLAG_SOLID) && !(fl[1] & FLAG_SOLID))
        nebb<true>(f[1], f[0], L.uin[y + (long long)L.ny * z], L.rho_out);
#pragma unroll
    for (int k = 1; k < V; ++k)
        if (x0 + k == L.nx - 1 && !(fl[k] & FLAG_SOLID) && !(fl[k - 1] & FLAG_SOLID))
            nebb<false>(f[k - 1], f[k], 0.f, L.rho_out);
    outlet_from_left_lane<V>(f, L, x0, lane, (fl[0] & FLAG_SOLID) != 0, (fl[V - 1] & FLAG_SOLID) != 0);
    if (!active) return;
    if constexpr (!OUT) {                                 // the wall function reads these next step
#pragma unroll
        for (int k = 0; k < V; ++k)
            if (fl[k] & FLAG_WALLFN) {
                L.rho[own + k] = R[k]; L.ux[own + k] = UX[k]; L.uy[own + k] = UY[k]; L.uz[own + k] = UZ[k];
            }
    } else {
        bool bad = false;
#pragma unroll
        for (int k = 0; k < V; ++k) bad |= !(fl[k] & FLAG_SOLID) && !(R[k] > 0.f && R[k] < 3.4e38f);
        if (bad) atomicOr(L.status, 1);
    }
    store_pops<V>(std::make_integer_sequence<int, Q>{}, fd, S, own, f, scale);
    if constexpr (OUT) store_fields<V, AVG>(L, own, R, UX, UY, UZ);
}

// Special list: each list segment of PASSES*32*V cells in PASSES warp passes through the
// general path.
// Occupancy: the 16-bit V = 2 variant fits 128 registers without spills, so 4 CTAs (16 warps)
// per SM hide more of its dependent flag -> pull -> wall-function latency (9.6 % less time for
// the special segments of reach36m than at 3 CTAs); the float32 one would spill there.
template <int V, int PASSES, bool OUT, bool UCOL, bool AVG, typename T>
__global__ void __launch_bounds__(128, V <= 2 ? (std::is_same<T, __half>::value ? 4 : 3) : 2)
    k_general(const lbm_lattice L, const PullOffsets po,
                                                    const uint32_t* __restrict__ list, int nlist,
                                                    const T* __restrict__ fs, T* __restrict__ fd, float scale)
{
    constexpr int SEG = PASSES * 32 * V, PASS = 32 * V;
    const int lane = threadIdx.x & 31;
    const int gw = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), W = (int)((gridDim.x * blockDim.x) >> 5);
    const int nseg = (L.pitch + SEG - 1) / SEG;
    const float inv_scale = 1.0f / scale;
    uint32_t next = gw < nlist ? __ldg(list + gw) : 0u;          // list entries are fetched one ahead
    for (int w = gw; w < nlist; w += W) {
        const uint32_t id = next;
        if (w + W < nlist) next = __ldg(list + w + W);
        int seg, y, z;
        decode_row(id, nseg, L.ny, seg, y, z);
#pragma unroll 1
        for (int part = 0; part < PASSES; ++part) {
            const int xa = seg * SEG + part * PASS;
            if (xa >= L.pitch) break;                                  // warp-uniform
            general_segment<V, OUT, UCOL, AVG, T>(L, po, fs, fd, scale, inv_scale, xa + lane * V, y, z, lane);
        }
    }
}

// Edge segment (first or last of an open interior row, no flags set below nx): the plain pull,
// then the x-edge copies (a direction whose source lies outside [0, nx) keeps the cell's own
// population, floodsim/lbm3d.py:48-49), collision without force, the inlet at x = 0 and the
// outlet at x = nx-1 (when x = nx-2 is in the same lane), and padding cells (x >= nx) held at
// rest.  Loads stay inside the population array: an interior row has rows on both sides.
template <int V, bool OUT, bool AVG, typename T>
__device__ __forceinline__ void edge_segment(const lbm_lattice& L, const PullOffsets& po, const T* __restrict__ fs,
                                             T* __restrict__ fd, float scale, float inv_scale, int x0, int y, int z,
                                             int lane)
{
    const long long S = L.cells;
    const long long rowc = ((long long)z * L.ny + y) * L.pitch;
    const bool active = x0 < L.pitch;
    const int x0c = active ? x0 : L.pitch - V;
    const long long own = rowc + x0c;
    float f[V][Q];
    float R[V], UX[V], UY[V], UZ[V];
    pull_fast_all<V>(std::make_integer_sequence<int, Q>{}, f, fs + own, po, lane, z == L.nz - 1);
    PullCtxT<T> pc{fs, S, rowc, own, x0, x0c, y, z, lane};
    const bool edge = (x0 == 0) || (x0 <= L.nx - 1 && L.nx - 1 < x0 + V);
    if (edge) pull_edges<V>(std::make_integer_sequence<int, Q>{}, f, L, pc);
    raw_to_pop<T, V>(f, inv_scale);
#pragma unroll
    for (int k = 0; k < V; ++k) {
        if (x0 + k >= L.nx) {
#pragma unroll
            for (int i = 0; i < Q; ++i) f[k][i] = wgt(i);
            R[k] = 1.f; UX[k] = 0.f; UY[k] = 0.f; UZ[k] = 0.f;
        } else {
            collide(f[k], 0.f, 0.f, 0.f, L.tau0, L.csmag2, R[k], UX[k], UY[k], UZ[k]);
        }
    }
    if (x0 == 0) nebb<true>(f[1], f[0], L.uin[y + (long long)L.ny * z], L.rho_out);
#pragma unroll
    for (int k = 1; k < V; ++k)
        if (x0 + k == L.nx - 1) nebb<false>(f[k - 1], f[k], 0.f, L.rho_out);
    outlet_from_left_lane<V>(f, L, x0, lane, false, false);
    if (!active) return;
    store_pops<V>(std::make_integer_sequence<int, Q>{}, fd, S, own, f, scale);
    if constexpr (OUT) {
        store_fields<V, AVG>(L, own, R, UX, UY, UZ);
        bool bad = false;
#pragma unroll
        for (int k = 0; k < V; ++k) bad |= !(R[k] > 0.f && R[k] < 3.4e38f);
        if (bad) atomicOr(L.status, 1);
    }
}

// Edge list: each list segment of PASSES*32*V cells in PASSES warp passes of 32*V cells.
template <int V, int PASSES, bool OUT, bool AVG, typename T>
__global__ void __launch_bounds__(128, 3) k_rows_edge(const lbm_lattice L, const PullOffsets po,
                                                      const uint32_t* __restrict__ list, int nlist,
                                                      const T* __restrict__ fs, T* __restrict__ fd, float scale)
{
    constexpr int SEG = PASSES * 32 * V;
    const int lane = threadIdx.x & 31;
    const int gw = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), W = (int)((gridDim.x * blockDim.x) >> 5);
    const int nseg = (L.pitch + SEG - 1) / SEG;
    const float inv_scale = 1.0f / scale;
    for (int w = gw; w < nlist; w += W) {
        int seg, y, z;
        decode_row(__ldg(list + w), nseg, L.ny, seg, y, z);
#pragma unroll 1
        for (int part = 0; part < PASSES; ++part) {
            const int xa = seg * SEG + part * 32 * V;
            if (xa >= L.pitch) break;                                  // warp-uniform
            edge_segment<V, OUT, AVG, T>(L, po, fs, fd, scale, inv_scale, xa + lane * V, y, z, lane);
        }
    }
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
        {
            const long long own = ((long long)z * L.ny + y) * L.pitch + x0;
            float f[V][Q];
            float R[V], UX[V], UY[V], UZ[V];
            pull_fast_all<V>(std::make_integer_sequence<int, Q>{}, f, fs + own, po, lane, z == L.nz - 1);
#pragma unroll
            for (int k = 0; k < V; ++k) collide(f[k], 0.f, 0.f, 0.f, L.tau0, L.csmag2, R[k], UX[k], UY[k], UZ[k]);
            store_pops<V>(std::make_integer_sequence<int, Q>{}, fd, S, own, f, 1.f);
            if constexpr (OUT) {
                store_fields<V, AVG>(L, own, R, UX, UY, UZ);
                bool bad = false;
#pragma unroll
                for (int k = 0; k < V; ++k) bad |= !(R[k] > 0.f && R[k] < 3.4e38f);
                if (bad) atomicOr(L.status, 1);
            }
        }
    }
}

// Output step: fields of one solid segment's V cells per lane (rho = 1, u = 0) and their
// time-average sums.
template <int V, bool AVG>
__device__ __forceinline__ void solid_segment(const lbm_lattice& L, uint32_t id, int lane)
{
    constexpr int SEG = 32 * V;
    const int nseg = (L.pitch + SEG - 1) / SEG;
    const long long S = L.cells;
    int seg, y, z;
    decode_row(id, nseg, L.ny, seg, y, z);
    const int x0 = seg * SEG + lane * V;
    if (x0 >= L.pitch) return;
    const long long own = ((long long)z * L.ny + y) * L.pitch + x0;
    float one[V], zero[V];
#pragma unroll
    for (int k = 0; k < V; ++k) { one[k] = 1.f; zero[k] = 0.f; }
    vstore_plain<V>(L.rho + own, one);
    vstore_plain<V>(L.ux + own, zero);
    vstore_plain<V>(L.uy + own, zero);
    vstore_plain<V>(L.uz + own, zero);
    if constexpr (AVG) {
        if (!L.avg) return;
        float a[V];
        vload_plain<V>(a, L.avg + 3 * S + own);
#pragma unroll
        for (int k = 0; k < V; ++k) a[k] += 1.f;
        vstore_plain<V>(L.avg + 3 * S + own, a);
    }
}

template <int V, bool AVG>
__global__ void k_solid_out(const lbm_lattice L, const uint32_t* __restrict__ list, int nlist)
{
    const int lane = threadIdx.x & 31;
    const int gw = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), W = (int)((gridDim.x * blockDim.x) >> 5);
    for (int w = gw; w < nlist; w += W) solid_segment<V, AVG>(L, __ldg(list + w), lane);
}

// Depth-mean speed of column q = x + pitch*y (floodsim/reach3d.py:412-417): the sums of ux
// and uy over the column's fluid cells, taken in z order, then sqrt(sx^2 + sy^2) / n.
// COH: read the velocities through coherent loads (the persistent batch chunk, where other
// CTAs wrote them earlier in the same launch).
template <bool COH = false>
__device__ __forceinline__ void column_mean_at(const lbm_lattice& L, long long q)
{
    if (q >= (long long)L.ny * L.pitch) return;
    const int x = (int)(q % L.pitch);
    if (x >= L.nx) return;
    const long long plane = (long long)L.ny * L.pitch;
    float sx = 0.f, sy = 0.f, n = 0.f;
    for (int z = 0; z < L.nz; ++z) {
        const long long c = q + plane * z;
        if (!(L.flags[c] & FLAG_SOLID)) {
            sx += COH ? __ldcg(L.ux + c) : L.ux[c];
            sy += COH ? __ldcg(L.uy + c) : L.uy[c];
            n += 1.f;
        }
    }
    L.colU[q] = sqrtf(sx * sx + sy * sy) / fmaxf(n, 1.f);
}

__global__ void k_column_mean(const lbm_lattice L)
{
    column_mean_at(L, (long long)blockIdx.x * blockDim.x + threadIdx.x);
}
