// fused_batch.cuh -- many lattices of one 16-bit run, stepped by one launch per kernel class.
// Included inside the anonymous namespace of lbm_kernels.cu, after fused_half.cuh and bc_row.
//
// A batch holds K lattices (boat cases of any sizes) in device memory: their lattice
// descriptors, pull-offset tables, 16-bit storage scales and both population buffers of each.
// Work-list entries carry the case in their top 8 bits and the row-segment id (of that case's
// own 64-cell segments, cells_per_lane 2) in the low 24.  One step of the whole batch is then
// a plain, an edge and a general launch over the concatenated lists (plus the solid-field,
// column-mean and outlet passes on output steps), whatever the sizes of the cases: small
// cases no longer leave the GPU idle between launches or in short tails, and the launch
// count of a step does not grow with the number of cases.  Population buffers alternate by
// step parity, so a chunk of an even number of steps can be captured once as a CUDA graph
// and replayed.
#pragma once

constexpr int kBatchCaseShift = 24;
constexpr uint32_t kBatchSegMask = (1u << kBatchCaseShift) - 1u;
constexpr int kBatchMaxCases = 256;

struct BatchDesc {
    const lbm_lattice* lat;    // K lattice descriptors
    const PullOffsets* po;     // K pull-offset tables
    const float* scale;        // K storage scales
    __half* const* pop0;       // K first population buffers
    __half* const* pop1;       // K second population buffers
};

struct BatchItem {
    int c;
    uint32_t id;
    const __half* fs;
    __half* fd;
};

__device__ __forceinline__ BatchItem batch_item(const BatchDesc& B, int parity, uint32_t e)
{
    BatchItem it;
    it.c = (int)(e >> kBatchCaseShift);
    it.id = e & kBatchSegMask;
    it.fs = parity ? B.pop1[it.c] : B.pop0[it.c];
    it.fd = parity ? B.pop0[it.c] : B.pop1[it.c];
    return it;
}

// Pull-offset tables of the K lattices (set-up).
__global__ void k_batch_pull_offsets(const lbm_lattice* __restrict__ lat, int K, PullOffsets* __restrict__ po)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;     // case * Q + direction
    if (t >= K * Q) return;
    const int c = t / Q, i = t % Q;
    const lbm_lattice& L = lat[c];
    const long long d = (long long)i * L.cells - (long long)cz(i) * L.ny * L.pitch - (long long)cy(i) * L.pitch;
    po[c].d[i] = d;
    po[c].lid[i] = cz(i) == -1 ? (long long)mirz(i) * L.cells - (long long)cy(i) * L.pitch : d;
}

template <int VP, int G, bool OUT, bool AVG>
__global__ void __launch_bounds__(128, VP == 8 ? 3 : 4) k_batch_plain(const BatchDesc B, int parity,
                                                                     const uint32_t* __restrict__ list, int nlist)
{
    constexpr int PER_WARP = 32 / G;
    const int lane = threadIdx.x & 31, gl = lane % G, grp = lane / G;
    const int gw = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), W = (int)((gridDim.x * blockDim.x) >> 5);
    for (long long b = (long long)gw * PER_WARP; b < nlist; b += (long long)W * PER_WARP) {
        const bool valid = b + grp < nlist;
        const BatchItem it = batch_item(B, parity, __ldg(list + (valid ? b + grp : b)));
        h_plain_segment<VP, G, OUT, AVG>(B.lat[it.c], B.po[it.c], it.fs, it.fd, __ldg(B.scale + it.c), it.id, gl,
                                         valid);
    }
}

template <bool OUT, bool AVG>
__global__ void __launch_bounds__(128, 3) k_batch_edge(const BatchDesc B, int parity, const uint32_t* __restrict__ list,
                                                       int nlist)
{
    constexpr int V = 2, SEG = 64;
    const int lane = threadIdx.x & 31;
    const int gw = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), W = (int)((gridDim.x * blockDim.x) >> 5);
    for (int w = gw; w < nlist; w += W) {
        const BatchItem it = batch_item(B, parity, __ldg(list + w));
        const lbm_lattice& L = B.lat[it.c];
        const float scale = __ldg(B.scale + it.c);
        int seg, y, z;
        decode_row(it.id, (L.pitch + SEG - 1) / SEG, L.ny, seg, y, z);
        edge_segment<V, OUT, AVG, __half>(L, B.po[it.c], it.fs, it.fd, scale, 1.0f / scale, seg * SEG + lane * V, y, z,
                                          lane);
    }
}

template <bool OUT, bool UCOL, bool AVG>
__global__ void __launch_bounds__(128, 4) k_batch_general(const BatchDesc B, int parity,
                                                          const uint32_t* __restrict__ list, int nlist)
{
    constexpr int V = 2, SEG = 64;
    const int lane = threadIdx.x & 31;
    const int gw = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), W = (int)((gridDim.x * blockDim.x) >> 5);
    for (int w = gw; w < nlist; w += W) {
        const BatchItem it = batch_item(B, parity, __ldg(list + w));
        const lbm_lattice& L = B.lat[it.c];
        const float scale = __ldg(B.scale + it.c);
        int seg, y, z;
        decode_row(it.id, (L.pitch + SEG - 1) / SEG, L.ny, seg, y, z);
        general_segment<V, OUT, UCOL, AVG, __half>(L, B.po[it.c], it.fs, it.fd, scale, 1.0f / scale,
                                                   seg * SEG + lane * V, y, z, lane);
    }
}

template <bool AVG>
__global__ void k_batch_solid_out(const BatchDesc B, const uint32_t* __restrict__ list, int nlist)
{
    const int lane = threadIdx.x & 31;
    const int gw = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), W = (int)((gridDim.x * blockDim.x) >> 5);
    for (int w = gw; w < nlist; w += W) {
        const uint32_t e = __ldg(list + w);
        solid_segment<2, AVG>(B.lat[e >> kBatchCaseShift], e & kBatchSegMask, lane);
    }
}

// blockIdx.y = case
__global__ void k_batch_column_mean(const BatchDesc B)
{
    column_mean_at(B.lat[blockIdx.y], (long long)blockIdx.x * blockDim.x + threadIdx.x);
}

// Outlet rows of the cases whose x = nx-2 and x = nx-1 fall in different segments; blockIdx.y = case.
__global__ void k_batch_bc_rows(const BatchDesc B, int parity)
{
    const lbm_lattice& L = B.lat[blockIdx.y];
    if ((L.nx - 1) % 64 != 0) return;
    __half* fd = parity ? B.pop0[blockIdx.y] : B.pop1[blockIdx.y];
    bc_row<__half>(L, fd, 2, __ldg(B.scale + blockIdx.y), (long long)blockIdx.x * blockDim.x + threadIdx.x);
}

// ---------------------------------------------------------------------------------------------
// Persistent chunk: `nsteps` steps of the whole batch in ONE cooperative launch.  Every CTA stays
// resident for the chunk; a step is two phases separated by grid barriers:
//   phase 1  the step's segment tasks, statically interleaved over all warps of the grid in one
//            task space [special | edge | plain groups]: a special or edge task is one 64-cell
//            segment (the general / edge path, 2 cells per lane), a plain task four segments
//            (8 lanes of 8 cells each); so every warp works through some of each kind and the
//            latency-bound special segments run beside the bandwidth-bound plain ones;
//   phase 2  the outlet rows of cases whose x = nx-2 and nx-1 lie in different segments, and on
//            the chunk's last (output) step the solid segments' fields and the column means.
// The per-segment device functions are those of the per-kernel batch step, so both give the
// same populations bit for bit.  Barrier waits are bounded by kBarrierTimeoutNs of the global
// timer: a CTA that runs out raises an abort flag in the sync words, every CTA then leaves the
// chunk, and bit 1 of every case's status word is set (the state is not to be trusted).
// sync: 4 uint32 of device memory, zeroed by the host before the launch (count, generation,
// abort flag, spare).
// ---------------------------------------------------------------------------------------------
constexpr unsigned long long kBarrierTimeoutNs = 2000000000ULL;

__device__ __forceinline__ unsigned long long global_timer_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Grid-wide barrier of a cooperative launch; false when a wait ran out (here or in another CTA).
__device__ bool grid_barrier(uint32_t* sync, unsigned nblocks)
{
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        ok = 1;
        volatile uint32_t* vgen = sync + 1;
        volatile uint32_t* vabort = sync + 2;
        const uint32_t g = *vgen;
        __threadfence();
        const uint32_t arrived = atomicAdd(sync, 1u);
        if (arrived == nblocks - 1) {
            atomicExch(sync, 0u);
            __threadfence();
            atomicAdd(sync + 1, 1u);
        } else {
            const unsigned long long t0 = global_timer_ns();
            while (*vgen == g) {
                if (*vabort) { ok = 0; break; }
                if (global_timer_ns() - t0 > kBarrierTimeoutNs) {
                    atomicExch(sync + 2, 1u);
                    ok = 0;
                    break;
                }
                __nanosleep(256);
            }
        }
        __threadfence();
    }
    __syncthreads();
    return ok != 0;
}

template <bool OUT, bool UCOL, bool AVG>
__device__ __forceinline__ void batch_tasks(const BatchDesc& B, int parity, const uint32_t* __restrict__ special,
                                            int n_special, const uint32_t* __restrict__ edge, int n_edge,
                                            const uint32_t* __restrict__ plain, int n_plain)
{
    constexpr int V = 2, SEG = 64, VP = 8, G = 8, PER_WARP = 32 / G;
    const int lane = threadIdx.x & 31;
    const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long W = ((long long)gridDim.x * blockDim.x) >> 5;
    const long long n_pgroups = (n_plain + PER_WARP - 1) / PER_WARP;
    const long long total = (long long)n_special + n_edge + n_pgroups;
    for (long long t = gw; t < total; t += W) {
        // populations are read with coherent loads (hcoh): this launch wrote them in earlier steps
        if (t < n_special) {
            const BatchItem it = batch_item(B, parity, __ldg(special + t));
            const lbm_lattice& L = B.lat[it.c];
            const float scale = __ldg(B.scale + it.c);
            int seg, y, z;
            decode_row(it.id, (L.pitch + SEG - 1) / SEG, L.ny, seg, y, z);
            general_segment<V, OUT, UCOL, AVG, hcoh>(L, B.po[it.c], reinterpret_cast<const hcoh*>(it.fs),
                                                     reinterpret_cast<hcoh*>(it.fd), scale, 1.0f / scale,
                                                     seg * SEG + lane * V, y, z, lane);
        } else if (t < (long long)n_special + n_edge) {
            const BatchItem it = batch_item(B, parity, __ldg(edge + (t - n_special)));
            const lbm_lattice& L = B.lat[it.c];
            const float scale = __ldg(B.scale + it.c);
            int seg, y, z;
            decode_row(it.id, (L.pitch + SEG - 1) / SEG, L.ny, seg, y, z);
            edge_segment<V, OUT, AVG, hcoh>(L, B.po[it.c], reinterpret_cast<const hcoh*>(it.fs),
                                            reinterpret_cast<hcoh*>(it.fd), scale, 1.0f / scale, seg * SEG + lane * V,
                                            y, z, lane);
        } else {
            const long long b = (t - n_special - n_edge) * PER_WARP;
            const int gl = lane % G, grp = lane / G;
            const bool valid = b + grp < n_plain;
            const BatchItem it = batch_item(B, parity, __ldg(plain + (valid ? b + grp : b)));
            h_plain_segment<VP, G, OUT, AVG, hcoh>(B.lat[it.c], B.po[it.c], reinterpret_cast<const hcoh*>(it.fs),
                                                   reinterpret_cast<hcoh*>(it.fd), __ldg(B.scale + it.c), it.id, gl,
                                                   valid);
        }
    }
}

template <bool UCOL, bool AVG_LAST>
__global__ void __launch_bounds__(128, 3) k_batch_chunk(const BatchDesc B, int K, int parity0, int nsteps,
                                                      const uint32_t* __restrict__ special, int n_special,
                                                      const uint32_t* __restrict__ edge, int n_edge,
                                                      const uint32_t* __restrict__ plain, int n_plain,
                                                      const uint32_t* __restrict__ solid, int n_solid,
                                                      int max_rows, int max_columns, uint32_t* sync)
{
    const unsigned nblocks = gridDim.x;
    const long long gtid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long nthreads = (long long)gridDim.x * blockDim.x;
    for (int s = 0; s < nsteps; ++s) {
        const int parity = (parity0 + s) & 1;
        const bool last = s == nsteps - 1;
        if (last) batch_tasks<true, UCOL, AVG_LAST>(B, parity, special, n_special, edge, n_edge, plain, n_plain);
        else batch_tasks<false, UCOL, false>(B, parity, special, n_special, edge, n_edge, plain, n_plain);
        bool ok = grid_barrier(sync, nblocks);
        if (ok) {
            // outlet rows of the cases that need their own pass (the fields they write are not
            // read by the solid-field or column-mean work of this phase)
            for (long long j = gtid; j < (long long)K * max_rows; j += nthreads) {
                const int c = (int)(j / max_rows);
                const lbm_lattice& L = B.lat[c];
                if ((L.nx - 1) % 64 != 0) continue;
                hcoh* fd = reinterpret_cast<hcoh*>(parity ? B.pop0[c] : B.pop1[c]);
                bc_row<hcoh>(L, fd, 2, __ldg(B.scale + c), j % max_rows);
            }
            if (last) {
                const int lane = threadIdx.x & 31;
                for (long long w = gtid >> 5; w < n_solid; w += nthreads >> 5) {
                    const uint32_t e = __ldg(solid + w);
                    solid_segment<2, AVG_LAST>(B.lat[e >> kBatchCaseShift], e & kBatchSegMask, lane);
                }
                if (UCOL)
                    for (long long j = gtid; j < (long long)K * max_columns; j += nthreads)
                        column_mean_at<true>(B.lat[j / max_columns], j % max_columns);
            }
            if (!last) ok = grid_barrier(sync, nblocks);
        }
        if (!ok) {
            if (gtid < K) atomicOr(B.lat[gtid].status, 2);
            return;
        }
    }
}
