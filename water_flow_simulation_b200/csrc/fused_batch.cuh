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
