// surrogate.cu -- BF16 tensor-core kernels of the learned warm start (sm_100a, tcgen05).
//
// The network is a small 3D convolutional encoder-decoder on a coarse copy of the lattice.
// Every convolution, forward and backward, is a GEMM on 5th-generation tensor cores:
//   D[M x N] = A[M x K] * B[N x K]^T      A, B bf16, both K-major; accumulation f32 in TMEM
// fed by CUDA-core gather/scatter kernels (im2col, col2im, transposes, pooling) and finished
// by fused epilogues (bias, ReLU, bf16 store).  Three GEMM kernels, chosen per call:
//   k_gemm_ws    products with >= 1024 rows and >= 128 columns: persistent, warp-specialised,
//                TMA ring + MMA thread + epilogue warps, accumulator transposed in TMEM;
//   k_gemm_tma   smaller products: one tile per CTA, TMA ring, MMA thread;
//   k_gemm_bf16  when no tensor map can be made: the register-staged kernel described here.
//
// k_gemm_bf16 tile: one CTA computes 128 rows x BN columns.  Per 64-wide K step, the 4 warps copy
// the A and B tiles (16-byte vectors, zero-filled past M, N, K) into shared memory in the
// 128-byte-swizzled K-major layout the UMMA matrix descriptors describe; one elected thread
// then issues four tcgen05.mma (K = 16 each) accumulating into TMEM and commits them to an
// mbarrier that every thread waits on (bounded: on timeout the block sets an error flag,
// skips the rest, still frees its TMEM and returns).  The epilogue reads the accumulator
// with tcgen05.ld (warp w owns TMEM lanes 32w..32w+31 = tile rows) and applies bias/ReLU.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "errors.cuh"
#include "../../include/lbm_b200.h"

using namespace wfs;

namespace {

constexpr int GM = 128;                     // tile rows = tcgen05.mma M
constexpr int GK = 64;                      // K per shared tile: one 128-byte row of bf16
constexpr long long kWaitPolls = 1LL << 22; // mbarrier polls before a block gives up

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Matrix descriptor of a K-major operand tile in the 128-byte swizzle: rows of 128 bytes,
// groups of 8 rows 1024 bytes apart (fields as in the PTX tcgen05 shared-memory descriptor).
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr)
{
    return (uint64_t)((saddr & 0x3FFFFu) >> 4)      // start address, 16-byte units
         | ((uint64_t)1 << 16)                      // leading byte offset (16 B; unused when swizzled)
         | ((uint64_t)(1024 >> 4) << 32)            // stride byte offset: 8 rows x 128 B
         | ((uint64_t)1 << 46)                      // descriptor version
         | ((uint64_t)2 << 61);                     // 128-byte swizzle
}

// Instruction descriptor: kind::f16 with bf16 A and B, f32 D, both K-major, M = 128, N = n.
__host__ __device__ constexpr uint32_t idesc_bf16(int n)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(GM >> 4) << 24);
}

// Byte offset of 16-byte chunk j (0..7) of row r in a 128-byte-swizzled tile.
__device__ __forceinline__ uint32_t sw128(int r, int j)
{
    return (uint32_t)((r >> 3) * 1024 + (r & 7) * 128 + ((j ^ (r & 7)) << 4));
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t acc)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
        :
        : "r"(tmem), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity)
{
    for (long long i = 0; i < kWaitPolls; ++i) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(mbar), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

enum GemmEpi { EPI_F32 = 0, EPI_F32_ADD = 1, EPI_BF16_BIAS = 2, EPI_BF16_BIAS_RELU = 3, EPI_F32_BIAS = 4 };

template <int BN, int EPI>
__global__ void __launch_bounds__(128, 1) k_gemm_bf16(const __nv_bfloat16* __restrict__ A, int lda,
                                                      const __nv_bfloat16* __restrict__ B, int ldb, int M, int N,
                                                      int K, void* __restrict__ D, int ldd,
                                                      const float* __restrict__ bias, int* __restrict__ err)
{
    static_assert(BN == 32 || BN == 64 || BN == 128 || BN == 256, "TMEM allocation is a power of two >= 32");
    extern __shared__ uint8_t smem_raw[];
    uint8_t* sm = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint8_t* tA = sm;                       // 128 x 128 B
    uint8_t* tB = sm + GM * 128;            // BN x 128 B
    __shared__ __align__(8) uint64_t mbar;
    __shared__ uint32_t tmem_slot;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.x * GM, n0 = blockIdx.y * BN;
    const uint32_t mb = smem_u32(&mbar);
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mb) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");   // visible to the commit's arrive
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_slot)),
                     "r"(BN)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_slot;
    const uint32_t idesc = idesc_bf16(BN);
    const int nk = (K + GK - 1) / GK;
    uint32_t parity = 0;
    bool failed = false;
    for (int kt = 0; kt < nk; ++kt) {
        const int k0 = kt * GK;
        for (int c = tid; c < GM * 8; c += blockDim.x) {
            const int r = c >> 3, j = c & 7, m = m0 + r, k = k0 + 8 * j;
            uint4 v = make_uint4(0, 0, 0, 0);
            if (m < M && k < K) v = *reinterpret_cast<const uint4*>(A + (size_t)m * lda + k);
            *reinterpret_cast<uint4*>(tA + sw128(r, j)) = v;
        }
        for (int c = tid; c < BN * 8; c += blockDim.x) {
            const int r = c >> 3, j = c & 7, n = n0 + r, k = k0 + 8 * j;
            uint4 v = make_uint4(0, 0, 0, 0);
            if (n < N && k < K) v = *reinterpret_cast<const uint4*>(B + (size_t)n * ldb + k);
            *reinterpret_cast<uint4*>(tB + sw128(r, j)) = v;
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");   // shared writes -> tensor core reads
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
            for (int kk = 0; kk < GK / 16; ++kk)
                mma_bf16(tmem, umma_desc(smem_u32(tA) + 32 * kk), umma_desc(smem_u32(tB) + 32 * kk), idesc,
                         (kt | kk) != 0);
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mb)
                         : "memory");
        }
        const bool ok = mbar_wait(mb, parity);                // the tiles are reused next K step
        parity ^= 1u;
        if (__syncthreads_or(!ok)) { failed = true; break; }
    }
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (failed) {
        if (tid == 0) atomicExch(err, 1);
    } else if (nk > 0) {
        const int m = m0 + warp * 32 + lane;
#pragma unroll 1
        for (int c0 = 0; c0 < BN; c0 += 16) {
            uint32_t r[16];
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
                "%14, %15}, [%16];"
                : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                  "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                  "=r"(r[15])
                : "r"(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (m < M) {
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    const int n = n0 + c0 + j;
                    if (n >= N) continue;
                    const float v = __uint_as_float(r[j]);
                    if constexpr (EPI == EPI_F32) {
                        static_cast<float*>(D)[(size_t)m * ldd + n] = v;
                    } else if constexpr (EPI == EPI_F32_ADD) {
                        static_cast<float*>(D)[(size_t)m * ldd + n] += v;
                    } else if constexpr (EPI == EPI_F32_BIAS) {
                        static_cast<float*>(D)[(size_t)m * ldd + n] = v + (bias ? bias[n] : 0.f);
                    } else {
                        float o = v + (bias ? bias[n] : 0.f);
                        if constexpr (EPI == EPI_BF16_BIAS_RELU) o = fmaxf(o, 0.f);
                        static_cast<__nv_bfloat16*>(D)[(size_t)m * ldd + n] = __float2bfloat16_rn(o);
                    }
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(BN) : "memory");
}

// ---------------------------------------------------------------------------------------------
// Pipelined GEMM: the same product and epilogues as k_gemm_bf16, with the operand tiles brought
// in by the Tensor Memory Accelerator.  A ring of S stages (A tile 128 x 64 and B tile BN x 64,
// bf16, 128-byte swizzled -- the layout the UMMA descriptors describe) is filled by one thread
// issuing cp.async.bulk.tensor loads (no multicast) that complete on the stage's `full` mbarrier;
// one thread of another warp waits on `full`, issues the four tcgen05.mma of the stage and
// commits them to the stage's `empty` mbarrier, which the loading thread waits on before it
// refills the stage; the last commit goes to `done`, on which the four warps wait before the
// epilogue reads TMEM.  Every wait is bounded: a thread that runs out sets `err`, the others'
// waits run out in turn, the loading thread waits (bounded) for the copies it issued, and the
// block frees its TMEM and returns.  Tile rows and columns past M, N and K come in as zeros
// (the tensor map's out-of-bounds fill).
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ void mbar_init(uint32_t mbar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t mbar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar), "r"(bytes) : "memory");
}
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int c0, int c1, uint32_t mbar)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
        ::"r"(dst), "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(mbar)
        : "memory");
}

template <int BN, int EPI, int S>
__global__ void __launch_bounds__(128, 1) k_gemm_tma(const __grid_constant__ CUtensorMap tmA,
                                                     const __grid_constant__ CUtensorMap tmB, int M, int N, int K,
                                                     void* __restrict__ D, int ldd, const float* __restrict__ bias,
                                                     int* __restrict__ err)
{
    static_assert(BN == 32 || BN == 64 || BN == 128 || BN == 256, "TMEM allocation is a power of two >= 32");
    constexpr uint32_t A_BYTES = GM * 128, B_BYTES = BN * 128, STAGE = A_BYTES + B_BYTES;
    extern __shared__ uint8_t smem_raw[];
    uint8_t* sm = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    __shared__ __align__(8) uint64_t full[S], empty[S], done;
    __shared__ uint32_t tmem_slot;
    __shared__ int failed;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.x * GM, n0 = blockIdx.y * BN;
    const int nk = (K + GK - 1) / GK;
    if (tid == 0) {
        for (int s = 0; s < S; ++s) {
            mbar_init(smem_u32(&full[s]), 1);
            mbar_init(smem_u32(&empty[s]), 1);
        }
        mbar_init(smem_u32(&done), 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        failed = 0;
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_slot)),
                     "r"(BN)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_slot;
    if (warp == 0 && lane == 0) {
        // loader: stage s = kt % S takes K tile kt once the MMAs of K tile kt - S have read it
        int issued = 0;
        for (int kt = 0; kt < nk; ++kt) {
            const int s = kt % S, round = kt / S;
            if (kt >= S && !mbar_wait(smem_u32(&empty[s]), (uint32_t)((round - 1) & 1))) {
                atomicExch(err, 1);
                failed = 1;
                break;
            }
            if (*(volatile int*)&failed) break;
            const uint32_t a = smem_u32(sm + (size_t)s * STAGE), fb = smem_u32(&full[s]);
            mbar_expect_tx(fb, STAGE);
            tma_load_2d(a, &tmA, kt * GK, m0, fb);
            tma_load_2d(a + A_BYTES, &tmB, kt * GK, n0, fb);
            ++issued;
        }
        // the copies of the last min(S, issued) K tiles must have landed before the block can
        // leave (on success the MMA thread has waited for all of them already)
        for (int kt = (issued > S ? issued - S : 0); kt < issued; ++kt)
            mbar_wait(smem_u32(&full[kt % S]), (uint32_t)((kt / S) & 1));
    } else if (warp == 1 && lane == 0) {
        const uint32_t idesc = idesc_bf16(BN);
        bool ok = true;
        for (int kt = 0; kt < nk; ++kt) {
            const int s = kt % S, round = kt / S;
            if (!mbar_wait(smem_u32(&full[s]), (uint32_t)(round & 1)) || *(volatile int*)&failed) {
                atomicExch(err, 1);
                failed = 1;
                ok = false;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t a = smem_u32(sm + (size_t)s * STAGE);
#pragma unroll
            for (int kk = 0; kk < GK / 16; ++kk)
                mma_bf16(tmem, umma_desc(a + 32 * kk), umma_desc(a + A_BYTES + 32 * kk), idesc, (kt | kk) != 0);
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                         ::"r"(smem_u32(&empty[s]))
                         : "memory");
        }
        if (ok)
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                         ::"r"(smem_u32(&done))
                         : "memory");
    }
    __syncwarp();
    const bool ok = nk > 0 && mbar_wait(smem_u32(&done), 0u);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (__syncthreads_or(!ok || failed)) {
        if (tid == 0 && nk > 0) atomicExch(err, 1);
    } else {
        const int m = m0 + warp * 32 + lane;
#pragma unroll 1
        for (int c0 = 0; c0 < BN; c0 += 16) {
            uint32_t r[16];
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
                "%14, %15}, [%16];"
                : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                  "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                  "=r"(r[15])
                : "r"(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (m < M) {
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    const int n = n0 + c0 + j;
                    if (n >= N) continue;
                    const float v = __uint_as_float(r[j]);
                    if constexpr (EPI == EPI_F32) {
                        static_cast<float*>(D)[(size_t)m * ldd + n] = v;
                    } else if constexpr (EPI == EPI_F32_ADD) {
                        static_cast<float*>(D)[(size_t)m * ldd + n] += v;
                    } else if constexpr (EPI == EPI_F32_BIAS) {
                        static_cast<float*>(D)[(size_t)m * ldd + n] = v + (bias ? bias[n] : 0.f);
                    } else {
                        float o = v + (bias ? bias[n] : 0.f);
                        if constexpr (EPI == EPI_BF16_BIAS_RELU) o = fmaxf(o, 0.f);
                        static_cast<__nv_bfloat16*>(D)[(size_t)m * ldd + n] = __float2bfloat16_rn(o);
                    }
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(BN) : "memory");
}

template <int BN, int EPI>
int launch_gemm(const __nv_bfloat16* A, int lda, const __nv_bfloat16* B, int ldb, int M, int N, int K, void* D, int ldd,
                const float* bias, int* err, cudaStream_t st)
{
    auto kern = k_gemm_bf16<BN, EPI>;
    const int smem = GM * 128 + BN * 128 + 1024;
    static bool attr_set = false;
    if (!attr_set) {
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        attr_set = true;
    }
    dim3 grid((unsigned)((M + GM - 1) / GM), (unsigned)((N + BN - 1) / BN));
    kern<<<grid, 128, smem, st>>>(A, lda, B, ldb, M, N, K, D, ldd, bias, err);
    return check_launch("k_gemm_bf16");
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (the library links no libcuda).
using PfnEncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                    const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                    CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
PfnEncodeTiled encode_tiled()
{
    static PfnEncodeTiled fn = nullptr;
    static bool resolved = false;
    if (!resolved) {
        resolved = true;
        void* p = nullptr;
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, nullptr) ==
            cudaSuccess)
            fn = reinterpret_cast<PfnEncodeTiled>(p);
    }
    return fn;
}

// Tensor map of a rows x K bf16 matrix with row stride ld (elements), boxes of 64 (K) x box_rows,
// 128-byte swizzle, zero fill out of bounds.
bool bf16_tile_map(CUtensorMap* map, const __nv_bfloat16* base, int rows, int K, int ld, int box_rows)
{
    PfnEncodeTiled enc = encode_tiled();
    if (!enc) return false;
    const cuuint64_t dims[2] = {(cuuint64_t)K, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)ld * 2};
    const cuuint32_t box[2] = {(cuuint32_t)GK, (cuuint32_t)box_rows};
    const cuuint32_t estr[2] = {1, 1};
    return enc(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<__nv_bfloat16*>(base), dims, strides, box, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

constexpr int kGemmStages = 3;

// The pipelined kernel when the tensor maps can be made; false: the caller runs k_gemm_bf16.
template <int BN, int EPI>
bool launch_gemm_tma(const __nv_bfloat16* A, int lda, const __nv_bfloat16* B, int ldb, int M, int N, int K, void* D,
                     int ldd, const float* bias, int* err, cudaStream_t st, int* status)
{
    CUtensorMap ta, tb;
    if (!bf16_tile_map(&ta, A, M, K, lda, GM) || !bf16_tile_map(&tb, B, N, K, ldb, BN)) return false;
    auto kern = k_gemm_tma<BN, EPI, kGemmStages>;
    const int smem = kGemmStages * (GM * 128 + BN * 128) + 1024;
    static bool attr_set = false;
    if (!attr_set) {
        if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess) return false;
        attr_set = true;
    }
    dim3 grid((unsigned)((M + GM - 1) / GM), (unsigned)((N + BN - 1) / BN));
    kern<<<grid, 128, smem, st>>>(ta, tb, M, N, K, D, ldd, bias, err);
    *status = check_launch("k_gemm_tma");
    return true;
}

template <int EPI>
int launch_gemm_bn(int bn, const __nv_bfloat16* A, int lda, const __nv_bfloat16* B, int ldb, int M, int N, int K,
                   void* D, int ldd, const float* bias, int* err, cudaStream_t st)
{
    int status = LBM_OK;
    switch (bn) {
    case 32:
        if (launch_gemm_tma<32, EPI>(A, lda, B, ldb, M, N, K, D, ldd, bias, err, st, &status)) return status;
        return launch_gemm<32, EPI>(A, lda, B, ldb, M, N, K, D, ldd, bias, err, st);
    case 64:
        if (launch_gemm_tma<64, EPI>(A, lda, B, ldb, M, N, K, D, ldd, bias, err, st, &status)) return status;
        return launch_gemm<64, EPI>(A, lda, B, ldb, M, N, K, D, ldd, bias, err, st);
    case 128:
        if (launch_gemm_tma<128, EPI>(A, lda, B, ldb, M, N, K, D, ldd, bias, err, st, &status)) return status;
        return launch_gemm<128, EPI>(A, lda, B, ldb, M, N, K, D, ldd, bias, err, st);
    default:
        if (launch_gemm_tma<256, EPI>(A, lda, B, ldb, M, N, K, D, ldd, bias, err, st, &status)) return status;
        return launch_gemm<256, EPI>(A, lda, B, ldb, M, N, K, D, ldd, bias, err, st);
    }
}

// ---------------------------------------------------------------------------------------------
// Persistent warp-specialised GEMM for products with many rows and N >= 128 (the convolutions'
// voxels x channels).  The accumulator is held transposed: tcgen05.mma with M = 128 takes a
// 128-row block of B (output channels n0..n0+127) as its A operand and a BV-row block of A
// (voxels m0..m0+BV-1, BV = 128..256) as its B operand, so TMEM lane l holds channel n0 + l and
// column j voxel m0 + j.  The epilogue thread of lane l then writes 32 voxels of one channel,
// and a warp's store covers 32 consecutive channels of one output row (64 or 128 contiguous
// bytes) instead of one element of 32 rows.  Each operand block is read from L2 once per tile
// of 128 x BV outputs, and BV is chosen so the tiles fill the SMs in as few waves as possible
// (32768 rows: BV = 224, 147 tiles on 148 SMs).
//
// One CTA of 6 warps per SM walks the tiles t = blockIdx.x, + gridDim.x, ...:
//   warp 0, one thread: TMA loads of both blocks into a ring of S stages (no multicast),
//     completing on full[s], refilling a stage once empty[s] says its MMAs are done;
//   warp 1, one thread: per stage four tcgen05.mma (K = 16) into accumulator buffer
//     tc & 1 (two buffers of 256 TMEM columns), commit to empty[s]; per tile commit to
//     acc_full[b] after waiting for acc_empty[b] (the epilogue has read the buffer);
//   warps 2-5: wait acc_full[b], tcgen05.ld 32 columns at a time from their lane quarter
//     (warp & 3), release the buffer to the MMA thread, apply the epilogue and store.
// The epilogue of one tile thus runs while the next tile's loads and MMAs proceed.  Every
// wait is bounded; a role that runs out sets `failed` and `err`, the others leave their loops,
// the MMA thread waits (bounded) for its issued MMAs, the loading thread for its copies, and
// the block frees TMEM and returns.
// ---------------------------------------------------------------------------------------------
constexpr int kWsThreads = 192;
constexpr int kWsMaxStages = 8;
constexpr uint32_t kWsChBytes = GM * 128;   // channel block: 128 rows x 64 bf16

template <int EPI>
__global__ void __launch_bounds__(kWsThreads, 1) k_gemm_ws(const __grid_constant__ CUtensorMap tmA,
                                                           const __grid_constant__ CUtensorMap tmB, int M, int N,
                                                           int K, int BV, int S, void* __restrict__ D, int ldd,
                                                           const float* __restrict__ bias, int* __restrict__ err)
{
    extern __shared__ uint8_t smem_raw[];
    uint8_t* sm = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    __shared__ __align__(8) uint64_t full[kWsMaxStages], empty[kWsMaxStages], acc_full[2], acc_empty[2], drain;
    __shared__ uint32_t tmem_slot;
    __shared__ int failed;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t stage_bytes = kWsChBytes + (uint32_t)BV * 128u;
    const int nk = (K + GK - 1) / GK;
    const int tiles_m = (M + BV - 1) / BV, tiles = tiles_m * ((N + GM - 1) / GM);
    if (tid == 0) {
        for (int s = 0; s < S; ++s) {
            mbar_init(smem_u32(&full[s]), 1);
            mbar_init(smem_u32(&empty[s]), 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(smem_u32(&acc_full[b]), 1);
            mbar_init(smem_u32(&acc_empty[b]), 4);
        }
        mbar_init(smem_u32(&drain), 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        failed = 0;
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_slot)),
                     "r"(512)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_slot;
    volatile int* vfailed = &failed;

    if (warp == 0) {
        if (lane == 0) {
            uint32_t it = 0;
            for (int t = blockIdx.x; t < tiles && !*vfailed; t += gridDim.x) {
                const int m0 = (t % tiles_m) * BV, n0 = (t / tiles_m) * GM;
                for (int kt = 0; kt < nk; ++kt, ++it) {
                    const uint32_t s = it % (uint32_t)S, r = it / (uint32_t)S;
                    if (it >= (uint32_t)S && !mbar_wait(smem_u32(&empty[s]), (r - 1) & 1u)) {
                        atomicExch(err, 1);
                        *vfailed = 1;
                    }
                    if (*vfailed) break;
                    const uint32_t base = smem_u32(sm + (size_t)s * stage_bytes), fb = smem_u32(&full[s]);
                    mbar_expect_tx(fb, stage_bytes);
                    tma_load_2d(base, &tmB, kt * GK, n0, fb);
                    tma_load_2d(base + kWsChBytes, &tmA, kt * GK, m0, fb);
                }
            }
            // copies of the last min(S, it) stages filled must have landed before the block leaves
            for (uint32_t j = (it > (uint32_t)S ? it - (uint32_t)S : 0u); j < it; ++j)
                mbar_wait(smem_u32(&full[j % (uint32_t)S]), (j / (uint32_t)S) & 1u);
        }
    } else if (warp == 1) {
        if (lane == 0) {
            const uint32_t idesc = idesc_bf16(BV);
            uint32_t it = 0, tc = 0;
            for (int t = blockIdx.x; t < tiles && !*vfailed; t += gridDim.x, ++tc) {
                const uint32_t b = tc & 1u, u = tc >> 1;
                if (tc >= 2 && !mbar_wait(smem_u32(&acc_empty[b]), (u - 1) & 1u)) {
                    atomicExch(err, 1);
                    *vfailed = 1;
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t d = tmem + b * 256u;
                bool ok = true;
                for (int kt = 0; kt < nk; ++kt, ++it) {
                    const uint32_t s = it % (uint32_t)S, r = it / (uint32_t)S;
                    if (!mbar_wait(smem_u32(&full[s]), r & 1u) || *vfailed) {
                        atomicExch(err, 1);
                        *vfailed = 1;
                        ok = false;
                        break;
                    }
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    const uint32_t base = smem_u32(sm + (size_t)s * stage_bytes);
#pragma unroll
                    for (int kk = 0; kk < GK / 16; ++kk)
                        mma_bf16(d, umma_desc(base + 32 * kk), umma_desc(base + kWsChBytes + 32 * kk), idesc,
                                 (kt | kk) != 0);
                    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                                 ::"r"(smem_u32(&empty[s]))
                                 : "memory");
                }
                if (!ok) break;
                asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                             ::"r"(smem_u32(&acc_full[b]))
                             : "memory");
            }
            // every MMA this thread issued has completed once `drain` does
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                         ::"r"(smem_u32(&drain))
                         : "memory");
            mbar_wait(smem_u32(&drain), 0u);
        }
    } else {
        const int q = warp & 3;                      // TMEM lanes 32q..32q+31 = channels
        uint32_t tc = 0;
        for (int t = blockIdx.x; t < tiles; t += gridDim.x, ++tc) {
            const uint32_t b = tc & 1u, u = tc >> 1;
            const bool ready = mbar_wait(smem_u32(&acc_full[b]), u & 1u);
            if (__any_sync(0xffffffffu, !ready || *vfailed)) {
                if (lane == 0) {
                    atomicExch(err, 1);
                    *vfailed = 1;
                }
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const int m0 = (t % tiles_m) * BV, n = (t / tiles_m) * GM + q * 32 + lane;
            const int mend = M < m0 + BV ? M : m0 + BV;   // rows of this block (BV: a multiple of 16)
            const float bn = (EPI >= EPI_BF16_BIAS && bias && n < N) ? bias[n] : 0.f;
            for (int j0 = 0; j0 < BV; j0 += 32) {
                uint32_t r[32];
                asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, "
                    "%13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, "
                    "[%32];"
                    : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
                      "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
                      "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]),
                      "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]),
                      "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
                    : "r"(tmem + b * 256u + ((uint32_t)(q * 32) << 16) + (uint32_t)j0));
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                if (j0 + 32 >= BV) {
                    // the whole buffer is in registers: hand it back to the MMA thread
                    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
                    __syncwarp();
                    if (lane == 0)
                        asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&acc_empty[b]))
                                     : "memory");
                }
                if (n < N) {
#pragma unroll
                    for (int j = 0; j < 32; ++j) {
                        const int m = m0 + j0 + j;
                        if (m >= mend) break;
                        const float v = __uint_as_float(r[j]);
                        const size_t o = (size_t)m * ldd + n;
                        if constexpr (EPI == EPI_F32) {
                            static_cast<float*>(D)[o] = v;
                        } else if constexpr (EPI == EPI_F32_ADD) {
                            static_cast<float*>(D)[o] += v;
                        } else if constexpr (EPI == EPI_F32_BIAS) {
                            static_cast<float*>(D)[o] = v + bn;
                        } else {
                            float x = v + bn;
                            if constexpr (EPI == EPI_BF16_BIAS_RELU) x = fmaxf(x, 0.f);
                            static_cast<__nv_bfloat16*>(D)[o] = __float2bfloat16_rn(x);
                        }
                    }
                }
            }
        }
    }
    __syncwarp();
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512) : "memory");
}

int sm_count()
{
    int dev = 0, n = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n < 1) n = 148;
    return n;
}

// Row-block width of k_gemm_ws: the fewest waves of tiles over the SMs times the width (the
// rows one SM streams), ties to the wider block (fewer reads of B).
int ws_block_rows(int M, int N, int nsm)
{
    const int tiles_n = (N + GM - 1) / GM;
    int best = 256;
    long long best_cost = -1;
    for (int bv = 256; bv >= 128; bv -= 32) {
        const long long tiles = (long long)((M + bv - 1) / bv) * tiles_n;
        const long long cost = (tiles + nsm - 1) / nsm * bv;
        if (best_cost < 0 || cost < best_cost) {
            best_cost = cost;
            best = bv;
        }
    }
    return best;
}

// k_gemm_ws for M >= 1024 rows and N >= 128 channels when the tensor maps can be made;
// false: the caller runs the one-tile-per-CTA kernels.
template <int EPI>
bool launch_gemm_ws(const __nv_bfloat16* A, int lda, const __nv_bfloat16* B, int ldb, int M, int N, int K, void* D,
                    int ldd, const float* bias, int* err, cudaStream_t st, int* status)
{
    if (M < 1024 || N < GM) return false;
    const int nsm = sm_count();
    const int bv = ws_block_rows(M, N, nsm);
    const int stage = (int)kWsChBytes + bv * 128;
    // as many stages as 225 KB of shared memory hold (row block 224: 5, which measured 1 % above 4)
    const int stages = (225 * 1024 - 1024) / stage < kWsMaxStages ? (225 * 1024 - 1024) / stage : kWsMaxStages;
    const int smem = stages * stage + 1024;         // > half the SM's shared memory: one CTA per SM
    CUtensorMap ta, tb;
    if (!bf16_tile_map(&ta, A, M, K, lda, bv) || !bf16_tile_map(&tb, B, N, K, ldb, GM)) return false;
    auto kern = k_gemm_ws<EPI>;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    const long long tiles = (long long)((M + bv - 1) / bv) * ((N + GM - 1) / GM);
    const int grid = (int)(tiles < nsm ? tiles : nsm);
    kern<<<grid, kWsThreads, smem, st>>>(ta, tb, M, N, K, bv, stages, D, ldd, bias, err);
    *status = check_launch("k_gemm_ws");
    return true;
}

template <int EPI>
int launch_gemm_any(int bn, const __nv_bfloat16* A, int lda, const __nv_bfloat16* B, int ldb, int M, int N, int K,
                    void* D, int ldd, const float* bias, int* err, cudaStream_t st)
{
    int status = LBM_OK;
    if (launch_gemm_ws<EPI>(A, lda, B, ldb, M, N, K, D, ldd, bias, err, st, &status)) return status;
    return launch_gemm_bn<EPI>(bn, A, lda, B, ldb, M, N, K, D, ldd, bias, err, st);
}

// ---------------------------------------------------------------------------------------------
// Network support kernels (CUDA cores).  Activations are channels-last: X[v * C + c], v = voxel
// index x + X*(y + Y*z) of a (Z, Y, X) grid.  A 3x3x3 tap t = (dz+1)*9 + (dy+1)*3 + (dx+1).
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ bool tap_src(int t, int x, int y, int z, int X, int Y, int Z, long long& v)
{
    const int xs = x + t % 3 - 1, ys = y + (t / 3) % 3 - 1, zs = z + t / 9 - 1;
    if (xs < 0 || xs >= X || ys < 0 || ys >= Y || zs < 0 || zs >= Z) return false;
    v = xs + (long long)X * (ys + (long long)Y * zs);
    return true;
}

// col[v][t*C + c] = X[neighbour t of v][c] (zero outside the grid).  One thread per (v, t, 8 channels).
__global__ void k_im2col(const __nv_bfloat16* __restrict__ Xin, int C, int X, int Y, int Z,
                         __nv_bfloat16* __restrict__ col)
{
    const long long V = (long long)X * Y * Z;
    const int C8 = C / 8;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;     // (v * 27 + t) * C8 + q
    if (i >= V * 27 * C8) return;
    const int q = (int)(i % C8);
    const long long vt = i / C8;
    const int t = (int)(vt % 27);
    const long long v = vt / 27;
    const int x = (int)(v % X), y = (int)((v / X) % Y), z = (int)(v / ((long long)X * Y));
    long long s;
    uint4 val = make_uint4(0, 0, 0, 0);
    if (tap_src(t, x, y, z, X, Y, Z, s)) val = *reinterpret_cast<const uint4*>(Xin + s * C + 8 * q);
    *reinterpret_cast<uint4*>(col + (v * 27 + t) * C + 8 * q) = val;
}

// dX[v][c] = sum_t dcol[u][t*C + c] over the voxels u whose tap t reads v (u = v - offset_t).
__global__ void k_col2im(const float* __restrict__ dcol, int C, int X, int Y, int Z, float* __restrict__ dX)
{
    const long long V = (long long)X * Y * Z;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;     // v * C + c
    if (i >= V * C) return;
    const int c = (int)(i % C);
    const long long v = i / C;
    const int x = (int)(v % X), y = (int)((v / X) % Y), z = (int)(v / ((long long)X * Y));
    float s = 0.f;
    for (int t = 0; t < 27; ++t) {
        long long u;
        // u reads v through tap t iff v is u's tap-t neighbour, i.e. u = v - offset_t = v's tap (26 - t)
        if (tap_src(26 - t, x, y, z, X, Y, Z, u)) s += dcol[(u * 27 + t) * C + c];
    }
    dX[i] = s;
}

// out[c][r] = in[r][c] for r < R; columns r in [R, Rp) of out are zero (K padding of the GEMMs).
__global__ void k_transpose_bf16(const __nv_bfloat16* __restrict__ in, long long R, int C, long long Rp,
                                 __nv_bfloat16* __restrict__ out)
{
    __shared__ __nv_bfloat16 tile[32][33];
    const long long r0 = (long long)blockIdx.x * 32;
    const int c0 = blockIdx.y * 32;
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const long long r = r0 + k;
        const int c = c0 + threadIdx.x;
        tile[k][threadIdx.x] = (r < R && c < C) ? in[r * C + c] : __float2bfloat16_rn(0.f);
    }
    __syncthreads();
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int c = c0 + k;
        const long long r = r0 + threadIdx.x;
        if (c < C && r < Rp) out[(long long)c * Rp + r] = tile[threadIdx.x][k];
    }
}

// Backward through ReLU: g = dY * (Y > 0) (or dY when relu == 0), as bf16, and its column sums
// (the bias gradient, float atomics).
__global__ void k_act_grad(const float* __restrict__ dY, const __nv_bfloat16* __restrict__ Y, long long V, int C,
                           int relu, __nv_bfloat16* __restrict__ g, float* __restrict__ dbias)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= V * C) return;
    float v = dY[i];
    if (relu && !(__bfloat162float(Y[i]) > 0.f)) v = 0.f;
    g[i] = __float2bfloat16_rn(v);
    atomicAdd(dbias + (i % C), v);
}

// 2x2x2 average pooling of a (Z, Y, X) grid (even sizes) and its backward.
__global__ void k_pool2(const __nv_bfloat16* __restrict__ in, int C, int X, int Y, int Z, __nv_bfloat16* __restrict__ out)
{
    const int Xh = X / 2, Yh = Y / 2, Zh = Z / 2;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;     // vh * C + c
    if (i >= (long long)Xh * Yh * Zh * C) return;
    const int c = (int)(i % C);
    const long long vh = i / C;
    const int x = (int)(vh % Xh), y = (int)((vh / Xh) % Yh), z = (int)(vh / ((long long)Xh * Yh));
    float s = 0.f;
    for (int d = 0; d < 8; ++d) {
        const long long v = (2 * x + (d & 1)) + (long long)X * ((2 * y + ((d >> 1) & 1)) + (long long)Y * (2 * z + (d >> 2)));
        s += __bfloat162float(in[v * C + c]);
    }
    out[i] = __float2bfloat16_rn(0.125f * s);
}
__global__ void k_pool2_back(const float* __restrict__ dout, int C, int X, int Y, int Z, float* __restrict__ din,
                             int accumulate)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;     // v * C + c
    if (i >= (long long)X * Y * Z * C) return;
    const int c = (int)(i % C);
    const long long v = i / C;
    const int x = (int)(v % X), y = (int)((v / X) % Y), z = (int)(v / ((long long)X * Y));
    const long long vh = (x / 2) + (long long)(X / 2) * ((y / 2) + (long long)(Y / 2) * (z / 2));
    const float g = 0.125f * dout[vh * C + c];
    din[i] = accumulate ? din[i] + g : g;
}

// out[v] = coarse[parent(v)] + skip[v] (nearest 2x upsampling plus the skip connection) and its
// backward for the coarse input: dcoarse[vh] = sum over the 8 children of dout.
__global__ void k_up2_add(const __nv_bfloat16* __restrict__ coarse, const __nv_bfloat16* __restrict__ skip, int C, int X,
                          int Y, int Z, __nv_bfloat16* __restrict__ out)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long long)X * Y * Z * C) return;
    const int c = (int)(i % C);
    const long long v = i / C;
    const int x = (int)(v % X), y = (int)((v / X) % Y), z = (int)(v / ((long long)X * Y));
    const long long vh = (x / 2) + (long long)(X / 2) * ((y / 2) + (long long)(Y / 2) * (z / 2));
    out[i] = __float2bfloat16_rn(__bfloat162float(coarse[vh * C + c]) + __bfloat162float(skip[i]));
}
__global__ void k_up2_back(const float* __restrict__ dout, int C, int X, int Y, int Z, float* __restrict__ dcoarse)
{
    const int Xh = X / 2, Yh = Y / 2, Zh = Z / 2;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long long)Xh * Yh * Zh * C) return;
    const int c = (int)(i % C);
    const long long vh = i / C;
    const int x = (int)(vh % Xh), y = (int)((vh / Xh) % Yh), z = (int)(vh / ((long long)Xh * Yh));
    float s = 0.f;
    for (int d = 0; d < 8; ++d) {
        const long long v = (2 * x + (d & 1)) + (long long)X * ((2 * y + ((d >> 1) & 1)) + (long long)Y * (2 * z + (d >> 2)));
        s += dout[v * C + c];
    }
    dcoarse[i] = s;
}

// Masked mean-square error of pred[v][0..nout) (row stride Cp) against target[v][0..nout):
// loss += sum m (p - t)^2 / n, dpred = 2 m (p - t) / n (padding channels get 0).
__global__ void k_mse(const float* __restrict__ pred, int Cp, const float* __restrict__ target, int nout,
                      const float* __restrict__ mask, long long V, float inv_n, float* __restrict__ dpred,
                      float* __restrict__ loss)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;     // v * Cp + c
    if (i >= V * Cp) return;
    const int c = (int)(i % Cp);
    const long long v = i / Cp;
    float g = 0.f;
    if (c < nout) {
        const float d = pred[i] - target[v * nout + c];
        const float m = mask[v];
        g = 2.f * m * d * inv_n;
        atomicAdd(loss, m * d * d * inv_n);
    }
    dpred[i] = g;
}

// Adam step on float32 master weights, refreshing their bf16 copy.
__global__ void k_adam(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m, float* __restrict__ s,
                       long long n, float lr, float b1, float b2, float eps, float c1, float c2,
                       __nv_bfloat16* __restrict__ wb)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi, si = b2 * s[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    s[i] = si;
    const float wi = w[i] - lr * (mi / c1) / (sqrtf(si / c2) + eps);
    w[i] = wi;
    if (wb) wb[i] = __float2bfloat16_rn(wi);
}

inline unsigned blocks(long long n, int t) { return (unsigned)((n + t - 1) / t); }

}  // namespace

extern "C" {

int lbm_nn_im2col(const uint16_t* x, int C, int X, int Y, int Z, uint16_t* col, void* stream)
{
    g_err[0] = 0;
    if (!x || !col || C % 8 || X < 1 || Y < 1 || Z < 1) return fail(LBM_ERR_ARG, "lbm_nn_im2col: bad arguments");
    const long long n = (long long)X * Y * Z * 27 * (C / 8);
    k_im2col<<<blocks(n, 256), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        reinterpret_cast<const __nv_bfloat16*>(x), C, X, Y, Z, reinterpret_cast<__nv_bfloat16*>(col));
    return check_launch("k_im2col");
}

int lbm_nn_col2im(const float* dcol, int C, int X, int Y, int Z, float* dx, void* stream)
{
    g_err[0] = 0;
    if (!dcol || !dx || C < 1 || X < 1 || Y < 1 || Z < 1) return fail(LBM_ERR_ARG, "lbm_nn_col2im: bad arguments");
    const long long n = (long long)X * Y * Z * C;
    k_col2im<<<blocks(n, 256), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(dcol, C, X, Y, Z, dx);
    return check_launch("k_col2im");
}

int lbm_nn_transpose(const uint16_t* in, int64_t R, int C, int64_t Rp, uint16_t* out, void* stream)
{
    g_err[0] = 0;
    if (!in || !out || R < 1 || C < 1 || Rp < R) return fail(LBM_ERR_ARG, "lbm_nn_transpose: bad arguments");
    dim3 grid(blocks(Rp, 32), blocks(C, 32));
    k_transpose_bf16<<<grid, dim3(32, 8), 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        reinterpret_cast<const __nv_bfloat16*>(in), R, C, Rp, reinterpret_cast<__nv_bfloat16*>(out));
    return check_launch("k_transpose_bf16");
}

int lbm_nn_act_grad(const float* dy, const uint16_t* y, int64_t V, int C, int relu, uint16_t* g, float* dbias,
                    void* stream)
{
    g_err[0] = 0;
    if (!dy || !g || !dbias || (relu && !y) || V < 1 || C < 1) return fail(LBM_ERR_ARG, "lbm_nn_act_grad: bad arguments");
    k_act_grad<<<blocks(V * C, 256), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        dy, reinterpret_cast<const __nv_bfloat16*>(y), V, C, relu, reinterpret_cast<__nv_bfloat16*>(g), dbias);
    return check_launch("k_act_grad");
}

int lbm_nn_pool2(const uint16_t* in, int C, int X, int Y, int Z, uint16_t* out, void* stream)
{
    g_err[0] = 0;
    if (!in || !out || C < 1 || X % 2 || Y % 2 || Z % 2 || X < 2 || Y < 2 || Z < 2)
        return fail(LBM_ERR_ARG, "lbm_nn_pool2: bad arguments (even grid sizes)");
    k_pool2<<<blocks((long long)X * Y * Z / 8 * C, 256), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        reinterpret_cast<const __nv_bfloat16*>(in), C, X, Y, Z, reinterpret_cast<__nv_bfloat16*>(out));
    return check_launch("k_pool2");
}

int lbm_nn_pool2_back(const float* dout, int C, int X, int Y, int Z, float* din, int accumulate, void* stream)
{
    g_err[0] = 0;
    if (!dout || !din || C < 1 || X % 2 || Y % 2 || Z % 2) return fail(LBM_ERR_ARG, "lbm_nn_pool2_back: bad arguments");
    k_pool2_back<<<blocks((long long)X * Y * Z * C, 256), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        dout, C, X, Y, Z, din, accumulate);
    return check_launch("k_pool2_back");
}

int lbm_nn_up2_add(const uint16_t* coarse, const uint16_t* skip, int C, int X, int Y, int Z, uint16_t* out,
                   void* stream)
{
    g_err[0] = 0;
    if (!coarse || !skip || !out || C < 1 || X % 2 || Y % 2 || Z % 2)
        return fail(LBM_ERR_ARG, "lbm_nn_up2_add: bad arguments");
    k_up2_add<<<blocks((long long)X * Y * Z * C, 256), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        reinterpret_cast<const __nv_bfloat16*>(coarse), reinterpret_cast<const __nv_bfloat16*>(skip), C, X, Y, Z,
        reinterpret_cast<__nv_bfloat16*>(out));
    return check_launch("k_up2_add");
}

int lbm_nn_up2_back(const float* dout, int C, int X, int Y, int Z, float* dcoarse, void* stream)
{
    g_err[0] = 0;
    if (!dout || !dcoarse || C < 1 || X % 2 || Y % 2 || Z % 2) return fail(LBM_ERR_ARG, "lbm_nn_up2_back: bad arguments");
    k_up2_back<<<blocks((long long)X * Y * Z / 8 * C, 256), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        dout, C, X, Y, Z, dcoarse);
    return check_launch("k_up2_back");
}

int lbm_nn_mse(const float* pred, int Cp, const float* target, int nout, const float* mask, int64_t V, float inv_n,
               float* dpred, float* loss, void* stream)
{
    g_err[0] = 0;
    if (!pred || !target || !mask || !dpred || !loss || nout > Cp || V < 1) return fail(LBM_ERR_ARG, "lbm_nn_mse: bad arguments");
    k_mse<<<blocks(V * Cp, 256), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(pred, Cp, target, nout, mask, V,
                                                                                   inv_n, dpred, loss);
    return check_launch("k_mse");
}

int lbm_nn_adam(float* w, const float* g, float* m, float* s, int64_t n, float lr, float b1, float b2, float eps,
                int step, uint16_t* wbf16, void* stream)
{
    g_err[0] = 0;
    if (!w || !g || !m || !s || n < 1 || step < 1) return fail(LBM_ERR_ARG, "lbm_nn_adam: bad arguments");
    const float c1 = 1.f - powf(b1, (float)step), c2 = 1.f - powf(b2, (float)step);
    k_adam<<<blocks(n, 256), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        w, g, m, s, n, lr, b1, b2, eps, c1, c2, reinterpret_cast<__nv_bfloat16*>(wbf16));
    return check_launch("k_adam");
}

int lbm_gemm_bf16(const uint16_t* A, int lda, const uint16_t* B, int ldb, int M, int N, int K, void* D, int ldd,
                  int epilogue, const float* bias, int* err, void* stream)
{
    g_err[0] = 0;
    if (!A || !B || !D || !err) return fail(LBM_ERR_ARG, "lbm_gemm_bf16: NULL pointer");
    if (M < 1 || N < 1 || K < 1) return fail(LBM_ERR_ARG, "lbm_gemm_bf16: empty product %dx%dx%d", M, N, K);
    if (K % 8 || lda % 8 || ldb % 8 || lda < K || ldb < K)
        return fail(LBM_ERR_ARG, "lbm_gemm_bf16: K, lda and ldb must be multiples of 8 with lda, ldb >= K");
    if ((reinterpret_cast<uintptr_t>(A) | reinterpret_cast<uintptr_t>(B)) & 15)
        return fail(LBM_ERR_ARG, "lbm_gemm_bf16: A and B must be 16-byte aligned");
    if (ldd < N) return fail(LBM_ERR_ARG, "lbm_gemm_bf16: ldd < N");
    if (epilogue < 0 || epilogue > 4) return fail(LBM_ERR_ARG, "lbm_gemm_bf16: unknown epilogue %d", epilogue);
    const int bn = N <= 32 ? 32 : N <= 64 ? 64 : N <= 128 ? 128 : 256;
    const __nv_bfloat16* a = reinterpret_cast<const __nv_bfloat16*>(A);
    const __nv_bfloat16* b = reinterpret_cast<const __nv_bfloat16*>(B);
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    switch (epilogue) {
    case EPI_F32: return launch_gemm_any<EPI_F32>(bn, a, lda, b, ldb, M, N, K, D, ldd, bias, err, st);
    case EPI_F32_ADD: return launch_gemm_any<EPI_F32_ADD>(bn, a, lda, b, ldb, M, N, K, D, ldd, bias, err, st);
    case EPI_BF16_BIAS: return launch_gemm_any<EPI_BF16_BIAS>(bn, a, lda, b, ldb, M, N, K, D, ldd, bias, err, st);
    case EPI_F32_BIAS: return launch_gemm_any<EPI_F32_BIAS>(bn, a, lda, b, ldb, M, N, K, D, ldd, bias, err, st);
    default: return launch_gemm_any<EPI_BF16_BIAS_RELU>(bn, a, lda, b, ldb, M, N, K, D, ldd, bias, err, st);
    }
}

}  // extern "C"
