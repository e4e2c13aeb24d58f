// surrogate.cu -- BF16 tensor-core kernels of the learned warm start (sm_100a, tcgen05).
//
// The network is a small 3D convolutional encoder-decoder on a coarse copy of the lattice.
// Every convolution, forward and backward, is a GEMM on 5th-generation tensor cores:
//   D[M x N] = A[M x K] * B[N x K]^T      A, B bf16, both K-major; accumulation f32 in TMEM
// (k_gemm_bf16), fed by CUDA-core gather/scatter kernels (im2col, col2im, transposes,
// pooling) and finished by fused epilogues (bias, ReLU, bf16 store).
//
// GEMM tile: one CTA computes 128 rows x BN columns.  Per 64-wide K step, the 4 warps copy
// the A and B tiles (16-byte vectors, zero-filled past M, N, K) into shared memory in the
// 128-byte-swizzled K-major layout the UMMA matrix descriptors describe; one elected thread
// then issues four tcgen05.mma (K = 16 each) accumulating into TMEM and commits them to an
// mbarrier that every thread waits on (bounded: on timeout the block sets an error flag,
// skips the rest, still frees its TMEM and returns).  The epilogue reads the accumulator
// with tcgen05.ld (warp w owns TMEM lanes 32w..32w+31 = tile rows) and applies bias/ReLU.
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

enum GemmEpi { EPI_F32 = 0, EPI_F32_ADD = 1, EPI_BF16_BIAS = 2, EPI_BF16_BIAS_RELU = 3 };

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

template <int EPI>
int launch_gemm_bn(int bn, const __nv_bfloat16* A, int lda, const __nv_bfloat16* B, int ldb, int M, int N, int K,
                   void* D, int ldd, const float* bias, int* err, cudaStream_t st)
{
    switch (bn) {
    case 32: return launch_gemm<32, EPI>(A, lda, B, ldb, M, N, K, D, ldd, bias, err, st);
    case 64: return launch_gemm<64, EPI>(A, lda, B, ldb, M, N, K, D, ldd, bias, err, st);
    case 128: return launch_gemm<128, EPI>(A, lda, B, ldb, M, N, K, D, ldd, bias, err, st);
    default: return launch_gemm<256, EPI>(A, lda, B, ldb, M, N, K, D, ldd, bias, err, st);
    }
}

}  // namespace

extern "C" {

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
    if (epilogue < 0 || epilogue > 3) return fail(LBM_ERR_ARG, "lbm_gemm_bf16: unknown epilogue %d", epilogue);
    const int bn = N <= 32 ? 32 : N <= 64 ? 64 : N <= 128 ? 128 : 256;
    const __nv_bfloat16* a = reinterpret_cast<const __nv_bfloat16*>(A);
    const __nv_bfloat16* b = reinterpret_cast<const __nv_bfloat16*>(B);
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    switch (epilogue) {
    case EPI_F32: return launch_gemm_bn<EPI_F32>(bn, a, lda, b, ldb, M, N, K, D, ldd, bias, err, st);
    case EPI_F32_ADD: return launch_gemm_bn<EPI_F32_ADD>(bn, a, lda, b, ldb, M, N, K, D, ldd, bias, err, st);
    case EPI_BF16_BIAS: return launch_gemm_bn<EPI_BF16_BIAS>(bn, a, lda, b, ldb, M, N, K, D, ldd, bias, err, st);
    default: return launch_gemm_bn<EPI_BF16_BIAS_RELU>(bn, a, lda, b, ldb, M, N, K, D, ldd, bias, err, st);
    }
}

}  // extern "C"
