// BF16 tensor-core GEMM on the 5th-generation tensor cores (tcgen05) of
// sm_100a, for the surrogate network's training and inference.
//
//   C[b](m, n) = alpha * sum_k bf16(A[b](m, k)) * bf16(B[b](n, k)) + beta * C[b](m, n)
//
// A, B and C are FP32 in global memory with arbitrary element strides (so a
// transposed operand costs nothing extra); operands are rounded to BF16 as
// they are staged in shared memory, products accumulate in FP32 in tensor
// memory (TMEM).  One CTA of 4 warps computes a 128 x 64 tile of C:
//   * warp 0 allocates 64 TMEM columns (the 128 x 64 FP32 accumulator);
//   * per 64-wide K chunk every thread converts its share of the A (128 x 64)
//     and B (64 x 64) tiles into the canonical K-major, no-swizzle layout of
//     8 x 16-byte core matrices, then one thread issues four
//     tcgen05.mma.cta_group::1.kind::f16 (M 128, N 64, K 16) from shared-
//     memory descriptors and commits them to an mbarrier (bounded wait);
//   * the epilogue reads the accumulator with tcgen05.ld (each warp its 32
//     TMEM lanes = 32 rows of C) and writes alpha * acc + beta * C.
// Shared-memory descriptor and instruction-descriptor fields follow the
// sm100 UMMA descriptors (start address >> 4 in bits 0-13, leading byte
// offset >> 4 in 16-29, stride byte offset >> 4 in 32-45, version 1 in
// 46-47, layout 0 = no swizzle in 61-63; instruction: FP32 accumulate,
// BF16 A and B, both K-major, N >> 3 in bits 17-22, M >> 4 in 24-28).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "../../include/mpd_b200.h"
#include "tma.cuh"

namespace mpd {
void SetLastError(const std::string &msg);
}

namespace {

using mpd::mbar_init;
using mpd::mbar_init_fence;
using mpd::mbar_wait_bounded;
using mpd::smem_addr;

constexpr int kTileM = 128;
constexpr int kTileN = 64;
constexpr int kTileK = 64;
constexpr int kGemmThreads = 128;
constexpr uint32_t kTmemCols = 64;

// Bytes of the core-matrix layouts: A tile = 8 K-chunks x 16 row groups,
// B tile = 8 K-chunks x 8 row groups, 128 bytes per core matrix.
constexpr int kABytes = kTileM * kTileK * 2;
constexpr int kBBytes = kTileN * kTileK * 2;

__device__ int g_gemm_wait_fail = 0;

__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1u << 46;  // descriptor version of sm100
    return d;                 // base offset 0, no swizzle
}

// FP32 accumulate, BF16 x BF16, K-major A and B, M = 128, N = 64.
constexpr uint32_t kInstrDesc = (1u << 4) | (1u << 7) | (1u << 10) |
                                ((uint32_t)(kTileN >> 3) << 17) | ((uint32_t)(kTileM >> 4) << 24);

__device__ __forceinline__ void tc_fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                         uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
        ::"r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(kInstrDesc), "r"(accumulate)
        : "memory");
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
    asm volatile(
        "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
        : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float v[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
        "%11, %12, %13, %14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
          "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// 8 consecutive-k elements of one operand row as BF16, packed for one
// 16-byte core-matrix row (element e in bytes 2e..2e+1).
__device__ __forceinline__ uint4 load8_bf16(const float *p, long long sk, int kvalid) {
    float f[8];
#pragma unroll
    for (int e = 0; e < 8; ++e) f[e] = e < kvalid ? __ldg(p + (long long)e * sk) : 0.0f;
    uint4 out;
    __nv_bfloat162 h;
    h = __floats2bfloat162_rn(f[0], f[1]);
    out.x = *reinterpret_cast<uint32_t *>(&h);
    h = __floats2bfloat162_rn(f[2], f[3]);
    out.y = *reinterpret_cast<uint32_t *>(&h);
    h = __floats2bfloat162_rn(f[4], f[5]);
    out.z = *reinterpret_cast<uint32_t *>(&h);
    h = __floats2bfloat162_rn(f[6], f[7]);
    out.w = *reinterpret_cast<uint32_t *>(&h);
    return out;
}

// Stage rows [r0, r0 + ROWS) x k [k0, k0 + 64) of an operand into the
// core-matrix layout: chunk c (8 k) of row group g at (c * ROWS/8 + g) * 128.
template <int ROWS>
__device__ __forceinline__ void stage(unsigned char *dst, const float *base, long long sr,
                                      long long sk, int nrows, int K, int r0, int k0) {
    constexpr int kUnits = ROWS * (kTileK / 8);
    const bool k_contig = sk == 1;
    for (int u = threadIdx.x; u < kUnits; u += kGemmThreads) {
        int rl, c;
        if (k_contig) {
            c = u & 7;
            rl = u >> 3;
        } else {
            rl = u % ROWS;
            c = u / ROWS;
        }
        const int r = r0 + rl, k = k0 + 8 * c;
        uint4 v = make_uint4(0u, 0u, 0u, 0u);
        if (r < nrows && k < K) v = load8_bf16(base + (long long)r * sr + (long long)k * sk, sk, K - k);
        *reinterpret_cast<uint4 *>(dst + (c * (ROWS / 8) + (rl >> 3)) * 128 + (rl & 7) * 16) = v;
    }
}

// The two tiles in dynamic shared memory (24 KB per block).
constexpr int kASpan = kABytes;
constexpr int kBSpan = kBBytes;
constexpr int kGemmSmem = kASpan + kBSpan;
static_assert(kABytes <= kASpan && kBBytes <= kBSpan, "tile spans");

__global__ void __launch_bounds__(kGemmThreads) nn_gemm_kernel(const mpd_gemm_desc d) {
    extern __shared__ __align__(1024) unsigned char gemm_smem[];
    unsigned char *sA = gemm_smem;
    unsigned char *sB = gemm_smem + kASpan;
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t tmem_slot;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m0 = blockIdx.x * kTileM, n0 = blockIdx.y * kTileN, b = blockIdx.z;
    const float *A = d.A + (long long)b * d.sab;
    const float *B = d.B + (long long)b * d.sbb;
    float *C = d.C + (long long)b * d.scb;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_addr(&tmem_slot)),
                     "r"(kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (threadIdx.x == 0) {
        mbar_init(smem_addr(&bar), 1);
        mbar_init_fence();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_slot;
    const uint32_t a_addr = smem_addr(sA), b_addr = smem_addr(sB);

    bool ok = true;
    const int nchunks = (d.K + kTileK - 1) / kTileK;
    for (int kc = 0; kc < nchunks; ++kc) {
        stage<kTileM>(sA, A, d.sam, d.sak, d.M, d.K, m0, kc * kTileK);
        stage<kTileN>(sB, B, d.sbn, d.sbk, d.N, d.K, n0, kc * kTileK);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (threadIdx.x == 0) {
            tc_fence_after();
#pragma unroll
            for (int s = 0; s < kTileK / 16; ++s) {
                // K slice s = core-matrix chunks 2s, 2s+1
                const uint64_t ad = smem_desc(a_addr + s * 2 * (kTileM / 8) * 128,
                                              (kTileM / 8) * 128, 128);
                const uint64_t bd = smem_desc(b_addr + s * 2 * (kTileN / 8) * 128,
                                              (kTileN / 8) * 128, 128);
                mma_bf16(tmem, ad, bd, (kc > 0 || s > 0) ? 1u : 0u);
            }
            mma_commit(smem_addr(&bar));
        }
        // the tiles may be overwritten once the MMAs that read them are done
        const bool arrived = mbar_wait_bounded(smem_addr(&bar), kc & 1);
        ok = __syncthreads_and(arrived);
        if (!ok) break;
    }
    tc_fence_after();
    if (ok && nchunks > 0) {
        const int m = m0 + warp * 32 + lane;
#pragma unroll
        for (int j = 0; j < kTileN / 16; ++j) {
            float v[16];
            tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(16 * j), v);
            if (m < d.M) {
#pragma unroll
                for (int i = 0; i < 16; ++i) {
                    const int n = n0 + 16 * j + i;
                    if (n < d.N) {
                        float *c = C + (long long)m * d.scm + (long long)n * d.scn;
                        *c = d.beta == 0.0f ? d.alpha * v[i] : d.alpha * v[i] + d.beta * *c;
                    }
                }
            }
        }
    } else if (!ok && threadIdx.x == 0) {
        atomicExch(&g_gemm_wait_fail, 1);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                     "r"(kTmemCols)
                     : "memory");
    }
}

}  // namespace

extern "C" {

int mpd_nn_gemm(const mpd_gemm_desc *d, void *stream) {
    if (!d || !d->A || !d->B || !d->C) {
        mpd::SetLastError("mpd_nn_gemm: NULL descriptor or operand");
        return MPD_ERR_INVALID;
    }
    if (d->M < 0 || d->N < 0 || d->K < 1 || d->batch < 0) {
        mpd::SetLastError("mpd_nn_gemm: sizes must be M, N, batch >= 0 and K >= 1");
        return MPD_ERR_INVALID;
    }
    if (d->M == 0 || d->N == 0 || d->batch == 0) return MPD_OK;
    if (d->batch > 65535 || (d->N + kTileN - 1) / kTileN > 65535) {
        mpd::SetLastError("mpd_nn_gemm: batch or N too large for one launch");
        return MPD_ERR_INVALID;
    }
    const dim3 grid((d->M + kTileM - 1) / kTileM, (d->N + kTileN - 1) / kTileN, d->batch);
    static bool attr_set = false;  // per process; the attribute is per function
    if (!attr_set) {
        const cudaError_t ea = cudaFuncSetAttribute(
            nn_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kGemmSmem);
        if (ea != cudaSuccess) {
            mpd::SetLastError(std::string("mpd_nn_gemm: ") + cudaGetErrorString(ea));
            return MPD_ERR_CUDA;
        }
        attr_set = true;
    }
    nn_gemm_kernel<<<grid, kGemmThreads, kGemmSmem, static_cast<cudaStream_t>(stream)>>>(*d);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        mpd::SetLastError(std::string("mpd_nn_gemm: ") + cudaGetErrorString(e));
        return MPD_ERR_CUDA;
    }
    return MPD_OK;
}

int mpd_nn_wait_status(void *stream) {
    cudaError_t e = cudaStreamSynchronize(static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) {
        mpd::SetLastError(std::string("mpd_nn_wait_status: ") + cudaGetErrorString(e));
        return MPD_ERR_CUDA;
    }
    int fail = 0;
    e = cudaMemcpyFromSymbol(&fail, g_gemm_wait_fail, sizeof(int));
    if (e != cudaSuccess) {
        mpd::SetLastError(std::string("mpd_nn_wait_status: ") + cudaGetErrorString(e));
        return MPD_ERR_CUDA;
    }
    if (fail) {
        mpd::SetLastError("a tensor-core GEMM's bounded wait gave up; its output is not valid");
        return MPD_ERR_TIMEOUT;
    }
    return MPD_OK;
}

}  // extern "C"
