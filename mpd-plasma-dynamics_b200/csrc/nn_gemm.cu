// BF16 tensor-core GEMM on the 5th-generation tensor cores (tcgen05) of
// sm_100a, for the surrogate network's training and inference.
//
//   C[b](m, n) = alpha * sum_k bf16(A[b](m, k)) * bf16(B[b](n, k)) + beta * C[b](m, n)
//
// A, B and C are FP32 in global memory with arbitrary element strides (so a
// transposed operand costs nothing extra); operands are rounded to BF16 in
// shared memory, products accumulate in FP32 in tensor memory (TMEM).  One
// CTA of 4 warps computes a 128 x 64 tile of C through a software pipeline
// over 32-wide K chunks:
//   * copies: the FP32 tiles of chunk k + 2 are fetched into a 3-stage
//     shared-memory ring with 16-byte cp.async copies (zero-filled past the
//     operand's edge) while chunk k is converted and chunk k - 1 multiplied;
//     an operand whose K or M/N direction is contiguous and 16-byte aligned
//     is copied as it lies (K-major rows or MN-major rows), any other one
//     element by element;
//   * conversion: every thread rounds its share of chunk k to BF16 and
//     writes it in the canonical K-major, no-swizzle layout of 8 x 16-byte
//     core matrices (double-buffered);
//   * MMA: one thread issues two tcgen05.mma.cta_group::1.kind::f16
//     (M 128, N 64, K 16) per chunk from shared-memory descriptors and
//     commits them to an mbarrier (bounded wait before the buffer is reused);
//   * warp 0 allocates 64 TMEM columns (the 128 x 64 FP32 accumulator); the
//     epilogue reads it with tcgen05.ld (each warp its 32 TMEM lanes = 32
//     rows of C) into shared memory and writes alpha * acc + beta * C along
//     C's contiguous direction (whole 128-byte lines per warp).
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
constexpr int kTileK = 32;          // K per pipeline chunk (two MMAs of K 16)
constexpr int kSplitUnit = 64;      // split-K spans are multiples of this
constexpr int kGemmThreads = 128;
constexpr int kCopyStages = 3;      // FP32 chunks in flight per CTA
constexpr uint32_t kTmemCols = 64;

// Bytes of the BF16 core-matrix layouts: A tile = 4 K-chunks x 16 row
// groups, B tile = 4 K-chunks x 8 row groups, 128 bytes per core matrix.
constexpr int kABytes = kTileM * kTileK * 2;
constexpr int kBBytes = kTileN * kTileK * 2;
// FP32 staging of one chunk: K-major tiles as [row][32 k + 4 padding] (the
// padding spreads a warp's 16-byte reads of consecutive rows over all
// banks), MN-major tiles as [k][rows].
constexpr int kKPad = kTileK + 4;
constexpr int kA32 = (kTileM * kKPad > kTileK * kTileM) ? kTileM * kKPad : kTileK * kTileM;
constexpr int kB32 = (kTileN * kKPad > kTileK * kTileN) ? kTileN * kKPad : kTileK * kTileN;

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

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    __nv_bfloat162 h = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t *>(&h);
}

// 16-byte asynchronous copy global -> shared; bytes past src_bytes (0..16)
// are zero-filled, and with src_bytes == 0 nothing is read.
__device__ __forceinline__ void cp_async16(uint32_t dst, const void *src, int src_bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src),
                 "r"(src_bytes)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
    asm volatile("cp.async.commit_group;" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// How an operand's FP32 tile is staged: rows of K (K contiguous in memory),
// rows of M or N (those contiguous), or element by element.
enum StageMode { kKMajor = 0, kMNMajor = 1, kScalar = 2 };

__device__ __forceinline__ int stage_mode(const float *base, long long s_rows, long long s_k) {
    const bool aligned = ((uintptr_t)base & 15) == 0;
    if (s_k == 1 && aligned && (s_rows % 4) == 0) return kKMajor;
    if (s_rows == 1 && aligned && (s_k % 4) == 0) return kMNMajor;
    return kScalar;
}

// Fetch rows [r0, r0 + ROWS) x k [k0, k0 + 32) of an operand into FP32
// staging: kKMajor as [row][kKPad], kMNMajor and kScalar as [k][ROWS rows].
// Past nrows or k1 the values are zero.  kScalar loads synchronously.
template <int ROWS>
__device__ __forceinline__ void fetch(float *dst, const float *base, long long sr, long long sk,
                                      int nrows, int k1, int r0, int k0, int mode) {
    if (mode == kKMajor) {
        constexpr int kChunks = ROWS * (kTileK / 4);
#pragma unroll
        for (int i = 0; i < kChunks / kGemmThreads; ++i) {
            const int u = threadIdx.x + i * kGemmThreads;
            const int rl = u / (kTileK / 4), c = u % (kTileK / 4);
            const int r = r0 + rl, k = k0 + 4 * c;
            const int valid = (r < nrows && k < k1) ? 4 * min(4, k1 - k) : 0;
            const float *src = valid ? base + (long long)r * sr + k : base;
            cp_async16(smem_addr(dst + rl * kKPad + 4 * c), src, valid);
        }
    } else if (mode == kMNMajor) {
        constexpr int kChunks = kTileK * (ROWS / 4);
#pragma unroll
        for (int i = 0; i < kChunks / kGemmThreads; ++i) {
            const int u = threadIdx.x + i * kGemmThreads;
            const int kl = u / (ROWS / 4), c = u % (ROWS / 4);
            const int k = k0 + kl, r = r0 + 4 * c;
            const int valid = (k < k1 && r < nrows) ? 4 * min(4, nrows - r) : 0;
            const float *src = valid ? base + (long long)k * sk + r : base;
            cp_async16(smem_addr(dst + kl * ROWS + 4 * c), src, valid);
        }
    } else {
#pragma unroll 4
        for (int u = threadIdx.x; u < ROWS * kTileK; u += kGemmThreads) {
            const int kl = u / ROWS, rl = u % ROWS;
            const int r = r0 + rl, k = k0 + kl;
            dst[kl * ROWS + rl] =
                (r < nrows && k < k1) ? __ldg(base + (long long)r * sr + (long long)k * sk) : 0.0f;
        }
    }
}

// Round the FP32 staging of a chunk to BF16 in the K-major core-matrix
// layout: 8-k chunk c of row group g at (c * ROWS/8 + g) * 128 bytes, row
// r & 7 at 16 (r & 7), element e at 2 e.
template <int ROWS>
__device__ __forceinline__ void convert(unsigned char *dst, const float *src, int mode) {
    constexpr int kUnits = ROWS * (kTileK / 8);
#pragma unroll
    for (int i = 0; i < kUnits / kGemmThreads; ++i) {
        const int u = threadIdx.x + i * kGemmThreads;
        const int rl = u % ROWS, c = u / ROWS;  // consecutive threads: consecutive rows
        float f[8];
        if (mode == kKMajor) {
            const float4 a = *reinterpret_cast<const float4 *>(src + rl * kKPad + 8 * c);
            const float4 b = *reinterpret_cast<const float4 *>(src + rl * kKPad + 8 * c + 4);
            f[0] = a.x; f[1] = a.y; f[2] = a.z; f[3] = a.w;
            f[4] = b.x; f[5] = b.y; f[6] = b.z; f[7] = b.w;
        } else {
#pragma unroll
            for (int e = 0; e < 8; ++e) f[e] = src[(8 * c + e) * ROWS + rl];
        }
        uint4 v;
        v.x = pack_bf16(f[0], f[1]);
        v.y = pack_bf16(f[2], f[3]);
        v.z = pack_bf16(f[4], f[5]);
        v.w = pack_bf16(f[6], f[7]);
        *reinterpret_cast<uint4 *>(dst + (c * (ROWS / 8) + (rl >> 3)) * 128 + (rl & 7) * 16) = v;
    }
}

// Dynamic shared memory: the FP32 staging ring, then two BF16 buffers.
constexpr int kStage32Bytes = (kA32 + kB32) * 4;
constexpr int kStageBytes = kABytes + kBBytes;
constexpr int kGemmSmem = kCopyStages * kStage32Bytes + 2 * kStageBytes;

// C tile (m0, n0) of batch b over K range [k_begin, k_end).  With ksplit > 1
// the raw FP32 sums go to work (split s of batch b: dense M x N at
// ((s * batch + b) * M * N)) and nn_gemm_reduce_kernel finishes C.
__global__ void __launch_bounds__(kGemmThreads) nn_gemm_kernel(const mpd_gemm_desc d, int ksplit,
                                                               int kspan) {
    extern __shared__ __align__(1024) unsigned char gemm_smem[];
    __shared__ __align__(8) uint64_t bar[2];
    __shared__ uint32_t tmem_slot;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m0 = blockIdx.x * kTileM, n0 = blockIdx.y * kTileN;
    const int b = blockIdx.z % d.batch, split = blockIdx.z / d.batch;
    const int k_begin = split * kspan;
    const int k_end = min(d.K, k_begin + kspan);
    const float *A = d.A + (long long)b * d.sab;
    const float *B = d.B + (long long)b * d.sbb;
    const int mode_a = stage_mode(A, d.sam, d.sak);
    const int mode_b = stage_mode(B, d.sbn, d.sbk);
    float *ring = reinterpret_cast<float *>(gemm_smem);
    unsigned char *bf = gemm_smem + kCopyStages * kStage32Bytes;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_addr(&tmem_slot)),
                     "r"(kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (threadIdx.x == 0) {
        mbar_init(smem_addr(&bar[0]), 1);
        mbar_init(smem_addr(&bar[1]), 1);
        mbar_init_fence();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_slot;

    const int nchunks = k_end > k_begin ? (k_end - k_begin + kTileK - 1) / kTileK : 0;
    auto fetch_chunk = [&](int kc) {
        float *st = ring + (kc % kCopyStages) * (kA32 + kB32);
        const int k0 = k_begin + kc * kTileK;
        fetch<kTileM>(st, A, d.sam, d.sak, d.M, k_end, m0, k0, mode_a);
        fetch<kTileN>(st + kA32, B, d.sbn, d.sbk, d.N, k_end, n0, k0, mode_b);
    };
    // prologue: chunks 0 .. kCopyStages-2 in flight, one commit group each
#pragma unroll
    for (int kc = 0; kc < kCopyStages - 1; ++kc) {
        if (kc < nchunks) fetch_chunk(kc);
        cp_async_commit();
    }
    bool ok = true;
    for (int kc = 0; kc < nchunks; ++kc) {
        // the stage chunk kc + 2 lands in held chunk kc - 1, converted last iteration
        if (kc + kCopyStages - 1 < nchunks) fetch_chunk(kc + kCopyStages - 1);
        cp_async_commit();
        cp_async_wait<kCopyStages - 1>();   // this thread's copies of chunk kc are in
        const int buf = kc & 1;
        if (kc >= 2) {
            // the MMAs of chunk kc - 2 read this BF16 buffer: wait for their commit
            const bool arrived = mbar_wait_bounded(smem_addr(&bar[buf]), ((kc - 2) >> 1) & 1);
            ok = __syncthreads_and(arrived);
            if (!ok) break;
        } else {
            __syncthreads();
        }
        const float *st = ring + (kc % kCopyStages) * (kA32 + kB32);
        unsigned char *sA = bf + buf * kStageBytes;
        unsigned char *sB = sA + kABytes;
        convert<kTileM>(sA, st, mode_a);
        convert<kTileN>(sB, st + kA32, mode_b);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (threadIdx.x == 0) {
            tc_fence_after();
            const uint32_t a_addr = smem_addr(sA), b_addr = smem_addr(sB);
#pragma unroll
            for (int s2 = 0; s2 < kTileK / 16; ++s2) {
                // K slice s2 = core-matrix chunks 2 s2, 2 s2 + 1
                const uint64_t ad = smem_desc(a_addr + s2 * 2 * (kTileM / 8) * 128,
                                              (kTileM / 8) * 128, 128);
                const uint64_t bd = smem_desc(b_addr + s2 * 2 * (kTileN / 8) * 128,
                                              (kTileN / 8) * 128, 128);
                mma_bf16(tmem, ad, bd, (kc > 0 || s2 > 0) ? 1u : 0u);
            }
            mma_commit(smem_addr(&bar[buf]));
        }
    }
    cp_async_wait<0>();  // no copy may still land after the CTA exits
    if (ok && nchunks > 0) {
        // commits complete in order: the last one covers every MMA
        const int last = nchunks - 1;
        ok = __syncthreads_and(mbar_wait_bounded(smem_addr(&bar[last & 1]), (last >> 1) & 1));
    }
    tc_fence_after();
    if (ok) {
        // The accumulator through shared memory (the copy ring is free now):
        // tcgen05.ld gives each thread one row of the tile; the tile is then
        // written along C's contiguous direction, so a warp's stores (and,
        // with beta != 0, its loads of C) are whole 128-byte lines.
        float *T = ring;              // kTileM x kTilePad floats
        constexpr int kTilePad = kTileN + 1;   // odd stride: conflict-free rows and columns
        const int row = warp * 32 + lane;
#pragma unroll
        for (int j = 0; j < kTileN / 16; ++j) {
            float v[16];
            if (nchunks > 0) {
                tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(16 * j), v);
            } else {
#pragma unroll
                for (int i = 0; i < 16; ++i) v[i] = 0.0f;
            }
#pragma unroll
            for (int i = 0; i < 16; ++i) T[row * kTilePad + 16 * j + i] = v[i];
        }
        __syncthreads();
        float *C = d.C + (long long)b * d.scb;
        float *W = ksplit > 1 ? d.work + ((long long)split * d.batch + b) * d.M * d.N : nullptr;
        // In both directions a warp takes 8 rows (or columns) at a time and
        // issues all its loads of C before any store: a store to C and a
        // later load of C are not reordered, so one element at a time would
        // serialise on the memory latency.  Every element of C is read and
        // written by one thread only, so its loads may use the read-only path.
        constexpr int kBatch = 8;
        if (W || d.scn == 1 || d.scm != 1) {
            // lanes along n: rows of C (or of the dense partials) are contiguous
            for (int r0 = warp; r0 < kTileM; r0 += kBatch * (kGemmThreads / 32)) {
                float cin[kBatch][kTileN / 32];
#pragma unroll
                for (int j = 0; j < kBatch; ++j) {
#pragma unroll
                    for (int h2 = 0; h2 < kTileN / 32; ++h2) {
                        const int m = m0 + r0 + j * (kGemmThreads / 32);
                        const int n = n0 + lane + 32 * h2;
                        cin[j][h2] = (!W && d.beta != 0.0f && m < d.M && n < d.N)
                                         ? __ldg(C + (long long)m * d.scm + (long long)n * d.scn)
                                         : 0.0f;
                    }
                }
#pragma unroll
                for (int j = 0; j < kBatch; ++j) {
#pragma unroll
                    for (int h2 = 0; h2 < kTileN / 32; ++h2) {
                        const int r = r0 + j * (kGemmThreads / 32), cc = lane + 32 * h2;
                        const int m = m0 + r, n = n0 + cc;
                        if (m >= d.M || n >= d.N) continue;
                        const float v = T[r * kTilePad + cc];
                        if (W)
                            W[(long long)m * d.N + n] = v;
                        else
                            C[(long long)m * d.scm + (long long)n * d.scn] =
                                d.alpha * v + d.beta * cin[j][h2];
                    }
                }
            }
        } else {
            // lanes along m: columns of C are contiguous
            for (int c0 = warp; c0 < kTileN; c0 += kBatch * (kGemmThreads / 32)) {
                float cin[kBatch][kTileM / 32];
#pragma unroll
                for (int j = 0; j < kBatch; ++j) {
#pragma unroll
                    for (int h2 = 0; h2 < kTileM / 32; ++h2) {
                        const int n = n0 + c0 + j * (kGemmThreads / 32);
                        const int m = m0 + lane + 32 * h2;
                        cin[j][h2] = (d.beta != 0.0f && m < d.M && n < d.N)
                                         ? __ldg(C + (long long)m * d.scm + (long long)n * d.scn)
                                         : 0.0f;
                    }
                }
#pragma unroll
                for (int j = 0; j < kBatch; ++j) {
#pragma unroll
                    for (int h2 = 0; h2 < kTileM / 32; ++h2) {
                        const int cc = c0 + j * (kGemmThreads / 32), r = lane + 32 * h2;
                        const int m = m0 + r, n = n0 + cc;
                        if (m >= d.M || n >= d.N) continue;
                        const float v = T[r * kTilePad + cc];
                        C[(long long)m * d.scm + (long long)n * d.scn] =
                            d.alpha * v + d.beta * cin[j][h2];
                    }
                }
            }
        }
    } else if (threadIdx.x == 0) {
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

// C = alpha * (sum of the ksplit partials, in split order) + beta * C.
__global__ void nn_gemm_reduce_kernel(const mpd_gemm_desc d, int ksplit) {
    const long long mn = (long long)d.M * d.N, total = mn * d.batch;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const int b = (int)(t / mn);
        const long long e = t % mn;
        const int m = (int)(e / d.N), n = (int)(e % d.N);
        float s = 0.0f;
        for (int k = 0; k < ksplit; ++k) s += d.work[((long long)k * d.batch + b) * mn + e];
        float *c = d.C + (long long)b * d.scb + (long long)m * d.scm + (long long)n * d.scn;
        *c = d.beta == 0.0f ? d.alpha * s : d.alpha * s + d.beta * *c;
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
    // split K when the tiles alone leave most SMs idle and the caller gave
    // room for the partial sums (summed in split order afterwards)
    const long long tiles = (long long)((d->M + kTileM - 1) / kTileM) *
                            ((d->N + kTileN - 1) / kTileN) * d->batch;
    int ksplit = 1;
    if (d->work && tiles < 296 && d->K >= 4 * kSplitUnit) {
        long long want = (296 + tiles - 1) / tiles;
        const long long by_k = d->K / (2 * kSplitUnit);
        const long long by_room = d->work_floats / ((long long)d->M * d->N * d->batch);
        want = want < by_k ? want : by_k;
        want = want < by_room ? want : by_room;
        want = want < 64 ? want : 64;
        if (want > 1) ksplit = (int)want;
    }
    const int kspan =
        ((d->K + ksplit - 1) / ksplit + kSplitUnit - 1) / kSplitUnit * kSplitUnit;
    ksplit = (d->K + kspan - 1) / kspan;
    if ((long long)d->batch * ksplit > 65535) {
        mpd::SetLastError("mpd_nn_gemm: batch too large for one launch");
        return MPD_ERR_INVALID;
    }
    const dim3 grid((d->M + kTileM - 1) / kTileM, (d->N + kTileN - 1) / kTileN,
                    d->batch * ksplit);
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
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    nn_gemm_kernel<<<grid, kGemmThreads, kGemmSmem, st>>>(*d, ksplit, kspan);
    if (ksplit > 1) {
        const long long total = (long long)d->M * d->N * d->batch;
        long long blocks = (total + 255) / 256;
        if (blocks > 148 * 16) blocks = 148 * 16;
        nn_gemm_reduce_kernel<<<(int)blocks, 256, 0, st>>>(*d, ksplit);
    }
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
