// BF16 GEMM core on the 5th-generation tensor cores (tcgen05), used by the 3-D convolutions of the
// learned pressure warm start.
//
// One block of 128 threads computes a 128 x N tile of C = A * B^T (FP32 accumulation in tensor
// memory). The K dimension is consumed in chunks of 64: the block's threads gather the A chunk
// (128 x 64) and the B chunk (N x 64) into shared memory in the canonical no-swizzle core-matrix
// layout (8 rows x 16 bytes per core matrix), one elected thread issues four
// tcgen05.mma.cta_group::1.kind::f16 (K = 16 each) and commits them to the stage's mbarrier, and the
// threads gather the next chunk into the other stage meanwhile. Operands are K-major (16-byte rows
// hold 8 consecutive K values) or MN-major (16-byte rows hold 8 consecutive M or N values), chosen
// per operand at compile time. The epilogue reads the accumulator with tcgen05.ld (warp w owns rows
// 32w..32w+31).
//
// Every mbarrier wait is bounded: when it runs out the block records error code 4, waits (bounded)
// for its own MMAs, frees its tensor memory and returns.
#pragma once
#include <cuda_bf16.h>
#include "common.cuh"

namespace clb {
namespace tc {

constexpr int TC_THREADS = 128;
constexpr int TC_M = 128;
constexpr int TC_KC = 64;                    // K per chunk
constexpr int TC_WAIT_LIMIT = 1 << 22;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor: no swizzle, Blackwell version field = 1.
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo_bytes, uint32_t sbo_bytes) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo_bytes >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo_bytes >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1u << 46;
    return d;
}

// Instruction descriptor of kind::f16 with BF16 A and B and an FP32 accumulator.
__host__ __device__ constexpr uint32_t instr_desc(int M, int N, bool a_mn_major, bool b_mn_major) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((a_mn_major ? 1u : 0u) << 15) | ((b_mn_major ? 1u : 0u) << 16) |
           ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred P;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, P;\n\t}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0u;
}

__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
    for (int i = 0; i < TC_WAIT_LIMIT; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

__device__ __forceinline__ void fence_proxy_async() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_alloc(uint32_t* dst_smem, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst_smem)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

// 32 lanes x 16 columns of FP32 from tensor memory (row = lane of the calling warp's quarter).
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int q = 0; q < 16; ++q) v[q] = __uint_as_float(r[q]);
}

// Byte offset of element (row, k) of a K-major chunk (rows x TC_KC): core matrices of 8 rows x 8 K,
// K groups adjacent (LBO = 128 B), row groups TC_KC/8 core matrices apart (SBO = 1024 B).
__device__ __forceinline__ uint32_t kmajor_off(int row, int kvec) {  // kvec = k / 8
    return (uint32_t)((((row >> 3) * (TC_KC / 8) + kvec) << 7) + ((row & 7) << 4));
}
// Byte offset of the 16-byte row holding elements (mn..mn+7, k) of an MN-major chunk
// (MN x TC_KC): K groups adjacent (LBO = 128 B), MN groups TC_KC/8 core matrices apart (SBO = 1024 B).
__device__ __forceinline__ uint32_t mnmajor_off(int mnvec, int k) {  // mnvec = mn / 8
    return (uint32_t)(((mnvec * (TC_KC / 8) + (k >> 3)) << 7) + ((k & 7) << 4));
}
constexpr uint32_t TC_LBO = 128, TC_SBO = 128 * (TC_KC / 8);

// Generic pipelined tile GEMM. Op supplies:
//   static constexpr bool A_MN, B_MN;            operand majors
//   __device__ void gather_a(uint8_t* stage, int chunk) const   fill a 128 x TC_KC chunk
//   __device__ void gather_b(uint8_t* stage, int chunk) const   fill an N x TC_KC chunk
//   __device__ void epilogue(int row, const float* acc, int col0) const  16 columns of one row
//   int chunks;                                   number of K chunks
template <class Op, int N>
__device__ __forceinline__ void tile_gemm(const Op& op, uint8_t* smem) {
    static_assert(N % 16 == 0 && N >= 16 && N <= 256, "N must be a multiple of 16 in [16, 256]");
    constexpr uint32_t A_BYTES = TC_M * TC_KC * 2, B_BYTES = N * TC_KC * 2;
    constexpr uint32_t NCOLS = N <= 32 ? 32 : (N <= 64 ? 64 : (N <= 128 ? 128 : 256));
    uint8_t* a_stage[2] = {smem, smem + A_BYTES};
    uint8_t* b_stage[2] = {smem + 2 * A_BYTES, smem + 2 * A_BYTES + B_BYTES};
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + 2 * A_BYTES + 2 * B_BYTES);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2);
    const int warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        fence_mbar_init();
    }
    if (warp == 0) tmem_alloc(tmem_slot, NCOLS);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    constexpr uint32_t idesc = instr_desc(TC_M, N, Op::A_MN, Op::B_MN);
    bool ok = true;
    const int chunks = op.chunks;
    for (int c = 0; c < chunks && ok; ++c) {
        const int s = c & 1;
        // one thread polls the barrier; the others wait at __syncthreads without taking issue slots
        if (c >= 2)
            ok = __syncthreads_and(threadIdx.x == 0 ? mbar_wait(&bars[s], (uint32_t)(((c - 2) >> 1) & 1)) : true) != 0;
        if (!ok) break;  // uniform across the block
        op.gather_a(a_stage[s], c);
        op.gather_b(b_stage[s], c);
        fence_proxy_async();
        __syncthreads();
        if (threadIdx.x == 0) {
            tc_fence_after();
            const uint32_t a0 = smem_u32(a_stage[s]), b0 = smem_u32(b_stage[s]);
#pragma unroll
            for (int ks = 0; ks < TC_KC / 16; ++ks) {
                // K step ks covers K groups 2ks and 2ks+1: 256 bytes further along K in both layouts
                const uint64_t ad = smem_desc(a0 + ks * 256, TC_LBO, TC_SBO);
                const uint64_t bd = smem_desc(b0 + ks * 256, TC_LBO, TC_SBO);
                mma_bf16(tmem, ad, bd, idesc, (c > 0 || ks > 0) ? 1u : 0u);
            }
            mma_commit(&bars[s]);
        }
    }
    if (ok && chunks > 0)
        ok = __syncthreads_and(threadIdx.x == 0 ? mbar_wait(&bars[(chunks - 1) & 1], (uint32_t)(((chunks - 1) >> 1) & 1))
                                                : true) != 0;
    if (!ok) {
        if (threadIdx.x == 0) {
            raise_device_error(4u);
            // let MMAs already issued finish before the memory they use is released
            mbar_wait(&bars[0], 0);
            mbar_wait(&bars[1], 0);
        }
        __syncthreads();
    }
    tc_fence_after();
    if (ok && chunks > 0 && warp < 4) {
        const int row = warp * 32 + (threadIdx.x & 31);
#pragma unroll
        for (int col = 0; col < N; col += 16) {
            float v[16];
            tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)col, v);
            op.epilogue(row, v, col);
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, NCOLS);
}

template <int N>
constexpr size_t tile_smem_bytes() {
    return 2 * (size_t)TC_M * TC_KC * 2 + 2 * (size_t)N * TC_KC * 2 + 16 + 16;
}

// ---- plain GEMM used to validate the operand layouts: C[M x N] = A[M x K] * B[N x K]^T ----------
// A_MN/B_MN = false: A and B are row-major [rows][K] (K-major); true: stored [K][rows] (MN-major).
template <bool AMN, bool BMN, int N>
struct TestGemm {
    static constexpr bool A_MN = AMN, B_MN = BMN;
    const __nv_bfloat16* a;
    const __nv_bfloat16* b;
    float* c;
    int M, K, m0, chunks;
    __device__ void gather_a(uint8_t* st, int chunk) const {
        const int k0 = chunk * TC_KC;
        if (!AMN) {
            for (int t = threadIdx.x; t < TC_M * (TC_KC / 8); t += TC_THREADS) {
                const int row = t / (TC_KC / 8), kv = t % (TC_KC / 8);
                uint4 val = make_uint4(0, 0, 0, 0);
                const int m = m0 + row, k = k0 + kv * 8;
                if (m < M && k < K) val = *reinterpret_cast<const uint4*>(a + (i64)m * K + k);
                *reinterpret_cast<uint4*>(st + kmajor_off(row, kv)) = val;
            }
        } else {
            for (int t = threadIdx.x; t < (TC_M / 8) * TC_KC; t += TC_THREADS) {
                const int mv = t % (TC_M / 8), kk = t / (TC_M / 8);
                uint4 val = make_uint4(0, 0, 0, 0);
                const int m = m0 + mv * 8, k = k0 + kk;
                if (m < M && k < K) val = *reinterpret_cast<const uint4*>(a + (i64)k * M + m);
                *reinterpret_cast<uint4*>(st + mnmajor_off(mv, kk)) = val;
            }
        }
    }
    __device__ void gather_b(uint8_t* st, int chunk) const {
        const int k0 = chunk * TC_KC;
        if (!BMN) {
            for (int t = threadIdx.x; t < N * (TC_KC / 8); t += TC_THREADS) {
                const int row = t / (TC_KC / 8), kv = t % (TC_KC / 8);
                uint4 val = make_uint4(0, 0, 0, 0);
                const int k = k0 + kv * 8;
                if (k < K) val = *reinterpret_cast<const uint4*>(b + (i64)row * K + k);
                *reinterpret_cast<uint4*>(st + kmajor_off(row, kv)) = val;
            }
        } else {
            for (int t = threadIdx.x; t < (N / 8) * TC_KC; t += TC_THREADS) {
                const int nv = t % (N / 8), kk = t / (N / 8);
                uint4 val = make_uint4(0, 0, 0, 0);
                const int k = k0 + kk;
                if (k < K) val = *reinterpret_cast<const uint4*>(b + (i64)k * N + nv * 8);
                *reinterpret_cast<uint4*>(st + mnmajor_off(nv, kk)) = val;
            }
        }
    }
    __device__ void epilogue(int row, const float* acc, int col0) const {
        const int m = m0 + row;
        if (m >= M) return;
#pragma unroll
        for (int q = 0; q < 16; ++q) c[(i64)m * N + col0 + q] = acc[q];
    }
};

template <bool AMN, bool BMN, int N>
__global__ void __launch_bounds__(TC_THREADS) k_tc_test_gemm(const __nv_bfloat16* a, const __nv_bfloat16* b, float* c,
                                                              int M, int K) {
    extern __shared__ __align__(1024) uint8_t smem[];
    TestGemm<AMN, BMN, N> op{a, b, c, M, K, (int)blockIdx.x * TC_M, (K + TC_KC - 1) / TC_KC};
    tile_gemm<TestGemm<AMN, BMN, N>, N>(op, smem);
}

}  // namespace tc
}  // namespace clb
