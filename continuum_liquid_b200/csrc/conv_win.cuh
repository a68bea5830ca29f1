// 3x3x3 convolution (forward and data gradient) as implicit GEMM on tcgen05 with the input tile
// staged once in shared memory and every tap read as a shifted window of it (no per-tap gathers).
//
// A block computes one z slice, TY rows and XT columns of the output for all N output channels.
// For each 16-channel chunk of the source it stages, with cp.async (zero fill outside the volume),
// the source voxels of the three z slices around it, TY + 2 rows and RW = XT + 2 columns, as two
// planes of 16 bytes per voxel (8 channels each) in padded row-major order L = (zz (TY+2) + yy) RW
// + xx, plus the chunk's weights of all 27 taps. In this layout eight consecutive voxels of a plane
// are one 8 x 16-byte core matrix, so the A operand of tap (dz, dy, dx) for 128 consecutive output
// positions is the plane itself seen from a start shifted by (dz (TY+2) + dy) RW + dx voxels: a
// no-swizzle K-major descriptor with SBO = 128 B (next 8 voxels) and LBO = one plane (next 8
// channels). The output positions are the padded rows of the centre slice in M tiles of 128; the
// two halo columns of each row are computed and dropped. One thread issues 27 MMAs (M = 128, K = 16)
// per tile and chunk into the tile's TMEM accumulator; chunks use two stages, so the next chunk is
// staged while the tensor core works. The epilogue reads TMEM with tcgen05.ld and stores each
// voxel's N channels (bias + ReLU fused in the forward pass, the ReLU mask in the data gradient).
//
// Operand rows that belong to dropped positions may read unstaged shared memory; they only feed
// their own (dropped) output rows. Every mbarrier wait is bounded (error code 4, as tile_gemm).
#pragma once
#include "conv3d.cuh"

namespace clb {
namespace conv {

constexpr int CW_THREADS = 256;  // 8 warps: all stage; warps w and w + 4 share TMEM lane quarter w % 4

struct WinPlan {
    int XT, TY, RW;        // output columns and rows per block, padded row length
    int tiles;             // M tiles of 128 positions
    int xtiles, ytiles;    // blocks along x and y
    int P;                 // voxels per plane (the region, its rounding to whole tiles, one slack voxel)
    int Lbeg;              // first position of the M range
    int nq;                // 16-channel chunks of the source
    int a_bytes, b_bytes;  // one stage: two planes; the chunk's weights of all taps
    int stages;            // 1 (single chunk) or 2
    int tmem_cols;         // power of two >= tiles * N
    int smem;              // dynamic shared memory
};

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src, bool valid) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(valid ? 16 : 0)
                 : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

template <int N, bool DGRAD>
__global__ void __launch_bounds__(CW_THREADS) k_conv_win(const __nv_bfloat16* __restrict__ src,
                                                          const __nv_bfloat16* __restrict__ wmat,
                                                          const float* __restrict__ bias,
                                                          const __nv_bfloat16* __restrict__ mask_src,
                                                          __nv_bfloat16* __restrict__ out, Vol g, int Cs, int Kpad,
                                                          int relu, WinPlan pl) {
    static_assert(N % 16 == 0 && N >= 16 && N <= 256, "N must be a multiple of 16 in [16, 256]");
    extern __shared__ __align__(1024) uint8_t smem[];
    using namespace tc;
    int r = blockIdx.x;
    const int xt = r % pl.xtiles;
    r /= pl.xtiles;
    const int yt = r % pl.ytiles;
    r /= pl.ytiles;
    const int z = r % g.D, b = r / g.D;
    const int x0 = xt * pl.XT, y0 = yt * pl.TY;
    const int TY2 = pl.TY + 2, RW = pl.RW;
    uint8_t* stage_a[2] = {smem, smem + (pl.a_bytes + pl.b_bytes)};
    uint8_t* stage_b[2] = {smem + pl.a_bytes, smem + (pl.a_bytes + pl.b_bytes) + pl.a_bytes};
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + pl.stages * (pl.a_bytes + pl.b_bytes));
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2);
    const int warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        fence_mbar_init();
    }
    if (warp == 0) tmem_alloc(tmem_slot, (uint32_t)pl.tmem_cols);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    constexpr uint32_t idesc = instr_desc(TC_M, N, false, false);
    const uint32_t plane_bytes = (uint32_t)pl.P * 16u;

    auto stage = [&](int q, int s) {
        const uint32_t a0 = smem_u32(stage_a[s]), w0 = smem_u32(stage_b[s]);
        const int lane = threadIdx.x & 31;
        for (int rr = warp; rr < 3 * TY2; rr += CW_THREADS / 32) {  // one padded row per warp, lanes along x
            const int zz = rr / TY2, yy = rr - zz * TY2;
            const int gz = z + zz - 1, gy = y0 + yy - 1;
            const bool row_in = gz >= 0 && gz < g.D && gy >= 0 && gy < g.H;
            const i64 row0 = (((i64)b * g.D + (row_in ? gz : 0)) * g.H + (row_in ? gy : 0)) * g.W;
            const uint32_t dst0 = a0 + (uint32_t)(rr * RW + 1) * 16u;
            for (int xx = lane; xx < RW; xx += 32) {
                const int gx = x0 + xx - 1;
                const bool inside = row_in && gx >= 0 && gx < g.W;
                const i64 vox = inside ? row0 + gx : 0;
#pragma unroll
                for (int pln = 0; pln < 2; ++pln) {
                    const int c0 = 16 * q + 8 * pln;
                    const bool ok = inside && c0 < Cs;
                    cp_async16(dst0 + pln * plane_bytes + (uint32_t)xx * 16u, src + vox * Cs + (ok ? c0 : 0), ok);
                }
            }
        }
        for (int t = threadIdx.x; t < 54 * N; t += CW_THREADS) {  // (tap, K group, n)
            const int n = t % N, tk = t / N, kg = tk & 1, tap = tk >> 1;
            const int c0 = 16 * q + 8 * kg;
            const bool ok = c0 < Cs;
            cp_async16(w0 + (uint32_t)t * 16u, wmat + (i64)n * Kpad + tap * Cs + (ok ? c0 : 0), ok);
        }
    };

    bool ok = true;
    for (int q = 0; q < pl.nq && ok; ++q) {
        const int s = q & 1;
        // one thread polls the barrier; the others wait at __syncthreads without taking issue slots
        if (q >= 2)
            ok = __syncthreads_and(threadIdx.x == 0 ? mbar_wait(&bars[s], (uint32_t)(((q - 2) >> 1) & 1)) : true) != 0;
        if (!ok) break;  // uniform across the block
        stage(q, s);
        cp_async_wait_all();
        fence_proxy_async();
        __syncthreads();
        if (threadIdx.x == 0) {
            tc_fence_after();
            // Descriptors are built once: the start-address field counts 16-byte units, so moving the
            // window by `off` voxels (16 bytes each) or to the next tap's weights adds to the descriptor
            // (shared-memory addresses stay below 2^18 bytes, so the 14-bit field never carries).
            const uint64_t a_base = smem_desc(smem_u32(stage_a[s]) + (uint32_t)(pl.Lbeg + 1) * 16u, plane_bytes, 128u);
            const uint64_t b_base = smem_desc(smem_u32(stage_b[s]), (uint32_t)(N * 16), 128u);
            const int slab = TY2 * RW;
            for (int m = 0; m < pl.tiles; ++m) {
                const uint64_t am = a_base + (uint64_t)(m * TC_M);
                const uint32_t dm = tmem + (uint32_t)(m * N);
#pragma unroll
                for (int tap = 0; tap < 27; ++tap) {
                    const int off = (tap / 9 - 1) * slab + ((tap / 3) % 3 - 1) * RW + (tap % 3 - 1);
                    const uint64_t ad = am + (uint64_t)(int64_t)(DGRAD ? -off : off);
                    mma_bf16(dm, ad, b_base + (uint64_t)(tap * 2 * N), idesc, (q > 0 || tap > 0) ? 1u : 0u);
                }
            }
            mma_commit(&bars[s]);
        }
    }
    if (ok && pl.nq > 0)
        ok = __syncthreads_and(threadIdx.x == 0 ? mbar_wait(&bars[(pl.nq - 1) & 1], (uint32_t)(((pl.nq - 1) >> 1) & 1))
                                                : true) != 0;
    if (!ok) {
        if (threadIdx.x == 0) {
            raise_device_error(4u);
            mbar_wait(&bars[0], 0);
            mbar_wait(&bars[1], 0);
        }
        __syncthreads();
    }
    tc_fence_after();
    if (ok) {
        // warp w reads TMEM lanes 32 (w % 4) ...; warps w and w + 4 take alternate 16-column groups
        const int quarter = warp & 3, half = warp >> 2;
        const int row = quarter * 32 + (threadIdx.x & 31);
        for (int m = 0; m < pl.tiles; ++m) {
            const int rel = m * TC_M + row;
            const int y = rel / RW, xx = rel - y * RW;
            const int gy = y0 + y, gx = x0 + xx - 1;
            const bool valid = y < pl.TY && xx >= 1 && xx <= pl.XT && gy < g.H && gx < g.W;
            const i64 v = (((i64)b * g.D + z) * g.H + gy) * g.W + gx;
            for (int col = 16 * half; col < N; col += 32) {
                float acc[16];
                tmem_ld16(tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(m * N + col), acc);
                if (!valid) continue;
                if (!DGRAD) {
                    float bv[16];
                    if (bias) {
                        const float4* b4 = reinterpret_cast<const float4*>(bias + col);
#pragma unroll
                        for (int h = 0; h < 4; ++h) {
                            const float4 t = __ldg(b4 + h);
                            bv[4 * h] = t.x;
                            bv[4 * h + 1] = t.y;
                            bv[4 * h + 2] = t.z;
                            bv[4 * h + 3] = t.w;
                        }
                    }
#pragma unroll
                    for (int e = 0; e < 16; ++e) {
                        float a = acc[e];
                        if (bias) a += bv[e];
                        if (relu) a = fmaxf(a, 0.0f);
                        acc[e] = a;
                    }
                } else if (mask_src) {
                    const uint4* m4 = reinterpret_cast<const uint4*>(mask_src + v * N + col);
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        const uint4 mv = __ldg(m4 + h);
                        const __nv_bfloat16* mb = reinterpret_cast<const __nv_bfloat16*>(&mv);
#pragma unroll
                        for (int e = 0; e < 8; ++e)
                            if (!(__bfloat162float(mb[e]) > 0.0f)) acc[8 * h + e] = 0.0f;
                    }
                }
                uint4* o4 = reinterpret_cast<uint4*>(out + v * N + col);
                o4[0] = make_uint4(pack_bf16x2(acc[0], acc[1]), pack_bf16x2(acc[2], acc[3]),
                                   pack_bf16x2(acc[4], acc[5]), pack_bf16x2(acc[6], acc[7]));
                o4[1] = make_uint4(pack_bf16x2(acc[8], acc[9]), pack_bf16x2(acc[10], acc[11]),
                                   pack_bf16x2(acc[12], acc[13]), pack_bf16x2(acc[14], acc[15]));
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, (uint32_t)pl.tmem_cols);
}

// Block shape for a layer: the (XT, TY) that minimises the estimated time (27 MMAs of about 16 cycles
// per M tile and chunk, plus staging at about 64 bytes per cycle), within the shared-memory and TMEM
// limits. Returns false when nothing fits.
static inline bool win_plan(int D, int H, int W, int Cs, int N, int B, WinPlan& best) {
    const int nq = (Cs + 15) / 16;
    const int stages = nq > 1 ? 2 : 1;
    const int b_bytes = 54 * N * 16;
    double best_cost = -1.0;
    for (int k = 1; k <= 4; ++k) {
        const int XT = (W + k - 1) / k;
        const int RW = XT + 2;
        for (int TY : {8, 4, 2, 1}) {
            if (TY > 1 && TY / 2 >= H) continue;
            const int tiles = (TY * RW + 127) / 128;
            const int Lbeg = (TY + 3) * RW;
            const int P = 2 * (TY + 3) * RW + tiles * 128 + 2;
            const int a_bytes = 2 * P * 16;
            const int smem = stages * (a_bytes + b_bytes) + 64;
            if (smem > 220 * 1024 || tiles * N > 512 || P >= (1 << 14)) continue;
            const int xtiles = (W + XT - 1) / XT, ytiles = (H + TY - 1) / TY;
            const double blocks = (double)B * D * xtiles * ytiles;
            int cols = 32;
            while (cols < tiles * N) cols *= 2;
            // a second resident block overlaps one block's staging with the other's MMAs
            const bool two = smem <= 113 * 1024 && cols <= 256;
            const double cost = blocks * nq * (27.0 * 16.0 * tiles + 3.0 * (TY + 2) * RW * 2 * 16 / 64.0) *
                                (two || stages == 2 ? 1.0 : 1.6);
            if (best_cost < 0 || cost < best_cost) {
                best_cost = cost;
                best = WinPlan{XT, TY, RW, tiles, xtiles, ytiles, P, Lbeg, nq, a_bytes, b_bytes, stages, cols,
                               smem};
                // more than half of TMEM: keep one block per SM by its shared-memory request
                if (cols > 256 && best.smem < 116 * 1024) best.smem = 116 * 1024;
            }
        }
    }
    return best_cost >= 0.0;
}

}  // namespace conv
}  // namespace clb
