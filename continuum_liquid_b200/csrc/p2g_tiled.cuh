// P2G as a tiled, deterministic scatter (the tolerance-mode path; the reference-order gather of
// binning.cuh stays the parity path). Same results as particles.cl:135-227 up to the order and
// rounding with which each cell's weighted sums are added: every weight is computed exactly as the
// reference computes it, the fluid fraction (an integer count) is identical, and a face that no
// particle weighs is 0 in both.
//
// The weights are the reference's, rounded as it rounds them; each velocity term is added with one
// fused multiply-add (one rounding instead of two).
//
// Why: the reference visits each particle from the 27 cells around its bin (27 tent evaluations per
// particle per face type). Here each particle is visited once. A particle in bin b (b = floor(s -
// 0.5) per axis, s = p / dx) has nonzero weights only on the faces of cells b-1..b+1 along the
// face's own axis and b..b+1 along the other two: 12 u faces, 12 v faces, 12 w faces, and it is
// counted in one of the 8 cells b..b+1. All particles of one bin share these candidates, so a lane
// sums its bin's particles into 72 register accumulators (velocity and weight sums) and adds them to
// the tile's shared-memory sums once per bin; the counts go to shared memory as they are found.
//
// Layout: a block owns a tile of TI x TJ x TK cells (10 x 10 x 30) and sums into shared memory the
// contributions of the bins of the tile and its one-bin halo: (TI+2) x (TJ+2) rows of TK+2 = 32 bins
// along k, one warp per row, one lane per bin. Rows run in 9 phases by (row i mod 3, row j mod 3):
// rows of one phase are at least 3 apart in i or j, so their candidate cells are disjoint and no two
// warps add to the same cell at the same time. Inside a row the lanes add one candidate offset at a
// time (distinct cells of each array per step, __syncwarp between steps). Every cell therefore receives its terms
// in a fixed order: no floating-point atomics (the counts use integer shared-memory atomics, which
// commute), and the same result on every run.
#pragma once
#include "common.cuh"

namespace clb {

constexpr int P2GT_TI = 10, P2GT_TJ = 10, P2GT_TK = 30;
constexpr int P2GT_ROWS_I = P2GT_TI + 2, P2GT_ROWS_J = P2GT_TJ + 2;
constexpr int P2GT_CELLS = P2GT_TI * P2GT_TJ * P2GT_TK;
constexpr int P2GT_WARPS = 8;
constexpr int P2GT_THREADS = 32 * P2GT_WARPS;
// shared memory: velocity sums u, v, w; weight sums u, v, w; counts
constexpr int P2GT_SMEM = 7 * P2GT_CELLS * 4;
static_assert(P2GT_TK + 2 == 32, "a row of bins is one warp");
static_assert(P2GT_ROWS_I % 3 == 0 && P2GT_ROWS_J % 3 == 0, "phases split the rows evenly");

__device__ __forceinline__ float p2gt_tent(float s, float f) { return fmaxf(0.0f, 1.0f - fabsf(s - f)); }

// One block's tile (the body of k_p2g_tiled; also run per scene by the batched P2G). The particle
// indices in offsets are indices into pos and vel.
__device__ __forceinline__ void p2g_tile(int tile, const float* __restrict__ pos, const float* __restrict__ vel,
                                         const int* __restrict__ offsets, const int* __restrict__ counts,
                                         float* __restrict__ u, float* __restrict__ v, float* __restrict__ w,
                                         float* __restrict__ ff, float inv_dx, float inv_ppc, int nx, int ny, int nz,
                                         int tiles_j, int tiles_k) {
    extern __shared__ __align__(16) float p2gt_smem[];
    float* s_vel = p2gt_smem;                    // [3][CELLS]
    float* s_wgt = p2gt_smem + 3 * P2GT_CELLS;  // [3][CELLS]
    int* s_cnt = reinterpret_cast<int*>(p2gt_smem + 6 * P2GT_CELLS);
    const int tk = tile % tiles_k, tj = (tile / tiles_k) % tiles_j, ti = tile / (tiles_k * tiles_j);
    const int i0 = ti * P2GT_TI, j0 = tj * P2GT_TJ, k0 = tk * P2GT_TK;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    // rows holding particles: bins (i0-1+ri, j0-1+rj, k0-1 .. k0+30) inside the bin range [0, n-2]
    const int bz_lo = max(k0 - 1, 0), bz_hi = min(k0 + P2GT_TK, nz - 2);
    int any = 0;
    for (int r = threadIdx.x; r < P2GT_ROWS_I * P2GT_ROWS_J; r += P2GT_THREADS) {
        const int bx = i0 - 1 + r / P2GT_ROWS_J, by = j0 - 1 + r % P2GT_ROWS_J;
        if (bx < 0 || bx > nx - 2 || by < 0 || by > ny - 2 || bz_lo > bz_hi) continue;
        const i64 first = gidx(bx, by, bz_lo, ny, nz), last = gidx(bx, by, bz_hi, ny, nz);
        any |= (__ldg(offsets + last) + __ldg(counts + last) - __ldg(offsets + first)) > 0;
    }
    any = __syncthreads_or(any);
    if (any) {
        for (int c = threadIdx.x; c < 7 * P2GT_CELLS; c += P2GT_THREADS) p2gt_smem[c] = 0.0f;
        __syncthreads();
        for (int phase = 0; phase < 9; ++phase) {
            const int pi = phase / 3, pj = phase % 3;
            // the 16 rows of this phase: row (pi + 3 a, pj + 3 b), a, b in 0..3
            for (int r = warp; r < (P2GT_ROWS_I / 3) * (P2GT_ROWS_J / 3); r += P2GT_WARPS) {
                const int ri = pi + 3 * (r / (P2GT_ROWS_J / 3)), rj = pj + 3 * (r % (P2GT_ROWS_J / 3));
                const int bx = i0 - 1 + ri, by = j0 - 1 + rj, bz = k0 - 1 + lane;
                const bool row_ok = bx >= 0 && bx <= nx - 2 && by >= 0 && by <= ny - 2;
                if (!__any_sync(0xffffffffu, row_ok)) continue;  // warp-uniform
                const bool bin_ok = row_ok && bz >= 0 && bz <= nz - 2;
                int begin = 0, end = 0;
                if (bin_ok) {
                    const i64 bin = gidx(bx, by, bz, ny, nz);
                    begin = __ldg(offsets + bin);
                    end = begin + __ldg(counts + bin);
                }
                if (!__any_sync(0xffffffffu, end > begin)) continue;  // a row without particles adds nothing
                float vu[12], wu[12], vv[12], wv[12], vw[12], ww[12];
#pragma unroll
                for (int a = 0; a < 12; ++a) vu[a] = wu[a] = vv[a] = wv[a] = vw[a] = ww[a] = 0.0f;
                const float fbx = (float)bx, fby = (float)by, fbz = (float)bz;
                const int li = bx - i0, lj = by - j0, lk = bz - k0;
                for (int q = begin; q < end; ++q) {
                    const float* P = pos + 3 * (i64)q;
                    const float* V = vel + 3 * (i64)q;
                    const float sx = __ldg(P) * inv_dx, sy = __ldg(P + 1) * inv_dx, sz = __ldg(P + 2) * inv_dx;
                    const float v0 = __ldg(V), v1 = __ldg(V + 1), v2 = __ldg(V + 2);
                    // the reference's face positions: cell c's u face at c + 1 on x, its v and w faces
                    // at c + 0.5; here c = b - 1, b, b + 1 (full) and b, b + 1 (half)
                    const float fx[3] = {p2gt_tent(sx, fbx), p2gt_tent(sx, fbx + 1.0f), p2gt_tent(sx, fbx + 2.0f)};
                    const float fy[3] = {p2gt_tent(sy, fby), p2gt_tent(sy, fby + 1.0f), p2gt_tent(sy, fby + 2.0f)};
                    const float fz[3] = {p2gt_tent(sz, fbz), p2gt_tent(sz, fbz + 1.0f), p2gt_tent(sz, fbz + 2.0f)};
                    const float hx[2] = {p2gt_tent(sx, fbx + 0.5f), p2gt_tent(sx, fbx + 1.5f)};
                    const float hy[2] = {p2gt_tent(sy, fby + 0.5f), p2gt_tent(sy, fby + 1.5f)};
                    const float hz[2] = {p2gt_tent(sz, fbz + 0.5f), p2gt_tent(sz, fbz + 1.5f)};
                    // weights multiplied x * y * z left to right, as the reference does
#pragma unroll
                    for (int a = 0; a < 3; ++a)
#pragma unroll
                        for (int b = 0; b < 2; ++b)
#pragma unroll
                            for (int c = 0; c < 2; ++c) {
                                const int t = (a * 2 + b) * 2 + c;
                                const float gu = fx[a] * hy[b] * hz[c];  // u: (a, b, c) = (x, y, z)
                                const float gv = hx[b] * fy[a] * hz[c];  // v: (b, a, c)
                                const float gw = hx[b] * hy[c] * fz[a];  // w: (b, c, a)
                                // the velocity sums as one fused multiply-add per term (this kernel is
                                // the tolerance mode's: its sums already differ from the reference's order)
                                vu[t] = __fmaf_rn(gu, v0, vu[t]);
                                wu[t] += gu;
                                vv[t] = __fmaf_rn(gv, v1, vv[t]);
                                wv[t] += gv;
                                vw[t] = __fmaf_rn(gw, v2, vw[t]);
                                ww[t] += gw;
                            }
                    // the particle's cell for the fluid fraction (b or b + 1 on each axis): integer adds
                    // commute, so a shared-memory atomic keeps the count exact and deterministic
                    const int ci = clampi((int)sx, 1, nx - 2) - i0, cj = clampi((int)sy, 1, ny - 2) - j0,
                              ck = clampi((int)sz, 1, nz - 2) - k0;
                    if (ci >= 0 && ci < P2GT_TI && cj >= 0 && cj < P2GT_TJ && ck >= 0 && ck < P2GT_TK)
                        atomicAdd(s_cnt + (ci * P2GT_TJ + cj) * P2GT_TK + ck, 1);
                }
                __syncwarp();
                // add the bin's sums to the tile's cells, one candidate offset at a time: within a step the
                // lanes write distinct cells of each array (u, v and w sums are separate arrays), and a
                // __syncwarp orders the steps, which can reach the same cell from neighbouring lanes
                auto add = [&](float* sv, float* sw, int di, int dj, int dk, float val, float wgt) {
                    const int ci = li + di, cj = lj + dj, ck = lk + dk;
                    if (bin_ok && ci >= 0 && ci < P2GT_TI && cj >= 0 && cj < P2GT_TJ && ck >= 0 && ck < P2GT_TK) {
                        const int c = (ci * P2GT_TJ + cj) * P2GT_TK + ck;
                        sv[c] += val;
                        sw[c] += wgt;
                    }
                };
#pragma unroll
                for (int a = 0; a < 3; ++a)
#pragma unroll
                    for (int b = 0; b < 2; ++b)
#pragma unroll
                        for (int c = 0; c < 2; ++c) {
                            const int t = (a * 2 + b) * 2 + c;
                            add(s_vel, s_wgt, a - 1, b, c, vu[t], wu[t]);
                            add(s_vel + P2GT_CELLS, s_wgt + P2GT_CELLS, b, a - 1, c, vv[t], wv[t]);
                            add(s_vel + 2 * P2GT_CELLS, s_wgt + 2 * P2GT_CELLS, b, c, a - 1, vw[t], ww[t]);
                            __syncwarp();
                        }
            }
            __syncthreads();
        }
    }
    // the tile's cells: the reference's normalisation (particles.cl:216-226)
    for (int c = threadIdx.x; c < P2GT_CELLS; c += P2GT_THREADS) {
        const int ci = i0 + c / (P2GT_TJ * P2GT_TK), cj = j0 + (c / P2GT_TK) % P2GT_TJ, ck = k0 + c % P2GT_TK;
        if (ci >= nx || cj >= ny || ck >= nz) continue;
        const i64 index = gidx(ci, cj, ck, ny, nz);
        if (!any) {
            u[index] = v[index] = w[index] = ff[index] = 0.0f;
            continue;
        }
        const float su = s_wgt[c], sv = s_wgt[P2GT_CELLS + c], sw = s_wgt[2 * P2GT_CELLS + c];
        u[index] = su > 0.0f ? s_vel[c] / su : 0.0f;
        v[index] = sv > 0.0f ? s_vel[P2GT_CELLS + c] / sv : 0.0f;
        w[index] = sw > 0.0f ? s_vel[2 * P2GT_CELLS + c] / sw : 0.0f;
        ff[index] = (float)s_cnt[c] * inv_ppc;
    }
}

__global__ void __launch_bounds__(P2GT_THREADS, 2)
    k_p2g_tiled(const float* __restrict__ pos, const float* __restrict__ vel, const int* __restrict__ offsets,
                const int* __restrict__ counts, float* __restrict__ u, float* __restrict__ v, float* __restrict__ w,
                float* __restrict__ ff, float inv_dx, float inv_ppc, int nx, int ny, int nz, int tiles_j,
                int tiles_k) {
    p2g_tile(blockIdx.x, pos, vel, offsets, counts, u, v, w, ff, inv_dx, inv_ppc, nx, ny, nz, tiles_j, tiles_k);
}

__host__ __device__ __forceinline__ int p2g_tiled_tiles(int nx, int ny, int nz, int* tiles_j, int* tiles_k) {
    const int ti = (nx + P2GT_TI - 1) / P2GT_TI;
    *tiles_j = (ny + P2GT_TJ - 1) / P2GT_TJ;
    *tiles_k = (nz + P2GT_TK - 1) / P2GT_TK;
    return ti * *tiles_j * *tiles_k;
}

}  // namespace clb
