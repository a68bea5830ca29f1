// The finest level's part of a W-cycle in two launches over 3-D fluid tiles (no counterpart in the
// reference, whose W-cycle (multigrid.py:53-187) launches each red-black colour (multigrid.cl:203-230),
// the restriction (multigrid.cl:90-180) and the prolongation (multigrid.cl:182-201) over the whole
// grid).
//
// A level-0 visit is: pre-smoothing, residual and restriction into level 1, the two visits of level 1,
// prolongation of level 1's correction, post-smoothing. With the colour sweeps on fluid tiles that is
// 2 pre + 2 post colour launches plus a restriction and a prolongation launch per visit, each streaming
// the fluid part of the grid. Here:
//   * the last pre-smoothing iteration, the residual and the restriction are one launch: a block stages
//     x (zero for a correction that starts from zero), the packed operator and b of its tile plus a
//     3-cell halo in shared memory, runs the red phase on the tile plus a 2-cell halo and the black
//     phase on the tile plus a 1-cell halo (halo cells are recomputed from the same inputs by every
//     block that stages them, so they hold the values the two-launch sweep gives), writes the tile's x
//     and, from the smoothed values, the residual of each child and the restricted right-hand side of
//     the coarse cells whose eight children lie in the tile (tiles start at odd indices, so every coarse
//     cell's children share one tile);
//   * the prolongation and the first post-smoothing iteration are one launch: the staged x of a fluid
//     interior cell is x + e(parent), the value the prolongation writes.
// Every update, residual and sum keeps the reference's term order (the colour kernels' order), so x,
// level 1's right-hand side and everything downstream are bit for bit those of the launch-per-step
// path. Neighbouring blocks read start-of-launch values, so each launch writes the other of two
// buffers; the caller alternates them. Tiles without a fluid cell are not listed: their cells are 0 in
// both buffers (not fluid), the value a sweep writes there.
#pragma once
#include "multigrid.cuh"

namespace clb {

constexpr int L0T_I = 8, L0T_J = 8, L0T_K = 32;  // output tile of one block
constexpr int L0T_THREADS = 256;
static_assert(L0T_I % 2 == 0 && L0T_J % 2 == 0 && L0T_K % 2 == 0, "tiles hold whole coarse cells");
static_assert((L0T_I / 2) * (L0T_J / 2) * (L0T_K / 2) == L0T_THREADS, "one thread per coarse cell");

// Tile (a, b, c) covers cells [1 + 8a, 9 + 8a) x [1 + 8b, 9 + 8b) x [1 + 32c, 33 + 32c); numbered
// (a * tiles_j + b) * tiles_k + c.
__host__ __device__ __forceinline__ void l0_tile_counts(int nx, int ny, int nz, int& ti, int& tj, int& tk) {
    ti = (nx - 2 + L0T_I - 1) / L0T_I;
    tj = (ny - 2 + L0T_J - 1) / L0T_J;
    tk = (nz - 2 + L0T_K - 1) / L0T_K;
}
__host__ __device__ __forceinline__ i64 l0_tile_capacity(int nx, int ny, int nz) {
    if (nx < 3 || ny < 3 || nz < 3) return 0;
    int ti, tj, tk;
    l0_tile_counts(nx, ny, nz, ti, tj, tk);
    return (i64)ti * tj * tk;
}

// One block per tile: lists it when one of its cells is fluid (bit 6 of the packed operator).
__global__ void __launch_bounds__(L0T_THREADS) k_l0_fused_tiles(const uint8_t* __restrict__ op0, int nx, int ny,
                                                                 int nz, int* __restrict__ list,
                                                                 int* __restrict__ count) {
    pdl_begin();
    int ti, tj, tk;
    l0_tile_counts(nx, ny, nz, ti, tj, tk);
    const int tile = blockIdx.x;
    const int c = tile % tk, rest = tile / tk, b = rest % tj, a = rest / tj;
    const int i0 = 1 + a * L0T_I, j0 = 1 + b * L0T_J, k0 = 1 + c * L0T_K;
    int fluid = 0;
    for (int t = threadIdx.x; t < L0T_I * L0T_J * L0T_K; t += L0T_THREADS) {
        const int i = i0 + t / (L0T_J * L0T_K), j = j0 + (t / L0T_K) % L0T_J, k = k0 + t % L0T_K;
        if (i < nx && j < ny && k < nz) fluid |= (__ldg(op0 + gidx(i, j, k, ny, nz)) & 64u) != 0u;
    }
    if (__syncthreads_or(fluid) && threadIdx.x == 0) list[atomicAdd(count, 1)] = tile;
}

template <int HALO>
struct L0Region {
    static constexpr int PI = L0T_I + 2 * HALO, PJ = L0T_J + 2 * HALO, PK = L0T_K + 2 * HALO;  // x, operator
    static constexpr int BI = PI - 2, BJ = PJ - 2, BK = PK - 2;                                   // b
    static constexpr int PCELLS = PI * PJ * PK, BCELLS = BI * BJ * BK;
    static constexpr size_t OP_SMEM = ((size_t)PCELLS + 15) & ~(size_t)15;
    static constexpr size_t smem() { return OP_SMEM + (size_t)PCELLS * 4 + (size_t)BCELLS * 4; }
};

enum { L0F_ZERO = 1, L0F_RESTRICT = 2, L0F_PROLONG = 4 };

// One red-black iteration of level 0 on the listed tiles, pin -> pout (distinct buffers).
//   L0F_ZERO:     x counts as 0 on entry (pin is not read);
//   L0F_RESTRICT: also the residual of the smoothed x and its restriction into level 1 (cp = 0,
//                 cb = the children's residual sum), as restrict_at writes them;
//   L0F_PROLONG:  x + w e(parent) on entry at fluid interior cells, e = level 1's p (prolong_at).
// Blocks walk the list (tile t, t + gridDim.x, ...).
template <int MODE>
__global__ void __launch_bounds__(L0T_THREADS) k_l0_iter_tiles(const int* __restrict__ list,
                                                                const int* __restrict__ count,
                                                                const float* __restrict__ pin, float* __restrict__ pout,
                                                                const float* __restrict__ b,
                                                                const uint8_t* __restrict__ op0, float delta, int nx,
                                                                int ny, int nz, float* __restrict__ cp,
                                                                float* __restrict__ cb, const float* __restrict__ ce,
                                                                int cnx, int cny, int cnz, float w) {
    pdl_begin();
    constexpr bool ZERO = (MODE & L0F_ZERO) != 0, RESTR = (MODE & L0F_RESTRICT) != 0, PROL = (MODE & L0F_PROLONG) != 0;
    static_assert(!(ZERO && PROL), "a prolongation adds to an x that is read");
    constexpr int HALO = RESTR ? 3 : 2;
    using G = L0Region<HALO>;
    constexpr int PI = G::PI, PJ = G::PJ, PK = G::PK, BJ = G::BJ, BK = G::BK;
    extern __shared__ __align__(16) unsigned char smem[];
    uint8_t* sop = smem;
    float* sp = reinterpret_cast<float*>(smem + G::OP_SMEM);
    float* sb = sp + G::PCELLS;
    int ti, tj, tk;
    l0_tile_counts(nx, ny, nz, ti, tj, tk);
    const int sxg = ny * nz;
    const float d2 = delta * delta;
    const int n = *count;
    for (int t = blockIdx.x; t < n; t += gridDim.x) {
        const int tile = __ldg(list + t);
        const int tc = tile % tk, rest = tile / tk, tb = rest % tj, ta = rest / tj;
        const int i0 = 1 + ta * L0T_I, j0 = 1 + tb * L0T_J, k0 = 1 + tc * L0T_K;
        const int gi = i0 - HALO, gj = j0 - HALO, gk = k0 - HALO;
        __syncthreads();  // the previous tile's reads of shared memory are done

        // x and the operator over the region, U cells per thread and round with every load of a round
        // issued before its stores; cells outside the grid stage x = 0 and operator 0 (never updated)
        constexpr int U = 12;
        for (int t0 = threadIdx.x; t0 < G::PCELLS; t0 += U * L0T_THREADS) {
            float pv[U];
            uint32_t ov[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int q = t0 + u * L0T_THREADS;
                const int a = q / (PJ * PK), r = q - a * (PJ * PK), bj = r / PK, ck = r - bj * PK;
                const int i = gi + a, j = gj + bj, k = gk + ck;
                pv[u] = 0.0f;
                ov[u] = 0u;
                if (q < G::PCELLS && i >= 0 && i < nx && j >= 0 && j < ny && k >= 0 && k < nz) {
                    const int c = i * sxg + j * nz + k;
                    ov[u] = (uint32_t)__ldg(op0 + c);
                    if (!ZERO) pv[u] = __ldg(pin + c);
                    if (PROL && (ov[u] & 64u) && i >= 1 && i <= nx - 2 && j >= 1 && j <= ny - 2 && k >= 1 &&
                        k <= nz - 2) {
                        const int I = min((i - 1) / 2 + 1, cnx - 2), J = min((j - 1) / 2 + 1, cny - 2),
                                  K = min((k - 1) / 2 + 1, cnz - 2);
                        pv[u] += w * __ldg(ce + gidx(I, J, K, cny, cnz));
                    }
                }
            }
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int q = t0 + u * L0T_THREADS;
                if (q < G::PCELLS) {
                    sop[q] = (uint8_t)ov[u];
                    sp[q] = (ov[u] & 64u) ? pv[u] : 0.0f;
                }
            }
        }
        constexpr int UB = 12;
        for (int t0 = threadIdx.x; t0 < G::BCELLS; t0 += UB * L0T_THREADS) {
            float bv[UB];
#pragma unroll
            for (int u = 0; u < UB; ++u) {
                const int q = t0 + u * L0T_THREADS;
                const int a = q / (BJ * BK), r = q - a * (BJ * BK), bj = r / BK, ck = r - bj * BK;
                const int i = gi + 1 + a, j = gj + 1 + bj, k = gk + 1 + ck;
                bv[u] = 0.0f;
                if (q < G::BCELLS && i >= 0 && i < nx && j >= 0 && j < ny && k >= 0 && k < nz)
                    bv[u] = __ldg(b + i * sxg + j * nz + k);
            }
#pragma unroll
            for (int u = 0; u < UB; ++u) {
                const int q = t0 + u * L0T_THREADS;
                if (q < G::BCELLS) sb[q] = bv[u];
            }
        }
        __syncthreads();

        // cells of colour `parity` ((i + j + k) & 1) in the box [lo, lo + w) of the region (w even
        // along k); the update of rbgs_colour_at: (ws - delta^2 b) / d, ws in (x+, x-, y+, y-, z+, z-)
        auto relax = [&](int parity, int lo, int wi, int wj, int wk) {
            const int half = wk / 2;
            for (int q0 = threadIdx.x; q0 < wi * wj * half; q0 += L0T_THREADS) {
                const int a = lo + q0 / (wj * half), r = q0 % (wj * half), bj = lo + r / half, m = r % half;
                const int i = gi + a, j = gj + bj;
                const int ck = lo + 2 * m + ((i + j + gk + lo + parity) & 1);
                const int k = gk + ck;
                if (i < 1 || i > nx - 2 || j < 1 || j > ny - 2 || k < 1 || k > nz - 2) continue;
                const int q = (a * PJ + bj) * PK + ck;
                const uint32_t o = sop[q];
                if (!(o & 64u)) continue;
                const float d = (float)(o & 7u);
                const float ws = bitf(o, 3) * sp[q + PJ * PK] + bitf(sop[q - PJ * PK], 3) * sp[q - PJ * PK] +
                                 bitf(o, 4) * sp[q + PK] + bitf(sop[q - PK], 4) * sp[q - PK] + bitf(o, 5) * sp[q + 1] +
                                 bitf(sop[q - 1], 5) * sp[q - 1];
                if (!(d > 0.0f)) continue;
                const int qb = ((a - 1) * BJ + (bj - 1)) * BK + (ck - 1);
                sp[q] = (ws - d2 * sb[qb]) / d;
            }
        };
        relax(0, 1, PI - 2, PJ - 2, PK - 2);  // red on the tile and a HALO - 1 halo
        __syncthreads();
        relax(1, 2, PI - 4, PJ - 4, PK - 4);  // black on the tile and a HALO - 2 halo
        __syncthreads();

        for (int q0 = threadIdx.x; q0 < L0T_I * L0T_J * L0T_K; q0 += L0T_THREADS) {
            const int a = q0 / (L0T_J * L0T_K), bj = (q0 / L0T_K) % L0T_J, ck = q0 % L0T_K;
            const int i = i0 + a, j = j0 + bj, k = k0 + ck;
            if (i < nx && j < ny && k < nz)
                pout[i * sxg + j * nz + k] = sp[((a + HALO) * PJ + (bj + HALO)) * PK + ck + HALO];
        }

        if (RESTR) {
            // coarse cell (I, J, K) of this thread; its children (2I - 1 + di, ...) are tile cells
            // (2 ci + di, 2 cj + dj, 2 ck + dk)
            const int ci = threadIdx.x / ((L0T_J / 2) * (L0T_K / 2)), cj = (threadIdx.x / (L0T_K / 2)) % (L0T_J / 2),
                      ck = threadIdx.x % (L0T_K / 2);
            const int I = (i0 + 1) / 2 + ci, J = (j0 + 1) / 2 + cj, K = (k0 + 1) / 2 + ck;
            if (I < cnx && J < cny && K < cnz) {
                float rhs = 0.0f;
                if (interior(I, J, K, cnx, cny, cnz)) {
                    const float inv_delta2 = 1.0f / (delta * delta);
#pragma unroll
                    for (int ch = 0; ch < 8; ++ch) {
                        const int di = ch >> 2, dj = (ch >> 1) & 1, dk = ch & 1;
                        const int i = 2 * I - 1 + di, j = 2 * J - 1 + dj, k = 2 * K - 1 + dk;
                        if (!interior(i, j, k, nx, ny, nz)) continue;
                        const int q = ((HALO + 2 * ci + di) * PJ + (HALO + 2 * cj + dj)) * PK + HALO + 2 * ck + dk;
                        const uint32_t o = sop[q];
                        if (!(o & 64u)) continue;
                        const float ws = bitf(o, 3) * sp[q + PJ * PK] + bitf(sop[q - PJ * PK], 3) * sp[q - PJ * PK] +
                                         bitf(o, 4) * sp[q + PK] + bitf(sop[q - PK], 4) * sp[q - PK] +
                                         bitf(o, 5) * sp[q + 1] + bitf(sop[q - 1], 5) * sp[q - 1];
                        const float ap = (ws - (float)(o & 7u) * sp[q]) * inv_delta2;
                        const int qb = ((HALO - 1 + 2 * ci + di) * BJ + (HALO - 1 + 2 * cj + dj)) * BK + HALO - 1 +
                                       2 * ck + dk;
                        rhs += sb[qb] - ap;
                    }
                }
                const i64 cidx = gidx(I, J, K, cny, cnz);
                cp[cidx] = 0.0f;
                cb[cidx] = rhs;
            }
        }
    }
}

}  // namespace clb
