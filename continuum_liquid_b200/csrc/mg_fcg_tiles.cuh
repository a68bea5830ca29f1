// Flexible-CG dots and the refinement / FCG step on the level-0 fluid tiles (no counterpart in the
// reference, whose pressure solve runs a fixed number of W-cycles, pressure_solve.py:61-84).
//
// The row kernels (k_fcg_dots, k_residual_rows in multigrid.cuh) give each warp whole rows: a lane's
// 32-cell steps along a row wait on their loads one after another, so the kernels are latency-bound.
// Here a block walks the listed level-0 tiles (one plane i, four rows j, TK cells k: the colour sweeps'
// tiles, mg_tiles.cuh). For each tile it first loads everything the tile's cells read -- the tile, the
// rows j - 1 and j + 4 of its plane and the tile's rows of planes i - 1 and i + 1, one cell further
// along k -- into shared memory, every load of a thread issued before any use, forming each cell's
// value once (the step's pressure p_in + alpha d with d = e + beta d_in); then it computes the tile's
// cells from shared memory. Per cell the arithmetic and its order are the row kernels', so the stored
// pressure, direction and residual are theirs bit for bit; only the order in which cells enter the
// FP64 sums differs. The tile list is built in ascending order (k_mg_tile_flags0 + k_compact_tiles) and
// blocks walk it
// in list order with a fixed grid, so the sums are the same on every run.
//
// Cells that are not interior fluid cells are neither read as centres nor written, as in the row
// kernels' skipping mode (their values stay 0 when the caller keeps that invariant).
#pragma once
#include "multigrid.cuh"
#include "mg_tiles.cuh"

namespace clb {

constexpr int FT_THREADS = 256;

template <int TK>
struct FcgTile {
    static constexpr int CK = TK + 2;           // centre-plane rows: k0 - 1 .. k0 + TK
    static constexpr int CENTRE = 6 * CK;       // rows j0 - 1 .. j0 + 4 of plane i
    static constexpr int SIDE = 4 * TK;         // rows j0 .. j0 + 3 of plane i -/+ 1
    static constexpr int CELLS = CENTRE + 2 * SIDE;
    static constexpr int OPS = CENTRE + SIDE;   // operator bytes: centre plane and plane i - 1
    static constexpr int OUT = 4 * TK;          // the tile's cells
};

// Staged index of cell (plane offset di in {-1, 0, 1}, row r = j - j0 + 1 in 0..5 (centre) or
// 1..4 (sides), kk = k - k0 + 1 in 0..TK + 1 (centre) or 1..TK (sides)).
template <int TK>
__device__ __forceinline__ int ft_index(int di, int r, int kk) {
    using G = FcgTile<TK>;
    if (di == 0) return r * G::CK + kk;
    return G::CENTRE + (di < 0 ? 0 : G::SIDE) + (r - 1) * TK + (kk - 1);
}

// Walks staged slots: centre rows first, then plane i - 1, then plane i + 1.
template <int TK>
__device__ __forceinline__ void ft_slot(int s, int& di, int& r, int& kk) {
    using G = FcgTile<TK>;
    if (s < G::CENTRE) {
        di = 0;
        r = s / G::CK;
        kk = s - r * G::CK;
    } else {
        const int t = s - G::CENTRE;
        di = t < G::SIDE ? -1 : 1;
        const int u = t < G::SIDE ? t : t - G::SIDE;
        r = 1 + u / TK;
        kk = 1 + u % TK;
    }
}

template <int TK>
__device__ __forceinline__ void ft_tile_origin(int tile, int ny, int nz, int& i, int& j0, int& k0) {
    const int jg = (ny + 3) / 4, kg = (nz + TK - 1) / TK;
    const int kb = tile % kg, rest = tile / kg;
    k0 = kb * TK;
    j0 = (rest % jg) * 4;
    i = rest / jg;
}

// Refinement (MODE RES_IR) or FCG (RES_FCG) step of k_residual_rows<double, MODE, true> on the listed
// tiles; per block partial sums {r^2, b^2} over interior fluid cells.
template <int MODE, int TK>
__global__ void __launch_bounds__(FT_THREADS) k_step_tiles(const int* __restrict__ list, const int* __restrict__ count,
                                                            const double* __restrict__ p_in, const float* __restrict__ e,
                                                            double* __restrict__ p_out, const float* __restrict__ b,
                                                            const uint8_t* __restrict__ op0, double inv_delta2, int nx,
                                                            int ny, int nz, float* __restrict__ r_out,
                                                            double2* __restrict__ partials,
                                                            const float* __restrict__ d_in, float* __restrict__ d_out,
                                                            const double* __restrict__ state) {
    pdl_begin();
    static_assert(MODE == RES_IR || MODE == RES_FCG, "a step mode");
    using G = FcgTile<TK>;
    __shared__ double s_p[G::CELLS];
    __shared__ float s_d[G::OUT];
    __shared__ uint8_t s_op[G::OPS];
    __shared__ double2 s_red[FT_THREADS / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double alpha = 0.0, beta = 0.0;
    if (MODE == RES_FCG) {
        alpha = state[0];
        beta = state[1];
    }
    const i64 sx = (i64)ny * nz, sy = nz;
    double rr = 0.0, bb = 0.0;
    const int n = *count;
    constexpr int PER = (G::CELLS + FT_THREADS - 1) / FT_THREADS;
    for (int t = blockIdx.x; t < n; t += gridDim.x) {
        int i, j0, k0;
        ft_tile_origin<TK>(__ldg(list + t), ny, nz, i, j0, k0);
        __syncthreads();  // the previous tile's shared-memory reads are done
        // loads of all slots first, then the values
        double pv[PER];
        float ev[PER], dv[PER];
        uint32_t ov[PER];
#pragma unroll
        for (int u = 0; u < PER; ++u) {
            const int s = threadIdx.x + u * FT_THREADS;
            pv[u] = 0.0;
            ev[u] = 0.0f;
            dv[u] = 0.0f;
            ov[u] = 0u;
            if (s < G::CELLS) {
                int di, r, kk;
                ft_slot<TK>(s, di, r, kk);
                const int ii = i + di, j = j0 + r - 1, k = k0 + kk - 1;
                if (ii >= 0 && ii < nx && j >= 0 && j < ny && k >= 0 && k < nz) {
                    const i64 c = (i64)ii * sx + (i64)j * sy + k;
                    pv[u] = __ldg(p_in + c);
                    ev[u] = __ldg(e + c);
                    if (MODE == RES_FCG) dv[u] = __ldg(d_in + c);
                    if (di <= 0) ov[u] = __ldg(op0 + c);
                }
            }
        }
#pragma unroll
        for (int u = 0; u < PER; ++u) {
            const int s = threadIdx.x + u * FT_THREADS;
            if (s < G::CELLS) {
                // the row kernel's pv(q): p_in + e (refinement) or p_in + alpha d, d = e + beta d_in
                double value;
                if (MODE == RES_IR) {
                    value = pv[u] + (double)ev[u];
                } else {
                    const float d = (float)((double)ev[u] + beta * (double)dv[u]);
                    value = pv[u] + alpha * (double)d;
                    int di, r, kk;
                    ft_slot<TK>(s, di, r, kk);
                    if (di == 0 && r >= 1 && r <= 4 && kk >= 1 && kk <= TK) s_d[(r - 1) * TK + (kk - 1)] = d;
                }
                s_p[s] = value;
                if (s < G::OPS) s_op[s] = (uint8_t)ov[u];
            }
        }
        __syncthreads();
        for (int q = threadIdx.x; q < G::OUT; q += FT_THREADS) {
            const int r = 1 + q / TK, kk = 1 + q % TK;
            const int j = j0 + r - 1, k = k0 + kk - 1;
            if (i < 1 || i > nx - 2 || j < 1 || j > ny - 2 || k < 1 || k > nz - 2) continue;
            const int sc = ft_index<TK>(0, r, kk);
            const uint32_t o = s_op[sc];
            if (!(o & 64u)) continue;
            const i64 c = (i64)i * sx + (i64)j * sy + k;
            const double pc = s_p[sc];
            p_out[c] = pc;
            if (MODE == RES_FCG) d_out[c] = s_d[q];
            const uint32_t ox = s_op[ft_index<TK>(-1, r, kk)], oy = s_op[ft_index<TK>(0, r - 1, kk)],
                           oz = s_op[sc - 1];
            const double ws = (double)bitf(o, 3) * s_p[ft_index<TK>(1, r, kk)] +
                              (double)bitf(ox, 3) * s_p[ft_index<TK>(-1, r, kk)] +
                              (double)bitf(o, 4) * s_p[ft_index<TK>(0, r + 1, kk)] +
                              (double)bitf(oy, 4) * s_p[ft_index<TK>(0, r - 1, kk)] +
                              (double)bitf(o, 5) * s_p[sc + 1] + (double)bitf(oz, 5) * s_p[sc - 1];
            const double bv = (double)__ldg(b + c);
            const double res = bv - (ws - (double)(o & 7u) * pc) * inv_delta2;
            rr += res * res;
            bb += bv * bv;
            r_out[c] = (float)res;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        rr += __shfl_xor_sync(0xffffffffu, rr, o);
        bb += __shfl_xor_sync(0xffffffffu, bb, o);
    }
    if (lane == 0) s_red[warp] = make_double2(rr, bb);
    __syncthreads();
    if (threadIdx.x == 0) {
        double2 acc = s_red[0];
        for (int q = 1; q < FT_THREADS / 32; ++q) {
            acc.x += s_red[q].x;
            acc.y += s_red[q].y;
        }
        partials[blockIdx.x] = acc;
    }
}

// k_fcg_dots on the listed tiles: per block partial sums of (A z).d, (A z).z, z.r, d.r.
template <int TK>
__global__ void __launch_bounds__(FT_THREADS) k_fcg_dots_tiles(const int* __restrict__ list,
                                                                const int* __restrict__ count,
                                                                const float* __restrict__ z,
                                                                const float* __restrict__ d,
                                                                const float* __restrict__ r,
                                                                const uint8_t* __restrict__ op0, double inv_delta2,
                                                                int nx, int ny, int nz, Sum4* __restrict__ partials) {
    pdl_begin();
    using G = FcgTile<TK>;
    __shared__ float s_z[G::CELLS];
    __shared__ uint8_t s_op[G::OPS];
    __shared__ Sum4 s_red[FT_THREADS / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const i64 sx = (i64)ny * nz, sy = nz;
    Sum4 acc = {0.0, 0.0, 0.0, 0.0};
    const int n = *count;
    constexpr int PER = (G::CELLS + FT_THREADS - 1) / FT_THREADS;
    for (int t = blockIdx.x; t < n; t += gridDim.x) {
        int i, j0, k0;
        ft_tile_origin<TK>(__ldg(list + t), ny, nz, i, j0, k0);
        __syncthreads();
        float zv[PER];
        uint32_t ov[PER];
#pragma unroll
        for (int u = 0; u < PER; ++u) {
            const int s = threadIdx.x + u * FT_THREADS;
            zv[u] = 0.0f;
            ov[u] = 0u;
            if (s < G::CELLS) {
                int di, rr, kk;
                ft_slot<TK>(s, di, rr, kk);
                const int ii = i + di, j = j0 + rr - 1, k = k0 + kk - 1;
                if (ii >= 0 && ii < nx && j >= 0 && j < ny && k >= 0 && k < nz) {
                    const i64 c = (i64)ii * sx + (i64)j * sy + k;
                    zv[u] = __ldg(z + c);
                    if (di <= 0) ov[u] = __ldg(op0 + c);
                }
            }
        }
#pragma unroll
        for (int u = 0; u < PER; ++u) {
            const int s = threadIdx.x + u * FT_THREADS;
            if (s < G::CELLS) {
                s_z[s] = zv[u];
                if (s < G::OPS) s_op[s] = (uint8_t)ov[u];
            }
        }
        __syncthreads();
        for (int q = threadIdx.x; q < G::OUT; q += FT_THREADS) {
            const int rr = 1 + q / TK, kk = 1 + q % TK;
            const int j = j0 + rr - 1, k = k0 + kk - 1;
            if (i < 1 || i > nx - 2 || j < 1 || j > ny - 2 || k < 1 || k > nz - 2) continue;
            const int sc = ft_index<TK>(0, rr, kk);
            const uint32_t o = s_op[sc];
            if (!(o & 64u)) continue;
            const i64 c = (i64)i * sx + (i64)j * sy + k;
            const uint32_t ox = s_op[ft_index<TK>(-1, rr, kk)], oy = s_op[ft_index<TK>(0, rr - 1, kk)],
                           oz = s_op[sc - 1];
            const double zc = (double)s_z[sc];
            const double ws = (double)bitf(o, 3) * (double)s_z[ft_index<TK>(1, rr, kk)] +
                              (double)bitf(ox, 3) * (double)s_z[ft_index<TK>(-1, rr, kk)] +
                              (double)bitf(o, 4) * (double)s_z[ft_index<TK>(0, rr + 1, kk)] +
                              (double)bitf(oy, 4) * (double)s_z[ft_index<TK>(0, rr - 1, kk)] +
                              (double)bitf(o, 5) * (double)s_z[sc + 1] + (double)bitf(oz, 5) * (double)s_z[sc - 1];
            const double az = (ws - (double)(o & 7u) * zc) * inv_delta2;
            const double dc = (double)__ldg(d + c), rc = (double)__ldg(r + c);
            acc.x += az * dc;
            acc.y += az * zc;
            acc.z += zc * rc;
            acc.w += dc * rc;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        acc.x += __shfl_xor_sync(0xffffffffu, acc.x, o);
        acc.y += __shfl_xor_sync(0xffffffffu, acc.y, o);
        acc.z += __shfl_xor_sync(0xffffffffu, acc.z, o);
        acc.w += __shfl_xor_sync(0xffffffffu, acc.w, o);
    }
    if (lane == 0) s_red[warp] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        Sum4 a = s_red[0];
        for (int q = 1; q < FT_THREADS / 32; ++q) {
            a.x += s_red[q].x;
            a.y += s_red[q].y;
            a.z += s_red[q].z;
            a.w += s_red[q].w;
        }
        partials[blockIdx.x] = a;
    }
}

}  // namespace clb
