// One red-black Gauss-Seidel iteration (both colours, multigrid.cl:203-230 launched twice by
// multigrid.py:190-220) in a single launch.
//
// A block owns a SW_TI x SW_TJ x SW_TK tile. It loads p (and, on the finest level, the packed
// operator) for the tile plus a two-cell halo and b for the tile plus a one-cell halo into shared
// memory in one pass, updates the red cells of the tile plus one-cell halo (their neighbours are all
// start-of-iteration black values), then the black cells of the tile (their red neighbours are all
// final), and writes the tile. Red halo cells are recomputed by the neighbouring block from the same
// inputs, so every value equals the two-launch reference. The result goes to a second buffer, since
// neighbouring blocks must read start-of-iteration values; callers alternate buffers.
//
// Cells that are not fluid are loaded and written as 0, which is what rbgs_step leaves there; each
// update uses the reference's term order.
#pragma once
#include "multigrid.cuh"

namespace clb {

constexpr int SW_THREADS = 256;

// Tile shapes: large levels use 8 x 8 x 32 tiles; levels with few tiles use 4 x 4 x 32 tiles so that
// more blocks share the (latency-bound) work.
template <bool L0, int SW_TI, int SW_TJ, int SW_TK>
__global__ void __launch_bounds__(SW_THREADS) k_rbgs_iter(const float* __restrict__ pin, float* __restrict__ pout,
                                                           const float* __restrict__ b,
                                                           const uint8_t* __restrict__ op0,
                                                           const float4* __restrict__ opc,
                                                           const uint8_t* __restrict__ mask, float delta, int nx,
                                                           int ny, int nz) {
    pdl_begin();
    constexpr int SW_PI = SW_TI + 4, SW_PJ = SW_TJ + 4, SW_PK = SW_TK + 4;  // p region (halo 2)
    constexpr int SW_BI = SW_TI + 2, SW_BJ = SW_TJ + 2, SW_BK = SW_TK + 2;  // b region (halo 1)
    constexpr int SW_PCELLS = SW_PI * SW_PJ * SW_PK;
    constexpr int SW_BCELLS = SW_BI * SW_BJ * SW_BK;
    __shared__ float sp[SW_PCELLS];
    __shared__ float sb[SW_BCELLS];
    __shared__ uint8_t sop[L0 ? SW_PCELLS : 4];  // finest level: packed operator, 0 outside the grid
    const int gi = blockIdx.z * SW_TI - 2, gj = blockIdx.y * SW_TJ - 2, gk = blockIdx.x * SW_TK - 2;
    const int sxg = ny * nz;
    const float d2 = delta * delta;

    // Staging: every load of the thread is issued before any shared-memory store (fully unrolled),
    // so a block keeps ~50 loads per thread in flight instead of one.
    constexpr int NP = (SW_PCELLS + SW_THREADS - 1) / SW_THREADS;
    constexpr int NB = (SW_BCELLS + SW_THREADS - 1) / SW_THREADS;
    float pv[NP];
    uint32_t ov[NP];
#pragma unroll
    for (int m = 0; m < NP; ++m) {
        const int t = threadIdx.x + m * SW_THREADS;
        const int a = t / (SW_PJ * SW_PK), r = t - a * (SW_PJ * SW_PK), bj = r / SW_PK, ck = r - bj * SW_PK;
        const int i = gi + a, j = gj + bj, k = gk + ck;
        pv[m] = 0.0f;
        ov[m] = 0u;
        if (t < SW_PCELLS && i >= 0 && i < nx && j >= 0 && j < ny && k >= 0 && k < nz) {
            const int c = i * sxg + j * nz + k;
            ov[m] = L0 ? (uint32_t)__ldg(op0 + c) : (uint32_t)__ldg(mask + c);
            pv[m] = __ldg(pin + c);
        }
    }
    float bvv[NB];
#pragma unroll
    for (int m = 0; m < NB; ++m) {
        const int t = threadIdx.x + m * SW_THREADS;
        const int a = t / (SW_BJ * SW_BK), r = t - a * (SW_BJ * SW_BK), bj = r / SW_BK, ck = r - bj * SW_BK;
        const int i = gi + 1 + a, j = gj + 1 + bj, k = gk + 1 + ck;
        bvv[m] = 0.0f;
        if (t < SW_BCELLS && i >= 0 && i < nx && j >= 0 && j < ny && k >= 0 && k < nz)
            bvv[m] = __ldg(b + i * sxg + j * nz + k);
    }
#pragma unroll
    for (int m = 0; m < NP; ++m) {
        const int t = threadIdx.x + m * SW_THREADS;
        if (t < SW_PCELLS) {
            const bool fluid = L0 ? (ov[m] & 64u) != 0u : ov[m] != 0u;
            sp[t] = fluid ? pv[m] : 0.0f;
            if (L0) sop[t] = (uint8_t)ov[m];
        }
    }
#pragma unroll
    for (int m = 0; m < NB; ++m) {
        const int t = threadIdx.x + m * SW_THREADS;
        if (t < SW_BCELLS) sb[t] = bvv[m];
    }
    __syncthreads();

    // cells of colour `parity` in the box [lo, lo + w) of the p region (w even along k)
    auto relax = [&](int parity, int lo, int wi, int wj, int wk) {
        const int half = wk / 2;
        for (int t = threadIdx.x; t < wi * wj * half; t += SW_THREADS) {
            const int a = lo + t / (wj * half), r = t % (wj * half), bj = lo + r / half, m = r % half;
            const int i = gi + a, j = gj + bj;
            const int ck = lo + 2 * m + ((i + j + gk + lo + parity) & 1);
            const int k = gk + ck;
            if (i < 1 || i > nx - 2 || j < 1 || j > ny - 2 || k < 1 || k > nz - 2) continue;
            const int q = (a * SW_PJ + bj) * SW_PK + ck;
            float d, wxp, wxm, wyp, wym, wzp, wzm;
            if (L0) {
                const uint32_t o = sop[q];
                if (!(o & 64u)) continue;
                d = (float)(o & 7u);
                wxp = bitf(o, 3);
                wyp = bitf(o, 4);
                wzp = bitf(o, 5);
                wxm = bitf(sop[q - SW_PJ * SW_PK], 3);
                wym = bitf(sop[q - SW_PK], 4);
                wzm = bitf(sop[q - 1], 5);
            } else {
                const int c = i * sxg + j * nz + k;
                if (!__ldg(mask + c)) continue;
                const float4 o = __ldg(opc + c);
                d = o.x;
                wxp = o.y;
                wyp = o.z;
                wzp = o.w;
                wxm = __ldg(opc + c - sxg).y;
                wym = __ldg(opc + c - nz).z;
                wzm = __ldg(opc + c - 1).w;
            }
            if (!(d > 0.0f)) continue;
            const float ws = wxp * sp[q + SW_PJ * SW_PK] + wxm * sp[q - SW_PJ * SW_PK] + wyp * sp[q + SW_PK] +
                             wym * sp[q - SW_PK] + wzp * sp[q + 1] + wzm * sp[q - 1];
            const int qb = ((a - 1) * SW_BJ + (bj - 1)) * SW_BK + (ck - 1);
            sp[q] = (ws - d2 * sb[qb]) / d;
        }
    };
    relax(0, 1, SW_TI + 2, SW_TJ + 2, SW_TK + 2);  // red on the tile + one-cell halo
    __syncthreads();
    relax(1, 2, SW_TI, SW_TJ, SW_TK);  // black on the tile
    __syncthreads();

    for (int t = threadIdx.x; t < SW_TI * SW_TJ * SW_TK; t += SW_THREADS) {
        const int a = t / (SW_TJ * SW_TK), r = t - a * (SW_TJ * SW_TK), bj = r / SW_TK, ck = r - bj * SW_TK;
        const int i = gi + 2 + a, j = gj + 2 + bj, k = gk + 2 + ck;
        if (i < nx && j < ny && k < nz) pout[i * sxg + j * nz + k] = sp[((a + 2) * SW_PJ + (bj + 2)) * SW_PK + ck + 2];
    }
}

}  // namespace clb

namespace clb {

// One red-black colour (multigrid.cl:203-230) with a 3-D launch and no index division: thread
// (x, y, z) of the grid owns VEC consecutive cells along k of row (i = z, j = y). With VEC = 4 the
// row is read with 16-byte loads (needs nz % 4 == 0); every cell of the vector is written back
// (unchanged cells of the other colour keep their value, cells that are not fluid are set to 0, as
// rbgs_step does). Each update keeps the reference's term order.
// Block (bx, by, bz) of the launch described above (block shape (32, 4)).
template <bool L0, int VEC>
__device__ __forceinline__ void rbgs_colour_at(int bx, int by, int bz, float* p, const float* __restrict__ b,
                                               const uint8_t* __restrict__ op0, const float4* __restrict__ opc,
                                               const uint8_t* __restrict__ mask, float delta, int parity, int nx,
                                               int ny, int nz) {
    const int k0 = (bx * 32 + threadIdx.x) * VEC;
    const int j = by * 4 + threadIdx.y;
    const int i = bz;
    if (k0 >= nz || j >= ny) return;
    const int sx = ny * nz, sy = nz;
    const int c0 = i * sx + j * sy + k0;
    const bool row_inner = i >= 1 && i <= nx - 2 && j >= 1 && j <= ny - 2;
    const float d2 = delta * delta;
    float pc[VEC], out[VEC];
    uint32_t fl[VEC];
    if (VEC == 4) {
        const float4 v = *reinterpret_cast<const float4*>(p + c0);
        pc[0] = v.x;
        pc[1] = v.y;
        pc[2] = v.z;
        pc[3] = v.w;
    } else {
#pragma unroll
        for (int q = 0; q < VEC; ++q) pc[q] = (k0 + q < nz) ? p[c0 + q] : 0.0f;
    }
    uint32_t ob[VEC];
#pragma unroll
    for (int q = 0; q < VEC; ++q) {
        const bool in = k0 + q < nz;
        if (L0) {
            ob[q] = in ? (uint32_t)__ldg(op0 + c0 + q) : 0u;
            fl[q] = (ob[q] >> 6) & 1u;
        } else {
            ob[q] = 0u;
            fl[q] = in ? (uint32_t)(__ldg(mask + c0 + q) != 0) : 0u;
        }
        out[q] = fl[q] ? pc[q] : 0.0f;
    }
    if (row_inner) {
#pragma unroll
        for (int q = 0; q < VEC; ++q) {
            const int k = k0 + q;
            if (!fl[q] || k < 1 || k > nz - 2 || ((i + j + k) & 1) != parity) continue;
            const int c = c0 + q;
            float d, wxp, wxm, wyp, wym, wzp, wzm;
            if (L0) {
                const uint32_t o = ob[q];
                d = (float)(o & 7u);
                wxp = bitf(o, 3);
                wyp = bitf(o, 4);
                wzp = bitf(o, 5);
                wxm = bitf(__ldg(op0 + c - sx), 3);
                wym = bitf(__ldg(op0 + c - sy), 4);
                wzm = bitf(q > 0 ? ob[q - 1] : (uint32_t)__ldg(op0 + c - 1), 5);
            } else {
                const float4 o = __ldg(opc + c);
                d = o.x;
                wxp = o.y;
                wyp = o.z;
                wzp = o.w;
                wxm = __ldg(opc + c - sx).y;
                wym = __ldg(opc + c - sy).z;
                wzm = __ldg(opc + c - 1).w;
            }
            if (!(d > 0.0f)) continue;
            const float kp = (q + 1 < VEC) ? pc[q + 1] : p[c + 1];
            const float km = (q > 0) ? pc[q - 1] : p[c - 1];
            const float ws = wxp * p[c + sx] + wxm * p[c - sx] + wyp * p[c + sy] + wym * p[c - sy] + wzp * kp +
                             wzm * km;
            out[q] = (ws - d2 * __ldg(b + c)) / d;
        }
    }
    if (VEC == 4) {
        *reinterpret_cast<float4*>(p + c0) = make_float4(out[0], out[1], out[2], out[3]);
    } else {
#pragma unroll
        for (int q = 0; q < VEC; ++q)
            if (k0 + q < nz) p[c0 + q] = out[q];
    }
}

template <bool L0, int VEC>
__global__ void __launch_bounds__(128) k_rbgs_colour(float* p, const float* __restrict__ b,
                                                      const uint8_t* __restrict__ op0,
                                                      const float4* __restrict__ opc,
                                                      const uint8_t* __restrict__ mask, float delta, int parity,
                                                      int nx, int ny, int nz) {
    pdl_begin();
    rbgs_colour_at<L0, VEC>(blockIdx.x, blockIdx.y, blockIdx.z, p, b, op0, opc, mask, delta, parity, nx, ny, nz);
}

}  // namespace clb
