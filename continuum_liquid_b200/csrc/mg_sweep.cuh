// T red-black Gauss-Seidel iterations (both colours each, multigrid.cl:203-230 launched twice per
// iteration by multigrid.py:190-220) in a single launch.
//
// A block owns a TI x TJ x TK tile. It stages p (and, on the finest level, the packed operator) for
// the tile plus a 2T-cell halo and b for the tile plus a (2T-1)-cell halo in shared memory, then runs
// the 2T colour phases in shared memory: phase s (colours alternate, red first) updates the tile plus
// a (2T-1-s)-cell halo, whose neighbours are all final values of phase s-1 (or start-of-launch values
// for s = 0). Halo cells are recomputed by the neighbouring blocks from the same inputs, so every value
// equals the two-launches-per-iteration reference. The result goes to a second buffer, since
// neighbouring blocks must read start-of-launch values; callers alternate buffers. More iterations per
// launch mean fewer launches (the latency floor of the small levels) for more recomputed halo cells.
//
// Cells that are not fluid are loaded and written as 0, which is what rbgs_step leaves there; each
// update uses the reference's term order. H: an FP16 level (mg_half.cuh): p, b and the operator are
// read as __half, kappa = scale[2] replaces delta^2, and every update is rounded to FP16 as the
// per-cell FP16 sweep stores it, so all FP16 sweep kinds agree bit for bit.
#pragma once
#include <type_traits>

#include "multigrid.cuh"

namespace clb {

constexpr int SW_THREADS = 256;

// Operator entry of a staged cell: finest level one byte (packed), FP32 coarse levels a float4, FP16
// coarse levels four halves; the diagonal of a cell that is not fluid is staged as -1.
template <bool L0, bool H>
struct StagedOp {
    using type = typename std::conditional<L0, uint8_t, typename std::conditional<H, uint2, float4>::type>::type;
};

template <bool L0, bool H, int TI, int TJ, int TK, int T>
struct SweepTile {
    static constexpr int HALO = 2 * T;
    static constexpr int PI = TI + 2 * HALO, PJ = TJ + 2 * HALO, PK = TK + 2 * HALO;  // p region
    static constexpr int BI = PI - 2, BJ = PJ - 2, BK = PK - 2;                       // b region
    static constexpr int PCELLS = PI * PJ * PK, BCELLS = BI * BJ * BK;
    static constexpr size_t OP_BYTES = sizeof(typename StagedOp<L0, H>::type);
    // operator first (16-byte aligned entries), then p, then b
    static constexpr size_t OP_SMEM = ((size_t)PCELLS * OP_BYTES + 15) & ~(size_t)15;
    static constexpr size_t smem() { return OP_SMEM + (size_t)PCELLS * 4 + (size_t)BCELLS * 4; }
};

__device__ __forceinline__ float4 h4_to_f4(uint2 u) {
    const __half2 a = *reinterpret_cast<const __half2*>(&u.x), b = *reinterpret_cast<const __half2*>(&u.y);
    return make_float4(__low2float(a), __high2float(a), __low2float(b), __high2float(b));
}

// Tile shapes: large levels use 8 x 8 x 32 tiles; levels with few tiles use 4 x 4 x 32 tiles so that
// more blocks share the (latency-bound) work. The operator of the whole p region is staged with p, so
// the phases read shared memory only.
template <bool L0, bool H, int TI, int TJ, int TK, int T>
__global__ void __launch_bounds__(SW_THREADS) k_rbgs_iter(const float* __restrict__ pin_, float* __restrict__ pout_,
                                                           const float* __restrict__ b_,
                                                           const uint8_t* __restrict__ op0,
                                                           const float4* __restrict__ opc_,
                                                           const uint8_t* __restrict__ mask, float delta,
                                                           const float* __restrict__ scale, int nx, int ny, int nz) {
    pdl_begin();
    static_assert(!(L0 && H), "the finest level is FP32");
    using G = SweepTile<L0, H, TI, TJ, TK, T>;
    using OpT = typename StagedOp<L0, H>::type;
    constexpr int HALO = G::HALO, PJ = G::PJ, PK = G::PK, BJ = G::BJ, BK = G::BK;
    extern __shared__ __align__(16) unsigned char smem[];
    OpT* sop = reinterpret_cast<OpT*>(smem);
    float* sp = reinterpret_cast<float*>(smem + G::OP_SMEM);
    float* sb = sp + G::PCELLS;
    const __half* pin_h = reinterpret_cast<const __half*>(pin_);
    const __half* b_h = reinterpret_cast<const __half*>(b_);
    const uint2* opc_h = reinterpret_cast<const uint2*>(opc_);
    const int gi = blockIdx.z * TI - HALO, gj = blockIdx.y * TJ - HALO, gk = blockIdx.x * TK - HALO;
    const int sxg = ny * nz;
    const float d2 = H ? scale[2] : delta * delta;
    const uint2 minus_one_h = make_uint2(0xBC00u, 0u);  // half -1 in the diagonal's slot

    // Staging: U cells per thread and round, every load of a round issued before its shared-memory
    // stores. Cells outside the grid stage p = 0 and an all-zero operator (never updated).
    constexpr int U = L0 ? 16 : (H ? 12 : 8);
    for (int t0 = threadIdx.x; t0 < G::PCELLS; t0 += U * SW_THREADS) {
        float pv[U];
        uint32_t mv[U];
        OpT ov[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int t = t0 + u * SW_THREADS;
            const int a = t / (PJ * PK), r = t - a * (PJ * PK), bj = r / PK, ck = r - bj * PK;
            const int i = gi + a, j = gj + bj, k = gk + ck;
            pv[u] = 0.0f;
            mv[u] = 0u;
            ov[u] = OpT{};
            if (t < G::PCELLS && i >= 0 && i < nx && j >= 0 && j < ny && k >= 0 && k < nz) {
                const int c = i * sxg + j * nz + k;
                if (L0) {
                    mv[u] = (uint32_t)__ldg(op0 + c);
                } else {
                    mv[u] = (uint32_t)__ldg(mask + c);
                    if constexpr (!L0) {
                        if constexpr (H) ov[u] = __ldg(opc_h + c);
                        else ov[u] = __ldg(opc_ + c);
                    }
                }
                pv[u] = H ? __half2float(pin_h[c]) : __ldg(pin_ + c);
            }
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int t = t0 + u * SW_THREADS;
            if (t < G::PCELLS) {
                const bool fluid = L0 ? (mv[u] & 64u) != 0u : mv[u] != 0u;
                sp[t] = fluid ? pv[u] : 0.0f;
                if constexpr (L0) {
                    sop[t] = (uint8_t)mv[u];
                } else if constexpr (H) {
                    uint2 o = ov[u];
                    if (!fluid) o.x = (o.x & 0xFFFF0000u) | minus_one_h.x;
                    sop[t] = o;
                } else {
                    float4 o = ov[u];
                    if (!fluid) o.x = -1.0f;
                    sop[t] = o;
                }
            }
        }
    }
    constexpr int UB = 16;
    for (int t0 = threadIdx.x; t0 < G::BCELLS; t0 += UB * SW_THREADS) {
        float bv[UB];
#pragma unroll
        for (int u = 0; u < UB; ++u) {
            const int t = t0 + u * SW_THREADS;
            const int a = t / (BJ * BK), r = t - a * (BJ * BK), bj = r / BK, ck = r - bj * BK;
            const int i = gi + 1 + a, j = gj + 1 + bj, k = gk + 1 + ck;
            bv[u] = 0.0f;
            if (t < G::BCELLS && i >= 0 && i < nx && j >= 0 && j < ny && k >= 0 && k < nz) {
                const int c = i * sxg + j * nz + k;
                bv[u] = H ? __half2float(b_h[c]) : __ldg(b_ + c);
            }
        }
#pragma unroll
        for (int u = 0; u < UB; ++u) {
            const int t = t0 + u * SW_THREADS;
            if (t < G::BCELLS) sb[t] = bv[u];
        }
    }
    __syncthreads();

    auto op4 = [&](int q) -> float4 {
        if constexpr (H) return h4_to_f4(sop[q]);
        else if constexpr (!L0) return sop[q];
        else return make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    };
    // cells of colour `parity` in the box [lo, lo + w) of the p region (w even along k)
    auto relax = [&](int parity, int lo, int wi, int wj, int wk) {
        const int half = wk / 2;
        for (int t = threadIdx.x; t < wi * wj * half; t += SW_THREADS) {
            const int a = lo + t / (wj * half), r = t % (wj * half), bj = lo + r / half, m = r % half;
            const int i = gi + a, j = gj + bj;
            const int ck = lo + 2 * m + ((i + j + gk + lo + parity) & 1);
            const int k = gk + ck;
            if (i < 1 || i > nx - 2 || j < 1 || j > ny - 2 || k < 1 || k > nz - 2) continue;
            const int q = (a * PJ + bj) * PK + ck;
            float d, wxp, wxm, wyp, wym, wzp, wzm;
            if constexpr (L0) {
                const uint32_t o = sop[q];
                if (!(o & 64u)) continue;
                d = (float)(o & 7u);
                wxp = bitf(o, 3);
                wyp = bitf(o, 4);
                wzp = bitf(o, 5);
                wxm = bitf(sop[q - PJ * PK], 3);
                wym = bitf(sop[q - PK], 4);
                wzm = bitf(sop[q - 1], 5);
            } else {
                const float4 o = op4(q);  // diagonal -1 where not fluid
                d = o.x;
                wxp = o.y;
                wyp = o.z;
                wzp = o.w;
                wxm = op4(q - PJ * PK).y;
                wym = op4(q - PK).z;
                wzm = op4(q - 1).w;
            }
            if (!(d > 0.0f)) continue;
            const float ws = wxp * sp[q + PJ * PK] + wxm * sp[q - PJ * PK] + wyp * sp[q + PK] + wym * sp[q - PK] +
                             wzp * sp[q + 1] + wzm * sp[q - 1];
            const int qb = ((a - 1) * BJ + (bj - 1)) * BK + (ck - 1);
            const float x = (ws - d2 * sb[qb]) / d;
            sp[q] = H ? __half2float(__float2half_rn(x)) : x;
        }
    };
#pragma unroll
    for (int s = 0; s < 2 * T; ++s) {
        relax(s & 1, 1 + s, G::PI - 2 - 2 * s, PJ - 2 - 2 * s, PK - 2 - 2 * s);
        __syncthreads();
    }

    for (int t = threadIdx.x; t < TI * TJ * TK; t += SW_THREADS) {
        const int a = t / (TJ * TK), r = t - a * (TJ * TK), bj = r / TK, ck = r - bj * TK;
        const int i = gi + HALO + a, j = gj + HALO + bj, k = gk + HALO + ck;
        if (i < nx && j < ny && k < nz) {
            const float v = sp[((a + HALO) * PJ + (bj + HALO)) * PK + ck + HALO];
            const int c = i * sxg + j * nz + k;
            if (H) reinterpret_cast<__half*>(pout_)[c] = __float2half_rn(v);
            else pout_[c] = v;
        }
    }
}

}  // namespace clb

namespace clb {

// One red-black colour (multigrid.cl:203-230) with a 3-D launch and no index division: thread
// (x, y, z) of the grid owns VEC consecutive cells along k of row (i = z, j = y). With VEC = 4 the
// row is read with 16-byte loads (needs nz % 4 == 0); every cell of the vector is written back
// (unchanged cells of the other colour keep their value, cells that are not fluid are set to 0, as
// rbgs_step does). Each update keeps the reference's term order.
// Z: the colour runs as if p held 0 at every cell (p is written but not read): the updated cells get
// (0 - delta^2 b) / d, which is the update's value when every neighbour is 0 (each weighted term is
// +0), and every other cell of the vector is set to 0.
// Block (bx, by, bz) of the launch described above (block shape (32, 4)).
template <bool L0, int VEC, bool Z = false>
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
    if (Z) {
#pragma unroll
        for (int q = 0; q < VEC; ++q) pc[q] = 0.0f;
    } else if (VEC == 4) {
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
            float ws = 0.0f;
            if (!Z) {
                const float kp = (q + 1 < VEC) ? pc[q + 1] : p[c + 1];
                const float km = (q > 0) ? pc[q - 1] : p[c - 1];
                ws = wxp * p[c + sx] + wxm * p[c - sx] + wyp * p[c + sy] + wym * p[c - sy] + wzp * kp + wzm * km;
            }
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
