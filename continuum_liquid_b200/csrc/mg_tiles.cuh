// Fluid tiles of the multigrid levels (no counterpart in the reference, whose kernels cover every
// cell of every level).
//
// Most of a free-surface domain is air: at 256^3 the benchmark's liquid block fills 17.5 % of the
// grid, and the coarse levels inherit that. A red-black sweep leaves a cell that is not fluid at 0
// (rbgs_step zeroes it), restriction writes 0 to a coarse cell without fluid children, and
// prolongation adds only to fluid cells. So once every cell without fluid holds 0 -- coarse p and b
// are zeroed when the operators are built, the restriction zeroes coarse p, and the tolerance mode
// hands the W-cycle a zero correction -- those kernels can visit only the tiles that hold a fluid
// cell and produce the reference's values bit for bit.
//
// A tile is one plane i, four rows j and TK cells along k (TK = 128 on the finest level when
// nz % 4 == 0, matching the 16-byte-vector colour sweep; 32 otherwise), i.e. exactly one block of the
// (32, 4)-thread colour sweep. The lists are rebuilt once per solve; their order is arbitrary (tiles
// are independent within a colour phase).
#pragma once
#include "multigrid.cuh"
#include "mg_sweep.cuh"

namespace clb {

__host__ __device__ __forceinline__ int tile_k(int nz, bool finest) { return (finest && nz % 4 == 0) ? 128 : 32; }
__host__ __device__ __forceinline__ i64 tile_capacity(int nx, int ny, int nz, bool finest) {
    const int tk = tile_k(nz, finest);
    return (i64)nx * ((ny + 3) / 4) * ((nz + tk - 1) / tk);
}

// One warp per tile: lists the tile when any of its cells is fluid (finest: bit 6 of the packed
// operator; coarse: the mask byte).
template <bool L0>
__global__ void __launch_bounds__(256) k_mg_tiles(const uint8_t* __restrict__ flags, int nx, int ny, int nz,
                                                  int* __restrict__ list, int* __restrict__ count) {
    pdl_begin();
    const int tk = tile_k(nz, L0), jg = (ny + 3) / 4, kg = (nz + tk - 1) / tk;
    const i64 tiles = (i64)nx * jg * kg;
    const i64 t = ((i64)blockIdx.x * 256 + threadIdx.x) / 32;
    const int lane = threadIdx.x & 31;
    bool fluid = false;
    if (t < tiles) {
        const int kb = (int)(t % kg), jb = (int)((t / kg) % jg), i = (int)(t / ((i64)kg * jg));
        // lane: row jb * 4 + lane / 8, cells k0 + (lane % 8) + 8 m
        const int j = jb * 4 + lane / 8;
        if (j < ny)
            for (int k = kb * tk + (lane & 7); k < kb * tk + tk && k < nz; k += 8) {
                const uint32_t v = __ldg(flags + gidx(i, j, k, ny, nz));
                fluid |= L0 ? (v & 64u) != 0u : v != 0u;
            }
    }
    const unsigned any = __ballot_sync(0xffffffffu, fluid);
    if (lane == 0 && t < tiles && any) list[atomicAdd(count, 1)] = (int)t;
}

// Red-black colour on the listed tiles: block b handles tiles b, b + gridDim.x, ... with the body of
// the dense colour sweep (rbgs_colour_at; VEC = 4 on the finest level when its tiles are 128 cells;
// Z: as if p were 0 on entry).
template <bool L0, int VEC, bool Z = false>
__global__ void __launch_bounds__(128) k_rbgs_colour_tiles(const int* __restrict__ list, const int* __restrict__ count,
                                                            float* p, const float* __restrict__ b,
                                                            const uint8_t* __restrict__ op0,
                                                            const float4* __restrict__ opc,
                                                            const uint8_t* __restrict__ mask, float delta, int parity,
                                                            int nx, int ny, int nz) {
    pdl_begin();
    const int tk = 32 * VEC, jg = (ny + 3) / 4, kg = (nz + tk - 1) / tk;
    const int n = *count;
    // the next tile's index is loaded while this tile is swept
    int next = blockIdx.x < n ? __ldg(list + blockIdx.x) : 0;
    for (int t = blockIdx.x; t < n; t += gridDim.x) {
        const int tile = next;
        if (t + (int)gridDim.x < n) next = __ldg(list + t + gridDim.x);
        const int kb = tile % kg, rest = tile / kg;
        rbgs_colour_at<L0, VEC, Z>(kb, rest % jg, rest / jg, p, b, op0, opc, mask, delta, parity, nx, ny, nz);
    }
}

// Restriction (restrict_at) of the coarse cells of the listed coarse tiles (32-cell tiles).
template <bool L0>
__global__ void __launch_bounds__(128) k_restrict_tiles(const int* __restrict__ list, const int* __restrict__ count,
                                                         const float* __restrict__ fp, const float* __restrict__ fb,
                                                         const uint8_t* __restrict__ fop0,
                                                         const float4* __restrict__ fopc,
                                                         const uint8_t* __restrict__ fmask, float* __restrict__ cp,
                                                         float* __restrict__ cb, float delta, int fnx, int fny, int fnz,
                                                         int cnx, int cny, int cnz) {
    pdl_begin();
    const int jg = (cny + 3) / 4, kg = (cnz + 31) / 32;
    const int n = *count;
    int next = blockIdx.x < n ? __ldg(list + blockIdx.x) : 0;
    for (int t = blockIdx.x; t < n; t += gridDim.x) {
        const int tile = next;
        if (t + (int)gridDim.x < n) next = __ldg(list + t + gridDim.x);
        const int kb = tile % kg, rest = tile / kg, i = rest / jg, j = (rest % jg) * 4 + threadIdx.y;
        const int k = kb * 32 + threadIdx.x;
        if (j < cny && k < cnz)
            restrict_at<L0>(gidx(i, j, k, cny, cnz), fp, fb, fop0, fopc, fmask, cp, cb, delta, fnx, fny, fnz, cnx,
                            cny, cnz);
    }
}

// Prolongation (prolong_at) into the fine cells of the listed fine tiles (TK = 32 VEC cells along k).
// V4 (finest level, VEC = 4; the caller checked that x is 16-byte and the operator 4-byte aligned):
// each thread's four cells as vectors.
template <bool L0, int VEC, bool V4 = false>
__global__ void __launch_bounds__(128) k_prolong_tiles(const int* __restrict__ list, const int* __restrict__ count,
                                                        const float* __restrict__ ce, float* __restrict__ fp,
                                                        const uint8_t* __restrict__ fop0,
                                                        const uint8_t* __restrict__ fmask, int cnx, int cny, int cnz,
                                                        int fnx, int fny, int fnz, float w) {
    pdl_begin();
    const int tk = 32 * VEC, jg = (fny + 3) / 4, kg = (fnz + tk - 1) / tk;
    const int n = *count;
    int next = blockIdx.x < n ? __ldg(list + blockIdx.x) : 0;
    for (int t = blockIdx.x; t < n; t += gridDim.x) {
        const int tile = next;
        if (t + (int)gridDim.x < n) next = __ldg(list + t + gridDim.x);
        const int kb = tile % kg, rest = tile / kg, i = rest / jg, j = (rest % jg) * 4 + threadIdx.y;
        if (j >= fny) continue;
        if constexpr (V4) {
            static_assert(L0 && VEC == 4, "the vector form is the finest level's");
            // the thread's four cells at once (nz % 4 == 0, 16-byte aligned rows): their operator bytes,
            // x and the parents' corrections in one round of loads; prolong_at's update per cell
            const int k0 = (kb * 32 + threadIdx.x) * 4;
            if (k0 >= fnz || i < 1 || i > fnx - 2 || j < 1 || j > fny - 2) continue;
            const i64 c0 = gidx(i, j, k0, fny, fnz);
            const uchar4 o = *reinterpret_cast<const uchar4*>(fop0 + c0);
            if (!((o.x | o.y | o.z | o.w) & 64u)) continue;
            float4 x = *reinterpret_cast<const float4*>(fp + c0);
            const i64 cb = gidx(min((i - 1) / 2 + 1, cnx - 2), min((j - 1) / 2 + 1, cny - 2), 0, cny, cnz);
            auto parent = [&](int k) { return __ldg(ce + cb + min((k - 1) / 2 + 1, cnz - 2)); };
            const float e0 = parent(k0), e1 = parent(k0 + 1), e2 = parent(k0 + 2), e3 = parent(k0 + 3);
            auto live = [&](unsigned ob, int k) { return (ob & 64u) && k >= 1 && k <= fnz - 2; };
            if (live(o.x, k0)) x.x += w * e0;
            if (live(o.y, k0 + 1)) x.y += w * e1;
            if (live(o.z, k0 + 2)) x.z += w * e2;
            if (live(o.w, k0 + 3)) x.w += w * e3;
            *reinterpret_cast<float4*>(fp + c0) = x;
        } else {
#pragma unroll
            for (int q = 0; q < VEC; ++q) {
                const int k = (kb * 32 + threadIdx.x) * VEC + q;
                if (k < fnz)
                    prolong_at<L0>(gidx(i, j, k, fny, fnz), ce, fp, fop0, fmask, cnx, cny, cnz, fnx, fny, fnz, w);
            }
        }
    }
}

}  // namespace clb
