// Batched scenes: one launch per stage for many independent scenes of different grid sizes (no
// counterpart in the reference, which bakes one scene at a time).
//
// Every field of a batch holds the scenes' grids back to back; a clb_batch_list names the scenes of a
// launch and the prefix of their items (cells of a level, particles, or blocks). A block copies the
// prefix into shared memory, each thread finds its scene by binary search and runs the single-scene
// stage's device body (the *_at / *_block functions of the other headers) on that scene's part of
// the arrays, with the scene's own sizes and float32 constants. So every scene's values are the ones
// a single-scene run computes.
#pragma once
#include "../../include/clb200.h"
#include "binning.cuh"
#include "grid.cuh"
#include "mg_bottom.cuh"
#include "mg_sweep.cuh"
#include "multigrid.cuh"
#include "p2g_tiled.cuh"
#include "particles.cuh"

namespace clb {

struct BList {
    const int32_t* scene;
    const int64_t* start;
    int32_t count;
};

struct BListSmem {
    i64 start[CLB_BATCH_MAX_SCENES + 1];
    int scene[CLB_BATCH_MAX_SCENES];
};

__device__ __forceinline__ void blist_load(const BList& L, BListSmem& m) {
    const int tid = threadIdx.x + threadIdx.y * blockDim.x, nt = blockDim.x * blockDim.y;
    for (int t = tid; t <= L.count; t += nt) m.start[t] = L.start[t];
    for (int t = tid; t < L.count; t += nt) m.scene[t] = L.scene[t];
}

// Position in the list of the scene holding item g: the largest q with start[q] <= g.
__device__ __forceinline__ int blist_find(const BListSmem& m, int count, i64 g) {
    int lo = 0, hi = count - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (m.start[mid] <= g) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// Grid-stride loop over the list's items; f(scene, local item index).
template <class F>
__device__ __forceinline__ void batch_items(const BList& L, i64 total, F&& f) {
    __shared__ BListSmem m;
    blist_load(L, m);
    __syncthreads();
    const i64 stride = (i64)gridDim.x * blockDim.x;
    for (i64 g = (i64)blockIdx.x * blockDim.x + threadIdx.x; g < total; g += stride) {
        const int q = blist_find(m, L.count, g);
        f(m.scene[q], g - m.start[q]);
    }
}

constexpr int BT = 256;

#define CLB_DIMS(g, l) (g).shape[l][0], (g).shape[l][1], (g).shape[l][2]

// ---- particles ------------------------------------------------------------------------------------
// k_bin_count over the batch: keys are offset by the scene's level-0 cell base.
__global__ void __launch_bounds__(PT) kb_bin_count(BList L, i64 n, const clb_batch_scene* __restrict__ G,
                                                   const float* __restrict__ pos, int* __restrict__ counts,
                                                   int* __restrict__ keys, int* __restrict__ ranks) {
    __shared__ BListSmem m;
    __shared__ __align__(16) float sm[3 * PT];
    blist_load(L, m);
    const i64 first = (i64)blockIdx.x * PT;
    stage_particles(pos, first, n, sm);
    __syncthreads();
    const i64 p = first + threadIdx.x;
    int key = -1;
    if (p < n) {
        const clb_batch_scene& g = G[m.scene[blist_find(m, L.count, p)]];
        key = (int)(g.base[0] + bin_key(sm[3 * threadIdx.x], sm[3 * threadIdx.x + 1], sm[3 * threadIdx.x + 2],
                                        g.inv_dx, CLB_DIMS(g, 0)));
    }
    const unsigned peers = __match_any_sync(0xffffffffu, key);
    if (key >= 0) {
        const int lane = threadIdx.x & 31;
        const int leader = __ffs(peers) - 1;
        int base = 0;
        if (lane == leader) base = atomicAdd(counts + key, __popc(peers));
        base = __shfl_sync(peers, base, leader);
        keys[p] = key;
        ranks[p] = base + __popc(peers & ((1u << lane) - 1u));
    }
}

// k_p2g_gather over the batch: eight lanes per cell; bin offsets are batch-wide particle indices.
__global__ void __launch_bounds__(P2G_THREADS) kb_p2g(BList L, i64 total, const clb_batch_scene* __restrict__ G,
                                                      const float* __restrict__ pos, const float* __restrict__ vel,
                                                      const int* __restrict__ offsets, const int* __restrict__ counts,
                                                      float* __restrict__ u, float* __restrict__ v,
                                                      float* __restrict__ w, float* __restrict__ ff, float inv_ppc) {
    __shared__ BListSmem m;
    blist_load(L, m);
    __syncthreads();
    const i64 gi = ((i64)blockIdx.x * P2G_THREADS + threadIdx.x) / P2G_LANES;
    int s = m.scene[0];
    i64 local = -1;
    if (gi < total) {
        const int q = blist_find(m, L.count, gi);
        s = m.scene[q];
        local = gi - m.start[q];
    }
    const clb_batch_scene& g = G[s];
    const i64 o = g.base[0];
    const i64 C = (i64)g.shape[0][0] * g.shape[0][1] * g.shape[0][2];
    p2g_cell(local >= 0 ? local : C, threadIdx.x & (P2G_LANES - 1), pos, vel, offsets + o, counts + o, u + o, v + o,
             w + o, ff + o, g.inv_dx, inv_ppc, CLB_DIMS(g, 0));
}

// k_p2g_tiled over the batch: the scenes' tiles are numbered scene after scene (in list order), block b
// runs tile b of that numbering on its scene; bin offsets are batch-wide particle indices.
__global__ void __launch_bounds__(P2GT_THREADS, 2) kb_p2g_tiled(BList L, const clb_batch_scene* __restrict__ G,
                                                                 const float* __restrict__ pos,
                                                                 const float* __restrict__ vel,
                                                                 const int* __restrict__ offsets,
                                                                 const int* __restrict__ counts, float* __restrict__ u,
                                                                 float* __restrict__ v, float* __restrict__ w,
                                                                 float* __restrict__ ff, float inv_ppc) {
    __shared__ i64 s_start[CLB_BATCH_MAX_SCENES + 1];
    for (int q = threadIdx.x; q < L.count; q += P2GT_THREADS) {
        const clb_batch_scene& g = G[L.scene[q]];
        int tj, tk;
        s_start[q + 1] = p2g_tiled_tiles(CLB_DIMS(g, 0), &tj, &tk);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        s_start[0] = 0;
        for (int q = 1; q <= L.count; ++q) s_start[q] += s_start[q - 1];
    }
    __syncthreads();
    const i64 b = blockIdx.x;
    if (b >= s_start[L.count]) return;  // the whole block leaves together
    int lo = 0, hi = L.count - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (s_start[mid] <= b) lo = mid;
        else hi = mid - 1;
    }
    const clb_batch_scene& g = G[L.scene[lo]];
    const i64 o = g.base[0];
    int tj, tk;
    p2g_tiled_tiles(CLB_DIMS(g, 0), &tj, &tk);
    p2g_tile((int)(b - s_start[lo]), pos, vel, offsets + o, counts + o, u + o, v + o, w + o, ff + o, g.inv_dx, inv_ppc,
             CLB_DIMS(g, 0), tj, tk);
}

// k_particle_update over the batch (records staged through shared memory per block).
__global__ void __launch_bounds__(PT) kb_particle_update(BList L, i64 n, const clb_batch_scene* __restrict__ G,
                                                         float* __restrict__ pos, float* __restrict__ vel,
                                                         const float* u, const float* v, const float* w,
                                                         const float* ou, const float* ov, const float* ow,
                                                         const uint8_t* __restrict__ obs, float flip_ratio, float dt) {
    __shared__ BListSmem m;
    __shared__ __align__(16) float sp[3 * PT];
    __shared__ __align__(16) float sv[3 * PT];
    blist_load(L, m);
    const i64 first = (i64)blockIdx.x * PT;
    stage_particles(pos, first, n, sp);
    stage_particles(vel, first, n, sv);
    __syncthreads();
    const i64 p = first + threadIdx.x;
    if (p < n) {
        const clb_batch_scene& g = G[m.scene[blist_find(m, L.count, p)]];
        const i64 o = g.base[0];
        const int t = 3 * threadIdx.x;
        float p0 = sp[t], p1 = sp[t + 1], p2 = sp[t + 2];
        float v0 = sv[t], v1 = sv[t + 1], v2 = sv[t + 2];
        particle_update_one(p0, p1, p2, v0, v1, v2, nullptr, u + o, v + o, w + o, ou + o, ov + o, ow + o, obs + o,
                            g.inv_dx, CLB_DIMS(g, 0), flip_ratio, dt, g.lower, g.upper[0], g.upper[1], g.upper[2]);
        sp[t] = p0;
        sp[t + 1] = p1;
        sp[t + 2] = p2;
        sv[t] = v0;
        sv[t + 1] = v1;
        sv[t + 2] = v2;
    }
    __syncthreads();
    unstage_particles(pos, first, n, sp);
    unstage_particles(vel, first, n, sv);
}

// ---- grid -------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(BT) kb_update_velocity(BList L, i64 total, const clb_batch_scene* __restrict__ G,
                                                         const float* u, const float* v, const float* w, float* ru,
                                                         float* rv, float* rw, const float* ff, float gx, float gy,
                                                         float gz, float fx, float fy, float fz, float rho, float nu,
                                                         float dt) {
    batch_items(L, total, [&](int s, i64 c) {
        const clb_batch_scene& g = G[s];
        const i64 o = g.base[0];
        update_velocity_at(c, u + o, v + o, w + o, ru + o, rv + o, rw + o, ff + o, gx, gy, gz, fx, fy, fz, rho, nu,
                           g.inv_dx2, dt, CLB_DIMS(g, 0));
    });
}

__global__ void __launch_bounds__(BT) kb_grid_domain_bc(BList L, i64 total, const clb_batch_scene* __restrict__ G,
                                                        float* u, float* v, float* w) {
    batch_items(L, total, [&](int s, i64 c) {
        const clb_batch_scene& g = G[s];
        const i64 o = g.base[0];
        grid_domain_bc_at(c, u + o, v + o, w + o, CLB_DIMS(g, 0));
    });
}

__global__ void __launch_bounds__(BT) kb_grid_obstacle_bc(BList L, i64 total, const clb_batch_scene* __restrict__ G,
                                                          float* u, float* v, float* w, float* ff,
                                                          const uint8_t* obs) {
    batch_items(L, total, [&](int s, i64 c) {
        const clb_batch_scene& g = G[s];
        const i64 o = g.base[0];
        grid_obstacle_bc_at(c, u + o, v + o, w + o, ff + o, obs + o, CLB_DIMS(g, 0));
    });
}

__global__ void __launch_bounds__(BT) kb_extrapolate(BList L, i64 total, const clb_batch_scene* __restrict__ G,
                                                     float* u, float* v, float* w, const uint8_t* obs) {
    batch_items(L, total, [&](int s, i64 c) {
        const clb_batch_scene& g = G[s];
        const i64 o = g.base[0];
        extrapolate_obstacle_velocity_at(c, u + o, v + o, w + o, obs + o, CLB_DIMS(g, 0));
    });
}

__global__ void __launch_bounds__(BT) kb_rhs_op0(BList L, i64 total, const clb_batch_scene* __restrict__ G,
                                                 const float* u, const float* v, const float* w, const float* ff,
                                                 float* rhs, uint8_t* op0) {
    batch_items(L, total, [&](int s, i64 c) {
        const clb_batch_scene& g = G[s];
        const i64 o = g.base[0];
        rhs_op0_at(c, u + o, v + o, w + o, ff + o, rhs + o, op0 + o, g.rho_over_dt, g.inv_dx, CLB_DIMS(g, 0));
    });
}

template <typename PT_>
__global__ void __launch_bounds__(BT) kb_pressure_correction(BList L, i64 total, const clb_batch_scene* __restrict__ G,
                                                             float* u, float* v, float* w, const PT_* p) {
    batch_items(L, total, [&](int s, i64 c) {
        const clb_batch_scene& g = G[s];
        const i64 o = g.base[0];
        pressure_correction_at<PT_>(c, u + o, v + o, w + o, p + o, g.dt_over_rho, g.inv_dx, CLB_DIMS(g, 0));
    });
}

// p32 = (float) p64 and the Neumann ghost copy of both (ghosts read interior cells only).
__global__ void __launch_bounds__(BT) kb_store_neumann(BList L, i64 total, const clb_batch_scene* __restrict__ G,
                                                       double* p64, float* p32) {
    batch_items(L, total, [&](int s, i64 c) {
        const clb_batch_scene& g = G[s];
        const i64 o = g.base[0];
        const int nx = g.shape[0][0], ny = g.shape[0][1], nz = g.shape[0][2];
        int i, j, k;
        gcoord(c, ny, nz, i, j, k);
        if (interior(i, j, k, nx, ny, nz)) {
            p32[o + c] = (float)p64[o + c];
            return;
        }
        const i64 src = o + gidx(clampi(i, 1, nx - 2), clampi(j, 1, ny - 2), clampi(k, 1, nz - 2), ny, nz);
        const double v = p64[src];  // an interior cell: never written by this launch
        p64[o + c] = v;
        p32[o + c] = (float)v;
    });
}

__global__ void __launch_bounds__(BT) kb_neumann(BList L, i64 total, const clb_batch_scene* __restrict__ G, float* p) {
    batch_items(L, total, [&](int s, i64 c) {
        const clb_batch_scene& g = G[s];
        neumann_domain_bc_at<float>(c, p + g.base[0], CLB_DIMS(g, 0));
    });
}

__global__ void __launch_bounds__(BT) kb_ir_init(BList L, i64 total, const clb_batch_scene* __restrict__ G,
                                                 const float* p, const uint8_t* op0, double* p64) {
    batch_items(L, total, [&](int s, i64 c) {
        const clb_batch_scene& g = G[s];
        const i64 o = g.base[0];
        ir_init_at(c, p + o, op0 + o, p64 + o, CLB_DIMS(g, 0));
    });
}

// ---- multigrid ----------------------------------------------------------------------------------------
template <int FS>  // 0: from the packed finest level, 1: from a float4 coarse level
__global__ void __launch_bounds__(BT) kb_coarse_operator(BList L, i64 total, const clb_batch_scene* __restrict__ G,
                                                         int level, const uint8_t* op0, const float4* fop,
                                                         const uint8_t* fmask, float4* cop, uint8_t* cmask) {
    batch_items(L, total, [&](int s, i64 ci) {
        const clb_batch_scene& g = G[s];
        const i64 of = g.base[level - 1], oc = g.base[level];
        coarse_operator_at<FS, false>(ci, FS == 0 ? op0 + of : nullptr, FS == 0 ? nullptr : fop + of,
                                      FS == 0 ? nullptr : fmask + of, cop + oc, cmask + oc, nullptr,
                                      CLB_DIMS(g, level - 1), CLB_DIMS(g, level));
    });
}

// One red-black colour, one thread per cell, on level `level` of the listed scenes.
template <bool L0>
__global__ void __launch_bounds__(BT) kb_rbgs(BList L, i64 total, const clb_batch_scene* __restrict__ G, int level,
                                              float* p, const float* b, const uint8_t* op0, const float4* opc,
                                              const uint8_t* mask, int parity) {
    batch_items(L, total, [&](int s, i64 c) {
        const clb_batch_scene& g = G[s];
        const i64 o = g.base[level];
        rbgs_at<L0>(c, p + o, b + o, L0 ? op0 + o : nullptr, L0 ? nullptr : opc + o, L0 ? nullptr : mask + o,
                    g.delta, parity, CLB_DIMS(g, level));
    });
}

// The level-0 row sweep (k_rbgs_colour) over the batch: list items are blocks of (32, 4) threads.
template <int VEC>
__global__ void __launch_bounds__(128) kb_rbgs_colour(BList L, const clb_batch_scene* __restrict__ G, float* p,
                                                      const float* b, const uint8_t* op0, int parity) {
    __shared__ BListSmem m;
    blist_load(L, m);
    __syncthreads();
    const int q = blist_find(m, L.count, blockIdx.x);
    const clb_batch_scene& g = G[m.scene[q]];
    const int nx = g.shape[0][0], ny = g.shape[0][1], nz = g.shape[0][2];
    const int gxb = (nz + 32 * VEC - 1) / (32 * VEC), gyb = (ny + 3) / 4;
    const int local = (int)(blockIdx.x - m.start[q]);
    const int bz = local / (gxb * gyb), r = local - bz * gxb * gyb, by = r / gxb, bx = r - by * gxb;
    const i64 o = g.base[0];
    rbgs_colour_at<true, VEC>(bx, by, bz, p + o, b + o, op0 + o, nullptr, nullptr, g.delta, parity, nx, ny, nz);
}

// Restriction of level `level` into level + 1; list items are coarse cells.
template <bool L0>
__global__ void __launch_bounds__(BT) kb_restrict(BList L, i64 total, const clb_batch_scene* __restrict__ G, int level,
                                                  const float* fp, const float* fb, const uint8_t* fop0,
                                                  const float4* fopc, const uint8_t* fmask, float* cp, float* cb) {
    batch_items(L, total, [&](int s, i64 ci) {
        const clb_batch_scene& g = G[s];
        const i64 of = g.base[level], oc = g.base[level + 1];
        restrict_at<L0>(ci, fp + of, fb + of, L0 ? fop0 + of : nullptr, L0 ? nullptr : fopc + of,
                        L0 ? nullptr : fmask + of, cp + oc, cb + oc, g.delta, CLB_DIMS(g, level),
                        CLB_DIMS(g, level + 1));
    });
}

// Prolongation of level + 1 into level `level`; list items are fine cells.
template <bool L0>
__global__ void __launch_bounds__(BT) kb_prolong(BList L, i64 total, const clb_batch_scene* __restrict__ G, int level,
                                                 const float* ce, float* fp, const uint8_t* fop0,
                                                 const uint8_t* fmask, float w) {
    batch_items(L, total, [&](int s, i64 f) {
        const clb_batch_scene& g = G[s];
        const i64 of = g.base[level], oc = g.base[level + 1];
        prolong_at<L0>(f, ce + oc, fp + of, L0 ? fop0 + of : nullptr, L0 ? nullptr : fmask + of,
                       CLB_DIMS(g, level + 1), CLB_DIMS(g, level), w);
    });
}

// Bottom visit of level `level` (and level + 1), one block per listed scene.
template <int KA, int KB>
__global__ void __launch_bounds__(BOTTOM_THREADS, 1)
    kb_bottom_visit(BList L, const clb_batch_scene* __restrict__ G, int level, float* pa, const float* ba,
                    const float4* opa, const uint8_t* ma, float* pb, float* bb, const float4* opb, const uint8_t* mb,
                    int pre, int post, int coarse_iters, float w) {
    const clb_batch_scene& g = G[L.scene[blockIdx.x]];
    const i64 oa = g.base[level], ob = g.base[level + 1];
    bottom_visit_block<KA, KB, false>(pa + oa, ba + oa, opa + oa, ma + oa, CLB_DIMS(g, level), pb + ob, bb + ob,
                                      opb + ob, mb + ob, CLB_DIMS(g, level + 1), g.delta, pre, post, coarse_iters,
                                      nullptr, 2, w);
}

// Coarse solve of level `level` from shared memory, one block per listed scene.
__global__ void __launch_bounds__(COARSE_THREADS) kb_coarse_solve(BList L, const clb_batch_scene* __restrict__ G,
                                                                  int level, float* p, const float* b,
                                                                  const float4* op, const uint8_t* mask,
                                                                  int iterations) {
    const clb_batch_scene& g = G[L.scene[blockIdx.x]];
    const i64 o = g.base[level];
    coarse_solve_block<true, false, false>(p + o, b + o, nullptr, op + o, mask + o, g.delta, iterations,
                                           CLB_DIMS(g, level), nullptr);
}

// ---- FP64 reductions: `R` blocks per scene (block b works for scene b / R) ------------------------------
template <typename PT_, int MODE>
__global__ void __launch_bounds__(RN_THREADS) kb_residual_rows(const clb_batch_scene* __restrict__ G, int R,
                                                               const PT_* p_in, const float* e, double* p_out,
                                                               const float* b, const uint8_t* op0, float* r_out,
                                                               double2* partials, const float* d_in, float* d_out,
                                                               const double* state) {
    const int s = blockIdx.x / R, blk = blockIdx.x - s * R;
    const clb_batch_scene& g = G[s];
    const i64 o = g.base[0];
    const double inv_delta2 = 1.0 / ((double)g.delta * (double)g.delta);
    residual_rows_block<PT_, MODE>(blk, R, p_in + o, e ? e + o : nullptr, p_out ? p_out + o : nullptr, b + o, op0 + o,
                                   inv_delta2, CLB_DIMS(g, 0), r_out ? r_out + o : nullptr, partials + blockIdx.x,
                                   d_in ? d_in + o : nullptr, d_out ? d_out + o : nullptr,
                                   state ? state + 4 * s : nullptr);
}

__global__ void kb_reduce_partials(int R, const double2* partials, double2* out) {
    reduce_partials_block(partials + (i64)blockIdx.x * R, R, out + blockIdx.x);
}

__global__ void __launch_bounds__(RN_THREADS) kb_fcg_dots(const clb_batch_scene* __restrict__ G, int R, const float* z,
                                                          const float* d, const float* r, const uint8_t* op0,
                                                          Sum4* partials) {
    const int s = blockIdx.x / R, blk = blockIdx.x - s * R;
    const clb_batch_scene& g = G[s];
    const i64 o = g.base[0];
    const double inv_delta2 = 1.0 / ((double)g.delta * (double)g.delta);
    fcg_dots_block(blk, R, z + o, d + o, r + o, op0 + o, inv_delta2, CLB_DIMS(g, 0), partials + blockIdx.x);
}

__global__ void kb_fcg_scalars(int R, const Sum4* partials, double* state) {
    fcg_scalars_block(partials + (i64)blockIdx.x * R, R, state + 4 * blockIdx.x);
}

#undef CLB_DIMS

}  // namespace clb
