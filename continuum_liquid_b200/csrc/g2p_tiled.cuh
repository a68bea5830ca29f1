// The fused particle update (G2P with the FLIP/PIC blend, previous-position copy, advection, domain and
// obstacle conditions; particles.cl:229-276, boundary_conditions.cl:69-97 and 175-264) walking the
// bins of a tile instead of the particle array.
//
// Why: k_particle_update samples six grid arrays at 8 nodes each per particle (48 loads), most from L2:
// neighbouring particles share nodes, but the working set of a launch is the whole grid. The particles
// are sorted by bin when the update runs (the step's counting sort), so a tile's particles are the
// concatenation of its bins' ranges. A block stages the six arrays over the tile's bins plus the nodes
// those bins' particles sample in shared memory once, then its warps run over the particles of one
// row of bins at a time, every lane on its own particle (a row's particles are contiguous, so lanes do
// not wait on a row's fullest bin).
//
// Which nodes a bin's particles sample: a particle in bin b (b = clamp(floor(s - 0.5), 0, n - 2) per
// axis, s = p / dx) samples the face component of its own axis at base clamp(floor(s - 1), 0, n - 2),
// which is b - 1 or b (s - 1 and s - 0.5 are exact in float32 at these magnitudes), and the two other
// components at base b; with the base's +1 node, nodes b - 1 .. b + 1 along every axis. So a tile of
// bins [i0, i0 + TI) x [j0, j0 + TJ) x [k0, k0 + TK) stages nodes [i0 - 1, i0 + TI] x ... .
//
// Every particle's arithmetic is k_particle_update's (particle_update_with with a fetch from shared
// memory): the results are the same bit for bit, whichever kernel runs.
#pragma once
#include "particles.cuh"

namespace clb {

constexpr int PUT_TI = 8, PUT_TJ = 8, PUT_TK = 30;
constexpr int PUT_RI = PUT_TI + 2, PUT_RJ = PUT_TJ + 2, PUT_RK = PUT_TK + 2;
constexpr int PUT_REGION = PUT_RI * PUT_RJ * PUT_RK;
constexpr int PUT_WARPS = 8;
constexpr int PUT_THREADS = 32 * PUT_WARPS;
constexpr int PUT_SMEM = 6 * PUT_REGION * 4;  // u, v, w, u_old, v_old, w_old over the region
static_assert(PUT_RK == 32, "a staged row is one warp wide");

__host__ __device__ __forceinline__ int particle_update_tiles(int nx, int ny, int nz, int* tiles_j, int* tiles_k) {
    // bins run over 0 .. n - 2 on every axis
    const int ti = (nx - 1 + PUT_TI - 1) / PUT_TI;
    *tiles_j = (ny - 1 + PUT_TJ - 1) / PUT_TJ;
    *tiles_k = (nz - 1 + PUT_TK - 1) / PUT_TK;
    return ti * *tiles_j * *tiles_k;
}

// One block per tile of bins. offsets/counts: the bins of the sorted particle arrays pos/vel.
template <bool MOVING>
__global__ void __launch_bounds__(PUT_THREADS, 2)
    k_particle_update_tiled(float* __restrict__ pos, float* __restrict__ vel, float* __restrict__ prev_out,
                            const float* __restrict__ u, const float* __restrict__ v, const float* __restrict__ w,
                            const float* __restrict__ ou, const float* __restrict__ ov, const float* __restrict__ ow,
                            const uint8_t* __restrict__ obs, const int* __restrict__ offsets,
                            const int* __restrict__ counts, float inv_dx, int nx, int ny, int nz, float flip_ratio,
                            float dt, float lower, float ux, float uy, float uz, int tiles_j, int tiles_k,
                            RigidMotion motion) {
    extern __shared__ __align__(16) float put_smem[];
    const int tile = blockIdx.x;
    const int tk = tile % tiles_k, tj = (tile / tiles_k) % tiles_j, ti = tile / (tiles_k * tiles_j);
    const int i0 = ti * PUT_TI, j0 = tj * PUT_TJ, k0 = tk * PUT_TK;
    const int gi = i0 - 1, gj = j0 - 1, gk = k0 - 1;  // region origin
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int k_last = min(k0 + PUT_TK, nz - 1) - 1;  // last bin along k of this tile

    // the tile's particle ranges, one per row of bins; a tile without particles stages nothing
    int any = 0;
    for (int r = threadIdx.x; r < PUT_TI * PUT_TJ; r += PUT_THREADS) {
        const int bx = i0 + r / PUT_TJ, by = j0 + r % PUT_TJ;
        if (bx > nx - 2 || by > ny - 2 || k0 > k_last) continue;
        const i64 first = gidx(bx, by, k0, ny, nz), last = gidx(bx, by, k_last, ny, nz);
        any |= (__ldg(offsets + last) + __ldg(counts + last) - __ldg(offsets + first)) > 0;
    }
    if (!__syncthreads_or(any)) return;

    // stage the six arrays (rows of 32 nodes along k: one warp per row and array); nodes outside the
    // grid are never sampled
    const float* src[6] = {u, v, w, ou, ov, ow};
#pragma unroll
    for (int a = 0; a < 6; ++a) {
        float* dst = put_smem + a * PUT_REGION;
        for (int row = warp; row < PUT_RI * PUT_RJ; row += PUT_WARPS) {
            const int i = gi + row / PUT_RJ, j = gj + row % PUT_RJ, k = gk + lane;
            float val = 0.0f;
            if (i >= 0 && i < nx && j >= 0 && j < ny && k >= 0 && k < nz) val = __ldg(src[a] + gidx(i, j, k, ny, nz));
            dst[row * PUT_RK + lane] = val;
        }
    }
    __syncthreads();

    const float* su = put_smem;
    auto sample = [&](int axis, float offx, float offy, float offz, float* old, float px, float py, float pz) {
        const float* cur = su + axis * PUT_REGION;
        const float* prv = su + (3 + axis) * PUT_REGION;
        auto fetch = [&](int i, int j, int k) {
            const int q = ((i - gi) * PUT_RJ + (j - gj)) * PUT_RK + (k - gk);
            return make_float2(cur[q], prv[q]);
        };
        return sample_pair_with(fetch, px, py, pz, inv_dx, offx, offy, offz, nx, ny, nz, old);
    };
    for (int r = warp; r < PUT_TI * PUT_TJ; r += PUT_WARPS) {
        const int bx = i0 + r / PUT_TJ, by = j0 + r % PUT_TJ;
        if (bx > nx - 2 || by > ny - 2 || k0 > k_last) continue;  // warp-uniform
        const int begin = __ldg(offsets + gidx(bx, by, k0, ny, nz));
        const i64 last = gidx(bx, by, k_last, ny, nz);
        const int end = __ldg(offsets + last) + __ldg(counts + last);
        // two particles per lane and round, both records loaded before either is updated (more loads in
        // flight at this occupancy)
        for (int p = begin + lane; p < end; p += 64) {
            const int q = p + 32;
            const bool two = q < end;
            float a[6], c[6] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
            for (int t = 0; t < 3; ++t) {
                a[t] = pos[3 * (i64)p + t];
                a[3 + t] = vel[3 * (i64)p + t];
            }
            if (two)
#pragma unroll
                for (int t = 0; t < 3; ++t) {
                    c[t] = pos[3 * (i64)q + t];
                    c[3 + t] = vel[3 * (i64)q + t];
                }
            auto update = [&](float* r, int idx) {
                const float x0 = r[0], x1 = r[1], x2 = r[2];  // the sampling position (pre-advection)
                auto at = [&](int axis, float offx, float offy, float offz, float* old) {
                    return sample(axis, offx, offy, offz, old, x0, x1, x2);
                };
                particle_update_with<MOVING>(r[0], r[1], r[2], r[3], r[4], r[5],
                                             prev_out ? prev_out + 3 * (i64)idx : nullptr, at, obs, inv_dx, nx, ny,
                                             nz, flip_ratio, dt, lower, ux, uy, uz, motion);
            };
            update(a, p);
            if (two) update(c, q);
#pragma unroll
            for (int t = 0; t < 3; ++t) {
                pos[3 * (i64)p + t] = a[t];
                vel[3 * (i64)p + t] = a[3 + t];
            }
            if (two)
#pragma unroll
                for (int t = 0; t < 3; ++t) {
                    pos[3 * (i64)q + t] = c[t];
                    vel[3 * (i64)q + t] = c[3 + t];
                }
        }
    }
}

}  // namespace clb
