// Triangle-mesh voxelisation (Solver/Kernel/OpenCL/voxelise_mesh.cl): each interior cell centre
// casts one ray along a fixed oblique direction and counts Moller-Trumbore hits; an odd count marks
// the cell solid. The ray-triangle arithmetic is the reference's, term for term, so occupancy is
// bit-exact against the CPU restatement.
//
// B200 mapping: a block owns a 4x4x16 brick of cells (k fastest). Triangles are staged through
// shared memory in chunks. Before the exact test, a triangle is skipped for the whole brick when it
// provably cannot be hit by any of the brick's rays:
//   a hit point is h = o + t*d with t > 0 and every component of d positive, so h >= o
//   componentwise, and o >= o_min, the brick's first cell centre (float rounding of the centre
//   formula is monotone in the cell index). A triangle whose largest vertex coordinate on some axis
//   is below o_min on that axis minus a margin lies behind every ray of the brick: its exact ray
//   parameter is below -margin, and the computed parameter of the exact test differs from it by
//   orders of magnitude less than that (margin = 8 cell widths + 1e-4 |o_min| + 1e-6), so the exact
//   test rejects it too. The cull is also checked against the unculled kernel in the tests.
#pragma once
#include "common.cuh"

namespace clb {

constexpr int VOX_BI = 4, VOX_BJ = 4, VOX_BK = 16;
constexpr int VOX_THREADS = VOX_BI * VOX_BJ * VOX_BK;
constexpr int VOX_CHUNK = 512;

// voxelise_mesh.cl:5-22 ray_hit
__device__ __forceinline__ int ray_hit(float o0, float o1, float o2, float d0, float d1, float d2,
                                       const float* __restrict__ t9) {
    const float a0 = t9[0], a1 = t9[1], a2 = t9[2];
    const float e10 = t9[3] - a0, e11 = t9[4] - a1, e12 = t9[5] - a2;
    const float e20 = t9[6] - a0, e21 = t9[7] - a1, e22 = t9[8] - a2;
    const float p0 = d1 * e22 - d2 * e21, p1 = d2 * e20 - d0 * e22, p2 = d0 * e21 - d1 * e20;
    const float det = e10 * p0 + e11 * p1 + e12 * p2;
    if (fabsf(det) < 1.0e-7f) return 0;
    const float inv = 1.0f / det;
    const float t0 = o0 - a0, t1 = o1 - a1, t2 = o2 - a2;
    const float uu = (t0 * p0 + t1 * p1 + t2 * p2) * inv;
    if (uu < 0.0f || uu > 1.0f) return 0;
    const float q0 = t1 * e12 - t2 * e11, q1 = t2 * e10 - t0 * e12, q2 = t0 * e11 - t1 * e10;
    const float vv = (d0 * q0 + d1 * q1 + d2 * q2) * inv;
    if (vv < 0.0f || uu + vv > 1.0f) return 0;
    return (e20 * q0 + e21 * q1 + e22 * q2) * inv > 1.0e-6f;
}

template <bool CULL>
__global__ void __launch_bounds__(VOX_THREADS) k_voxelise(const float* __restrict__ tris, uint8_t* __restrict__ mask,
                                                           int T, int nx, int ny, int nz, float delta, float ox,
                                                           float oy, float oz, float d0, float d1, float d2) {
    __shared__ float s_tri[VOX_CHUNK * 9];
    __shared__ int s_list[VOX_CHUNK];
    __shared__ int s_count;
    const int tk = threadIdx.x % VOX_BK, tj = (threadIdx.x / VOX_BK) % VOX_BJ, ti = threadIdx.x / (VOX_BK * VOX_BJ);
    const int k = blockIdx.x * VOX_BK + tk, j = blockIdx.y * VOX_BJ + tj, i = blockIdx.z * VOX_BI + ti;
    const bool active = i >= 1 && j >= 1 && k >= 1 && i < nx - 1 && j < ny - 1 && k < nz - 1;
    const float o0 = ox + ((float)i + 0.5f) * delta, o1 = oy + ((float)j + 0.5f) * delta,
                o2 = oz + ((float)k + 0.5f) * delta;
    // smallest ray origin of the brick on each axis (the brick's first cell centres)
    const float m0 = ox + ((float)(blockIdx.z * VOX_BI) + 0.5f) * delta;
    const float m1 = oy + ((float)(blockIdx.y * VOX_BJ) + 0.5f) * delta;
    const float m2 = oz + ((float)(blockIdx.x * VOX_BK) + 0.5f) * delta;
    const float g0 = m0 - (8.0f * delta + 1.0e-4f * fabsf(m0) + 1.0e-6f);
    const float g1 = m1 - (8.0f * delta + 1.0e-4f * fabsf(m1) + 1.0e-6f);
    const float g2 = m2 - (8.0f * delta + 1.0e-4f * fabsf(m2) + 1.0e-6f);
    int hits = 0;
    for (int base = 0; base < T; base += VOX_CHUNK) {
        const int n = min(VOX_CHUNK, T - base);
        if (CULL) {
            if (threadIdx.x == 0) s_count = 0;
            __syncthreads();
            for (int t = threadIdx.x; t < n; t += VOX_THREADS) {
                const float* src = tris + 9 * (i64)(base + t);
                const float x = fmaxf(fmaxf(__ldg(src), __ldg(src + 3)), __ldg(src + 6));
                const float y = fmaxf(fmaxf(__ldg(src + 1), __ldg(src + 4)), __ldg(src + 7));
                const float z = fmaxf(fmaxf(__ldg(src + 2), __ldg(src + 5)), __ldg(src + 8));
                if (!(x < g0 || y < g1 || z < g2)) s_list[atomicAdd(&s_count, 1)] = base + t;
            }
            __syncthreads();
            const int m = s_count;
            // the kept triangles arrive in any order; the hit count (an integer) does not depend on it
            for (int t = threadIdx.x; t < m * 9; t += VOX_THREADS) {
                const int q = t / 9, r = t - q * 9;
                s_tri[t] = __ldg(tris + 9 * (i64)s_list[q] + r);
            }
            __syncthreads();
            if (active)
                for (int t = 0; t < m; ++t) hits += ray_hit(o0, o1, o2, d0, d1, d2, s_tri + 9 * t);
        } else {
            for (int t = threadIdx.x; t < n * 9; t += VOX_THREADS) s_tri[t] = __ldg(tris + 9 * (i64)base + t);
            __syncthreads();
            if (active)
                for (int t = 0; t < n; ++t) hits += ray_hit(o0, o1, o2, d0, d1, d2, s_tri + 9 * t);
        }
        __syncthreads();
    }
    if (active && (hits & 1)) mask[gidx(i, j, k, ny, nz)] = 1;
}

// voxelise_mesh.cl:24 normalize((1, 0.3713907, 0.2178311)), restated as v / sqrt(dot(v, v)) in
// correctly rounded float arithmetic; evaluated on the host so every launch uses the same three
// floats.
static inline void voxelise_direction(float out[3]) {
    volatile float x = 1.0f, y = 0.3713907f, z = 0.2178311f;
    volatile float xx = x * x, yy = y * y, zz = z * z;
    volatile float s = xx + yy;
    s = s + zz;
    const float len = sqrtf(s);
    out[0] = x / len;
    out[1] = y / len;
    out[2] = z / len;
}

}  // namespace clb
