// Grid-to-particle transfer, advection and particle boundary conditions
// (Solver/Kernel/OpenCL/particles.cl:229-276, boundary_conditions.cl:69-97 and 175-264).
#pragma once
#include "binning.cuh"
#include "moving.cuh"

namespace clb {

// particles.cl:12-42 staggered_interpolation_base/fraction + sample_field for one face component of
// the current and the old grid at once. `fetch(i, j, k)` returns {cur, old} at node (i, j, k).
// Returns the sample of `cur` and writes the sample of `old` into *old_sample.
template <class Fetch>
__device__ __forceinline__ float sample_pair_with(Fetch&& fetch, float px, float py, float pz, float inv_dx,
                                                  float offx, float offy, float offz, int nx, int ny, int nz,
                                                  float* old_sample) {
    const float sx = px * inv_dx - offx, sy = py * inv_dx - offy, sz = pz * inv_dx - offz;
    const int bx = clampi((int)floorf(sx), 0, nx - 2);
    const int by = clampi((int)floorf(sy), 0, ny - 2);
    const int bz = clampi((int)floorf(sz), 0, nz - 2);
    const float fx = fminf(fmaxf(px * inv_dx - offx - (float)bx, 0.0f), 1.0f);
    const float fy = fminf(fmaxf(py * inv_dx - offy - (float)by, 0.0f), 1.0f);
    const float fz = fminf(fmaxf(pz * inv_dx - offz - (float)bz, 0.0f), 1.0f);
    float a = 0.0f, b = 0.0f;
#pragma unroll
    for (int ox = 0; ox <= 1; ++ox)
#pragma unroll
        for (int oy = 0; oy <= 1; ++oy)
#pragma unroll
            for (int oz = 0; oz <= 1; ++oz) {
                const float wgt = (ox ? fx : 1.0f - fx) * (oy ? fy : 1.0f - fy) * (oz ? fz : 1.0f - fz);
                const float2 val = fetch(bx + ox, by + oy, bz + oz);
                a += wgt * val.x;
                b += wgt * val.y;
            }
    *old_sample = b;
    return a;
}

__device__ __forceinline__ float sample_pair(const float* __restrict__ cur, const float* __restrict__ old, float px,
                                             float py, float pz, float inv_dx, float offx, float offy, float offz,
                                             int nx, int ny, int nz, float* old_sample) {
    auto fetch = [&](int i, int j, int k) {
        const i64 c = gidx(i, j, k, ny, nz);
        return make_float2(__ldg(cur + c), __ldg(old + c));
    };
    return sample_pair_with(fetch, px, py, pz, inv_dx, offx, offy, offz, nx, ny, nz, old_sample);
}

// particles.cl:229-262 grid_to_particle with the FLIP/PIC blend extension (flip_ratio == 1 is the
// reference's pure FLIP update v += I(u) - I(u_old)). `sample(axis, offx, offy, offz, &old)` samples
// face component `axis` of the current and the old grid.
template <class Sample>
__device__ __forceinline__ void g2p_velocity_with(float& v0, float& v1, float& v2, Sample&& sample, float flip_ratio) {
    float o0, o1, o2;
    const float c0 = sample(0, 1.0f, 0.5f, 0.5f, &o0);
    const float c1 = sample(1, 0.5f, 1.0f, 0.5f, &o1);
    const float c2 = sample(2, 0.5f, 0.5f, 1.0f, &o2);
    const float f0 = v0 + (c0 - o0), f1 = v1 + (c1 - o1), f2 = v2 + (c2 - o2);
    if (flip_ratio == 1.0f) {
        v0 = f0;
        v1 = f1;
        v2 = f2;
    } else {
        const float pic = 1.0f - flip_ratio;
        v0 = flip_ratio * f0 + pic * c0;
        v1 = flip_ratio * f1 + pic * c1;
        v2 = flip_ratio * f2 + pic * c2;
    }
}

__device__ __forceinline__ void g2p_velocity(float& v0, float& v1, float& v2, float px, float py, float pz,
                                             const float* u, const float* v, const float* w, const float* ou,
                                             const float* ov, const float* ow, float inv_dx, int nx, int ny, int nz,
                                             float flip_ratio) {
    auto sample = [&](int axis, float offx, float offy, float offz, float* old) {
        const float* cur = axis == 0 ? u : (axis == 1 ? v : w);
        const float* prev = axis == 0 ? ou : (axis == 1 ? ov : ow);
        return sample_pair(cur, prev, px, py, pz, inv_dx, offx, offy, offz, nx, ny, nz, old);
    };
    g2p_velocity_with(v0, v1, v2, sample, flip_ratio);
}

// boundary_conditions.cl:69-97 particle_domain_bc for one component.
__device__ __forceinline__ void domain_bc_axis(float& x, float& vel, float lower, float upper) {
    const bool lo = x < lower, hi = x > upper;
    float y = x;
    if (lo) y = 2.0f * lower - x;
    if (hi) y = 2.0f * upper - y;
    y = y < lower ? lower : (y > upper ? upper : y);
    x = y;
    if (lo || hi) vel = 0.0f;
}

__device__ __forceinline__ int cell_of(float x, float inv_dx, int n) { return clampi((int)(x * inv_dx), 0, n - 1); }

// boundary_conditions.cl:175-264 particle_obstacle_bc. MOVING (no counterpart in the reference): the
// collider moves with `motion`, and only the velocity relative to it loses its inward component.
template <bool MOVING = false>
__device__ __forceinline__ void obstacle_bc(float& p0, float& p1, float& p2, float q0, float q1, float q2, float& v0,
                                            float& v1, float& v2, const uint8_t* __restrict__ obs, float inv_dx,
                                            int nx, int ny, int nz, RigidMotion motion = RigidMotion{}) {
    const int c0 = cell_of(p0, inv_dx, nx), c1 = cell_of(p1, inv_dx, ny), c2 = cell_of(p2, inv_dx, nz);
    if (!__ldg(obs + gidx(c0, c1, c2, ny, nz))) return;
    const int r0 = cell_of(q0, inv_dx, nx), r1 = cell_of(q1, inv_dx, ny), r2 = cell_of(q2, inv_dx, nz);
    float n0 = 0.0f, n1 = 0.0f, n2 = 0.0f;
    if ((r0 != c0 || r1 != c1 || r2 != c2) && !__ldg(obs + gidx(r0, r1, r2, ny, nz))) {
        n0 = (float)(r0 - c0);
        n1 = (float)(r1 - c1);
        n2 = (float)(r2 - c2);
    } else {
        if (c0 > 0 && !__ldg(obs + gidx(c0 - 1, c1, c2, ny, nz))) n0 -= 1.0f;
        if (c0 + 1 < nx && !__ldg(obs + gidx(c0 + 1, c1, c2, ny, nz))) n0 += 1.0f;
        if (c1 > 0 && !__ldg(obs + gidx(c0, c1 - 1, c2, ny, nz))) n1 -= 1.0f;
        if (c1 + 1 < ny && !__ldg(obs + gidx(c0, c1 + 1, c2, ny, nz))) n1 += 1.0f;
        if (c2 > 0 && !__ldg(obs + gidx(c0, c1, c2 - 1, ny, nz))) n2 -= 1.0f;
        if (c2 + 1 < nz && !__ldg(obs + gidx(c0, c1, c2 + 1, ny, nz))) n2 += 1.0f;
    }
    const float len = sqrtf(n0 * n0 + n1 * n1 + n2 * n2);
    if (len > 0.0f) {
        n0 = n0 / len;
        n1 = n1 / len;
        n2 = n2 / len;
    } else {
        const float f0 = q0 - p0, f1 = q1 - p1, f2 = q2 - p2;
        const float fl = sqrtf(f0 * f0 + f1 * f1 + f2 * f2);
        if (fl > 0.0f) {
            n0 = f0 / fl;
            n1 = f1 / fl;
            n2 = f2 / fl;
        } else {
            n0 = 0.0f;
            n1 = 0.0f;
            n2 = 1.0f;
        }
    }
    float vn;
    if constexpr (MOVING) {
        float s0, s1, s2;
        rigid_velocity(motion, p0, p1, p2, s0, s1, s2);
        const float r0 = v0 - s0, r1 = v1 - s1, r2 = v2 - s2;
        vn = r0 * n0 + r1 * n1 + r2 * n2;
    } else {
        vn = v0 * n0 + v1 * n1 + v2 * n2;
    }
    if (vn < 0.0f) {
        v0 = v0 - vn * n0;
        v1 = v1 - vn * n1;
        v2 = v2 - vn * n2;
    }
    const float dx = 1.0f / inv_dx;
    float k0 = p0, k1 = p1, k2 = p2;
    if (n0 < 0.0f) k0 = 2.0f * ((float)c0 * dx) - p0;
    else if (n0 > 0.0f) k0 = 2.0f * ((float)(c0 + 1) * dx) - p0;
    if (n1 < 0.0f) k1 = 2.0f * ((float)c1 * dx) - p1;
    else if (n1 > 0.0f) k1 = 2.0f * ((float)(c1 + 1) * dx) - p1;
    if (n2 < 0.0f) k2 = 2.0f * ((float)c2 * dx) - p2;
    else if (n2 > 0.0f) k2 = 2.0f * ((float)(c2 + 1) * dx) - p2;
    if (__ldg(obs + gidx(cell_of(k0, inv_dx, nx), cell_of(k1, inv_dx, ny), cell_of(k2, inv_dx, nz), ny, nz))) {
        k0 = q0;
        k1 = q1;
        k2 = q2;
    }
    p0 = k0;
    p1 = k1;
    p2 = k2;
}

// Reference kernels, one launch each (used by the stage API and the per-kernel parity tests).
__global__ void __launch_bounds__(PT) k_grid_to_particle(float* __restrict__ vel, const float* __restrict__ pos,
                                                          const float* u, const float* v, const float* w,
                                                          const float* ou, const float* ov, const float* ow, i64 n,
                                                          float inv_dx, int nx, int ny, int nz, float flip_ratio) {
    const i64 p = (i64)blockIdx.x * PT + threadIdx.x;
    if (p >= n) return;
    float v0 = vel[3 * p], v1 = vel[3 * p + 1], v2 = vel[3 * p + 2];
    g2p_velocity(v0, v1, v2, __ldg(pos + 3 * p), __ldg(pos + 3 * p + 1), __ldg(pos + 3 * p + 2), u, v, w, ou, ov, ow,
                 inv_dx, nx, ny, nz, flip_ratio);
    vel[3 * p] = v0;
    vel[3 * p + 1] = v1;
    vel[3 * p + 2] = v2;
}

__global__ void __launch_bounds__(PT) k_advect(float* __restrict__ pos, const float* __restrict__ vel, i64 n3,
                                                float dt) {
    const i64 i = (i64)blockIdx.x * PT + threadIdx.x;
    if (i < n3) pos[i] = pos[i] + dt * vel[i];
}

__global__ void __launch_bounds__(PT) k_particle_domain_bc(float* __restrict__ pos, float* __restrict__ vel, i64 n,
                                                            float lower, float ux, float uy, float uz) {
    const i64 p = (i64)blockIdx.x * PT + threadIdx.x;
    if (p >= n) return;
    domain_bc_axis(pos[3 * p], vel[3 * p], lower, ux);
    domain_bc_axis(pos[3 * p + 1], vel[3 * p + 1], lower, uy);
    domain_bc_axis(pos[3 * p + 2], vel[3 * p + 2], lower, uz);
}

template <bool MOVING = false>
__global__ void __launch_bounds__(PT) k_particle_obstacle_bc(float* __restrict__ pos, const float* __restrict__ prev,
                                                              float* __restrict__ vel, const uint8_t* __restrict__ obs,
                                                              i64 n, float inv_dx, int nx, int ny, int nz,
                                                              RigidMotion motion = RigidMotion{}) {
    const i64 p = (i64)blockIdx.x * PT + threadIdx.x;
    if (p >= n) return;
    float p0 = pos[3 * p], p1 = pos[3 * p + 1], p2 = pos[3 * p + 2];
    float v0 = vel[3 * p], v1 = vel[3 * p + 1], v2 = vel[3 * p + 2];
    obstacle_bc<MOVING>(p0, p1, p2, prev[3 * p], prev[3 * p + 1], prev[3 * p + 2], v0, v1, v2, obs, inv_dx, nx, ny, nz,
                        motion);
    pos[3 * p] = p0;
    pos[3 * p + 1] = p1;
    pos[3 * p + 2] = p2;
    vel[3 * p] = v0;
    vel[3 * p + 1] = v1;
    vel[3 * p + 2] = v2;
}

// Fused particle update for one step: G2P (solver.py:454-465), copy to previous positions
// (solver.py:469-474), advection (particles.cl:264-276), domain reflection (boundary_conditions.cl:
// 69-97) and obstacle push-out (boundary_conditions.cl:175-264), in the reference's order, with the
// particle records staged through shared memory by 16-byte loads and stores. The previous position
// lives in registers; it is written out only when the caller asks for it.
// The per-particle part of k_particle_update on registers (prev, when non-null, is this particle's
// previous-position record).
// The same with the grid velocity sampled by `sample` (g2p_velocity_with).
template <bool MOVING, class Sample>
__device__ __forceinline__ void particle_update_with(float& p0, float& p1, float& p2, float& v0, float& v1, float& v2,
                                                     float* __restrict__ prev, Sample&& sample,
                                                     const uint8_t* __restrict__ obs, float inv_dx, int nx, int ny,
                                                     int nz, float flip_ratio, float dt, float lower, float ux,
                                                     float uy, float uz, RigidMotion motion) {
    g2p_velocity_with(v0, v1, v2, sample, flip_ratio);
    const float q0 = p0, q1 = p1, q2 = p2;
    if (prev) {
        prev[0] = q0;
        prev[1] = q1;
        prev[2] = q2;
    }
    p0 = p0 + dt * v0;
    p1 = p1 + dt * v1;
    p2 = p2 + dt * v2;
    domain_bc_axis(p0, v0, lower, ux);
    domain_bc_axis(p1, v1, lower, uy);
    domain_bc_axis(p2, v2, lower, uz);
    if (obs) obstacle_bc<MOVING>(p0, p1, p2, q0, q1, q2, v0, v1, v2, obs, inv_dx, nx, ny, nz, motion);
}

template <bool MOVING = false>
__device__ __forceinline__ void particle_update_one(float& p0, float& p1, float& p2, float& v0, float& v1, float& v2,
                                                    float* __restrict__ prev, const float* u, const float* v,
                                                    const float* w, const float* ou, const float* ov, const float* ow,
                                                    const uint8_t* __restrict__ obs, float inv_dx, int nx, int ny,
                                                    int nz, float flip_ratio, float dt, float lower, float ux,
                                                    float uy, float uz, RigidMotion motion = RigidMotion{}) {
    g2p_velocity(v0, v1, v2, p0, p1, p2, u, v, w, ou, ov, ow, inv_dx, nx, ny, nz, flip_ratio);
    const float q0 = p0, q1 = p1, q2 = p2;
    if (prev) {
        prev[0] = q0;
        prev[1] = q1;
        prev[2] = q2;
    }
    p0 = p0 + dt * v0;
    p1 = p1 + dt * v1;
    p2 = p2 + dt * v2;
    domain_bc_axis(p0, v0, lower, ux);
    domain_bc_axis(p1, v1, lower, uy);
    domain_bc_axis(p2, v2, lower, uz);
    if (obs) obstacle_bc<MOVING>(p0, p1, p2, q0, q1, q2, v0, v1, v2, obs, inv_dx, nx, ny, nz, motion);
}

template <bool MOVING = false>
__global__ void __launch_bounds__(PT) k_particle_update(float* __restrict__ pos, float* __restrict__ vel,
                                                         float* __restrict__ prev_out, const float* u, const float* v,
                                                         const float* w, const float* ou, const float* ov,
                                                         const float* ow, const uint8_t* __restrict__ obs, i64 n,
                                                         float inv_dx, int nx, int ny, int nz, float flip_ratio,
                                                         float dt, float lower, float ux, float uy, float uz,
                                                         RigidMotion motion = RigidMotion{}) {
    __shared__ __align__(16) float sp[3 * PT];
    __shared__ __align__(16) float sv[3 * PT];
    const i64 first = (i64)blockIdx.x * PT;
    stage_particles(pos, first, n, sp);
    stage_particles(vel, first, n, sv);
    __syncthreads();
    const i64 p = first + threadIdx.x;
    if (p < n) {
        const int t = 3 * threadIdx.x;
        float p0 = sp[t], p1 = sp[t + 1], p2 = sp[t + 2];
        float v0 = sv[t], v1 = sv[t + 1], v2 = sv[t + 2];
        particle_update_one<MOVING>(p0, p1, p2, v0, v1, v2, prev_out ? prev_out + 3 * p : nullptr, u, v, w, ou, ov,
                                    ow, obs, inv_dx, nx, ny, nz, flip_ratio, dt, lower, ux, uy, uz, motion);
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

}  // namespace clb
