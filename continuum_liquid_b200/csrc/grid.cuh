// Cell-wide kernels: forces/viscosity, MAC boundary conditions, pressure right-hand side and
// projection (Solver/Kernel/OpenCL/velocity_update.cl, boundary_conditions.cl, pressure_solve.cl).
#pragma once
#include "common.cuh"

namespace clb {

constexpr int GT = 256;  // threads per block for cell-wide kernels

// helper.cl:54-66 laplacian
__device__ __forceinline__ float laplacian(const float* __restrict__ f, i64 c, i64 sx, i64 sy, float inv_dx2) {
    const float center = __ldg(f + c);
    const float s = __ldg(f + c + sx) + __ldg(f + c - sx) + __ldg(f + c + sy) + __ldg(f + c - sy) + __ldg(f + c + 1) +
                    __ldg(f + c - 1);
    return (s - 6.0f * center) * inv_dx2;
}

// velocity_update.cl:3-43 update_velocity
__device__ __forceinline__ void update_velocity_at(i64 c, const float* __restrict__ u, const float* __restrict__ v,
                                                         const float* __restrict__ w, float* __restrict__ ru,
                                                         float* __restrict__ rv, float* __restrict__ rw,
                                                         const float* __restrict__ ff, float gx, float gy, float gz,
                                                         float fx, float fy, float fz, float rho, float nu,
                                                         float inv_dx2, float dt, int nx, int ny, int nz) {
    int i, j, k;
    gcoord(c, ny, nz, i, j, k);
    float r0 = __ldg(u + c), r1 = __ldg(v + c), r2 = __ldg(w + c);
    if (__ldg(ff + c) > 0.0f) {
        r0 += dt * (gx + fx / rho);
        r1 += dt * (gy + fy / rho);
        r2 += dt * (gz + fz / rho);
    }
    if (interior(i, j, k, nx, ny, nz)) {
        const i64 sx = (i64)ny * nz, sy = nz;
        r0 += nu * dt * laplacian(u, c, sx, sy, inv_dx2);
        r1 += nu * dt * laplacian(v, c, sx, sy, inv_dx2);
        r2 += nu * dt * laplacian(w, c, sx, sy, inv_dx2);
    }
    ru[c] = r0;
    rv[c] = r1;
    rw[c] = r2;
}

__global__ void __launch_bounds__(GT) k_update_velocity(const float* __restrict__ u, const float* __restrict__ v,
                                                         const float* __restrict__ w, float* __restrict__ ru,
                                                         float* __restrict__ rv, float* __restrict__ rw,
                                                         const float* __restrict__ ff, float gx, float gy, float gz,
                                                         float fx, float fy, float fz, float rho, float nu,
                                                         float inv_dx2, float dt, int nx, int ny, int nz) {
    const i64 C = (i64)nx * ny * nz;
    const i64 c = (i64)blockIdx.x * GT + threadIdx.x;
    if (c >= C) return;
    update_velocity_at(c, u, v, w, ru, rv, rw, ff, gx, gy, gz, fx, fy, fz, rho, nu, inv_dx2, dt, nx, ny, nz);
}

// boundary_conditions.cl:33-67 grid_domain_bc. A ghost copies a component from its clamped
// interior cell only where the ghost's own wall flag for that component is clear, and the interior
// source shares that flag, so the source component is never written by the same launch.
__device__ __forceinline__ void grid_domain_bc_at(i64 c, float* u, float* v, float* w, int nx, int ny, int nz) {
    int i, j, k;
    gcoord(c, ny, nz, i, j, k);
    const bool ghost = !interior(i, j, k, nx, ny, nz);
    const bool wu = i == 0 || i >= nx - 2, wv = j == 0 || j >= ny - 2, ww = k == 0 || k >= nz - 2;
    if (!ghost && !wu && !wv && !ww) return;
    if (ghost) {
        const i64 s = gidx(clampi(i, 1, nx - 2), clampi(j, 1, ny - 2), clampi(k, 1, nz - 2), ny, nz);
        u[c] = wu ? 0.0f : u[s];
        v[c] = wv ? 0.0f : v[s];
        w[c] = ww ? 0.0f : w[s];
        return;
    }
    if (wu) u[c] = 0.0f;
    if (wv) v[c] = 0.0f;
    if (ww) w[c] = 0.0f;
}

__global__ void __launch_bounds__(GT) k_grid_domain_bc(float* u, float* v, float* w, int nx, int ny, int nz) {
    const i64 C = (i64)nx * ny * nz;
    const i64 c = (i64)blockIdx.x * GT + threadIdx.x;
    if (c >= C) return;
    grid_domain_bc_at(c, u, v, w, nx, ny, nz);
}

// The shell of a grid: the cells within `lo` planes of a low face or `hi` planes of a high face on
// some axis, counted without repeats (needs every extent >= lo + hi). The domain boundary conditions
// change only such cells (grid_domain_bc: lo 1, hi 2; neumann_domain_bc: lo 1, hi 1), and since
// their writes never feed their own reads, a launch over the shell alone leaves the same values as
// one over the whole grid for a few percent of the threads.
__host__ __device__ __forceinline__ i64 shell_cells(int nx, int ny, int nz, int lo, int hi) {
    const i64 w = lo + hi;
    return w * ny * nz + (nx - w) * w * nz + (nx - w) * (ny - w) * w;
}

// Shell cell t (< shell_cells): the lo + hi face planes of x, then the face rows of y in the other
// planes, then the face cells of z in the other rows.
__device__ __forceinline__ i64 shell_cell(i64 t, int nx, int ny, int nz, int lo, int hi) {
    const int w = lo + hi;
    auto side = [&](int q, int n) { return q < lo ? q : n - hi + (q - lo); };
    const i64 a = (i64)w * ny * nz;
    if (t < a) {
        const i64 plane = (i64)ny * nz;
        const int p = (int)(t / plane), r = (int)(t - p * plane);
        return gidx(side(p, nx), r / nz, r % nz, ny, nz);
    }
    t -= a;
    const i64 b = (i64)(nx - w) * w * nz;
    if (t < b) {
        const i64 slab = (i64)w * nz;
        const int p = (int)(t / slab), r = (int)(t - p * slab);
        return gidx(lo + p, side(r / nz, ny), r % nz, ny, nz);
    }
    t -= b;
    const i64 rows = (i64)(ny - w) * w;
    const int p = (int)(t / rows), r = (int)(t - p * rows);
    return gidx(lo + p, lo + r / w, side(r % w, nz), ny, nz);
}

__global__ void __launch_bounds__(GT) k_grid_domain_bc_shell(float* u, float* v, float* w, int nx, int ny, int nz) {
    const i64 t = (i64)blockIdx.x * GT + threadIdx.x;
    if (t >= shell_cells(nx, ny, nz, 1, 2)) return;
    grid_domain_bc_at(shell_cell(t, nx, ny, nz, 1, 2), u, v, w, nx, ny, nz);
}

// boundary_conditions.cl:99-119 grid_obstacle_bc
__device__ __forceinline__ void grid_obstacle_bc_at(i64 c, float* __restrict__ u, float* __restrict__ v,
                                                          float* __restrict__ w, float* __restrict__ ff,
                                                          const uint8_t* __restrict__ obs, int nx, int ny, int nz) {
    int i, j, k;
    gcoord(c, ny, nz, i, j, k);
    const bool self = __ldg(obs + c) != 0;
    if (self) ff[c] = 0.0f;
    const bool xs = self || (i + 1 < nx && __ldg(obs + c + (i64)ny * nz));
    const bool ys = self || (j + 1 < ny && __ldg(obs + c + nz));
    const bool zs = self || (k + 1 < nz && __ldg(obs + c + 1));
    if (xs) u[c] = 0.0f;
    if (ys) v[c] = 0.0f;
    if (zs) w[c] = 0.0f;
}

__global__ void __launch_bounds__(GT) k_grid_obstacle_bc(float* __restrict__ u, float* __restrict__ v,
                                                          float* __restrict__ w, float* __restrict__ ff,
                                                          const uint8_t* __restrict__ obs, int nx, int ny, int nz) {
    const i64 C = (i64)nx * ny * nz;
    const i64 c = (i64)blockIdx.x * GT + threadIdx.x;
    if (c >= C) return;
    grid_obstacle_bc_at(c, u, v, w, ff, obs, nx, ny, nz);
}

// boundary_conditions.cl:121-173 extrapolate_obstacle_velocity (reads non-obstacle cells only and
// writes obstacle cells only, so one launch has no read/write overlap).
__device__ __forceinline__ void extrapolate_obstacle_velocity_at(i64 c, float* u, float* v, float* w,
                                                                 const uint8_t* __restrict__ obs, int nx, int ny,
                                                                 int nz) {
    if (!__ldg(obs + c)) return;
    int i, j, k;
    gcoord(c, ny, nz, i, j, k);
    float t0 = 0.0f, t1 = 0.0f, t2 = 0.0f;
    int n = 0, ax = 0, ay = 0, az = 0;
    const i64 sx = (i64)ny * nz, sy = nz;
#define CLB_ACC(q, axis)          \
    if (!__ldg(obs + (q))) {      \
        t0 += u[q];               \
        t1 += v[q];               \
        t2 += w[q];               \
        n += 1;                   \
        axis = 1;                 \
    }
    if (i > 0) CLB_ACC(c - sx, ax);
    if (i + 1 < nx) CLB_ACC(c + sx, ax);
    if (j > 0) CLB_ACC(c - sy, ay);
    if (j + 1 < ny) CLB_ACC(c + sy, ay);
    if (k > 0) CLB_ACC(c - 1, az);
    if (k + 1 < nz) CLB_ACC(c + 1, az);
#undef CLB_ACC
    if (n == 0) return;
    const float fn = (float)n;
    t0 = t0 / fn;
    t1 = t1 / fn;
    t2 = t2 / fn;
    u[c] = ax ? 0.0f : t0;
    v[c] = ay ? 0.0f : t1;
    w[c] = az ? 0.0f : t2;
}

__global__ void __launch_bounds__(GT) k_extrapolate_obstacle_velocity(float* u, float* v, float* w,
                                                                       const uint8_t* __restrict__ obs, int nx, int ny,
                                                                       int nz) {
    const i64 C = (i64)nx * ny * nz;
    const i64 c = (i64)blockIdx.x * GT + threadIdx.x;
    if (c >= C) return;
    extrapolate_obstacle_velocity_at(c, u, v, w, obs, nx, ny, nz);
}

// pressure_solve.cl:3-24 pressure_rhs (helper.cl:39-52 divergence)
__device__ __forceinline__ float rhs_at(const float* __restrict__ u, const float* __restrict__ v,
                                        const float* __restrict__ w, i64 c, i64 sx, i64 sy, float rho_over_dt,
                                        float inv_dx) {
    const float du = __ldg(u + c) - __ldg(u + c - sx);
    const float dv = __ldg(v + c) - __ldg(v + c - sy);
    const float dw = __ldg(w + c) - __ldg(w + c - 1);
    return rho_over_dt * ((du + dv + dw) * inv_dx);
}

__global__ void __launch_bounds__(GT) k_pressure_rhs(const float* __restrict__ u, const float* __restrict__ v,
                                                      const float* __restrict__ w, const float* __restrict__ ff,
                                                      float* __restrict__ rhs, float rho_over_dt, float inv_dx, int nx,
                                                      int ny, int nz) {
    const i64 C = (i64)nx * ny * nz;
    const i64 c = (i64)blockIdx.x * GT + threadIdx.x;
    if (c >= C) return;
    int i, j, k;
    gcoord(c, ny, nz, i, j, k);
    if (!interior(i, j, k, nx, ny, nz) || __ldg(ff + c) <= 0.0f) {
        rhs[c] = 0.0f;
        return;
    }
    rhs[c] = rhs_at(u, v, w, c, (i64)ny * nz, nz, rho_over_dt, inv_dx);
}

// pressure_solve.cl:26-47 pressure_correction (helper.cl:25-37 gradient). PT = float is the
// reference's arithmetic; PT = double takes the gradient of an FP64 pressure in FP64 and rounds the
// updated velocity once (the projection of a refined solve, whose FP64 pressure is the one that
// meets the residual tolerance).
template <typename PT>
__device__ __forceinline__ void pressure_correction_at(i64 c, float* __restrict__ u, float* __restrict__ v,
                                                             float* __restrict__ w, const PT* __restrict__ p,
                                                             float dt_over_rho, float inv_dx, int nx, int ny, int nz) {
    int i, j, k;
    gcoord(c, ny, nz, i, j, k);
    if (!interior(i, j, k, nx, ny, nz)) return;
    const PT center = __ldg(p + c);
    const PT gx = (__ldg(p + c + (i64)ny * nz) - center) * (PT)inv_dx;
    const PT gy = (__ldg(p + c + nz) - center) * (PT)inv_dx;
    const PT gz = (__ldg(p + c + 1) - center) * (PT)inv_dx;
    u[c] = (float)((PT)u[c] - (PT)dt_over_rho * gx);
    v[c] = (float)((PT)v[c] - (PT)dt_over_rho * gy);
    w[c] = (float)((PT)w[c] - (PT)dt_over_rho * gz);
}

template <typename PT>
__global__ void __launch_bounds__(GT) k_pressure_correction(float* __restrict__ u, float* __restrict__ v,
                                                             float* __restrict__ w, const PT* __restrict__ p,
                                                             float dt_over_rho, float inv_dx, int nx, int ny, int nz) {
    pdl_begin();
    const i64 C = (i64)nx * ny * nz;
    const i64 c = (i64)blockIdx.x * GT + threadIdx.x;
    if (c >= C) return;
    pressure_correction_at<PT>(c, u, v, w, p, dt_over_rho, inv_dx, nx, ny, nz);
}

// boundary_conditions.cl:18-31 neumann_domain_bc (ghosts read interior cells only)
template <typename PT>
__device__ __forceinline__ void neumann_domain_bc_at(i64 c, PT* p, int nx, int ny, int nz) {
    int i, j, k;
    gcoord(c, ny, nz, i, j, k);
    if (interior(i, j, k, nx, ny, nz)) return;
    p[c] = p[gidx(clampi(i, 1, nx - 2), clampi(j, 1, ny - 2), clampi(k, 1, nz - 2), ny, nz)];
}

template <typename PT>
__global__ void __launch_bounds__(GT) k_neumann_domain_bc(PT* p, int nx, int ny, int nz) {
    pdl_begin();
    const i64 C = (i64)nx * ny * nz;
    const i64 c = (i64)blockIdx.x * GT + threadIdx.x;
    if (c >= C) return;
    neumann_domain_bc_at<PT>(c, p, nx, ny, nz);
}

// The same over the grid's shell of non-interior cells only (shell_cells with lo = hi = 1).
template <typename PT>
__global__ void __launch_bounds__(GT) k_neumann_domain_bc_shell(PT* p, int nx, int ny, int nz) {
    pdl_begin();
    const i64 t = (i64)blockIdx.x * GT + threadIdx.x;
    if (t >= shell_cells(nx, ny, nz, 1, 1)) return;
    neumann_domain_bc_at<PT>(shell_cell(t, nx, ny, nz, 1, 1), p, nx, ny, nz);
}

}  // namespace clb
