// Moving colliders (no counterpart in the reference, which voxelises its colliders once and keeps
// them at rest: boundary_conditions.cl:99-264 sets solid faces and solid velocities to 0).
//
// One rigid motion per scene: velocity V, angular velocity W (rad/s) and the pivot C at the step's
// time, in grid-local coordinates. The solid's velocity at x is V + W x (x - C). With it:
//  * grid_obstacle_bc: a solid face takes the solid's velocity component at the face centre (the u
//    face of cell (i, j, k) sits at ((i+1) dx, (j+0.5) dx, (k+0.5) dx)) instead of 0;
//  * extrapolate_obstacle_velocity: a solid cell next to fluid keeps the fluid's averaged tangential
//    velocity and takes the solid's normal component at its face centre;
//  * particle_obstacle_bc: the same normal and push-out, but only the velocity relative to the solid
//    at the particle's position loses its inward normal component.
// At rest (V = W = 0) these give the reference's values.
#pragma once
#include "common.cuh"

namespace clb {

struct RigidMotion {
    float vx, vy, vz, wx, wy, wz, cx, cy, cz;
};

// V + W x (x - C), evaluated in this order
__device__ __forceinline__ void rigid_velocity(const RigidMotion& m, float x, float y, float z, float& a, float& b,
                                               float& c) {
    const float rx = x - m.cx, ry = y - m.cy, rz = z - m.cz;
    a = m.vx + (m.wy * rz - m.wz * ry);
    b = m.vy + (m.wz * rx - m.wx * rz);
    c = m.vz + (m.wx * ry - m.wy * rx);
}

__global__ void __launch_bounds__(256) k_grid_obstacle_bc_moving(float* __restrict__ u, float* __restrict__ v,
                                                                  float* __restrict__ w, float* __restrict__ ff,
                                                                  const uint8_t* __restrict__ obs, int nx, int ny,
                                                                  int nz, RigidMotion m, float dx) {
    const i64 C = (i64)nx * ny * nz;
    const i64 c = (i64)blockIdx.x * 256 + threadIdx.x;
    if (c >= C) return;
    int i, j, k;
    gcoord(c, ny, nz, i, j, k);
    const bool self = __ldg(obs + c) != 0;
    if (self) ff[c] = 0.0f;
    const bool xs = self || (i + 1 < nx && __ldg(obs + c + (i64)ny * nz));
    const bool ys = self || (j + 1 < ny && __ldg(obs + c + nz));
    const bool zs = self || (k + 1 < nz && __ldg(obs + c + 1));
    const float fi = (float)i, fj = (float)j, fk = (float)k;
    float a, b, e;
    if (xs) {
        rigid_velocity(m, (fi + 1.0f) * dx, (fj + 0.5f) * dx, (fk + 0.5f) * dx, a, b, e);
        u[c] = a;
    }
    if (ys) {
        rigid_velocity(m, (fi + 0.5f) * dx, (fj + 1.0f) * dx, (fk + 0.5f) * dx, a, b, e);
        v[c] = b;
    }
    if (zs) {
        rigid_velocity(m, (fi + 0.5f) * dx, (fj + 0.5f) * dx, (fk + 1.0f) * dx, a, b, e);
        w[c] = e;
    }
}

// reads non-obstacle cells and writes obstacle cells only: one launch has no read/write overlap
__global__ void __launch_bounds__(256) k_extrapolate_obstacle_velocity_moving(float* u, float* v, float* w,
                                                                               const uint8_t* __restrict__ obs,
                                                                               int nx, int ny, int nz, RigidMotion m,
                                                                               float dx) {
    const i64 C = (i64)nx * ny * nz;
    const i64 c = (i64)blockIdx.x * 256 + threadIdx.x;
    if (c >= C || !__ldg(obs + c)) return;
    int i, j, k;
    gcoord(c, ny, nz, i, j, k);
    float t0 = 0.0f, t1 = 0.0f, t2 = 0.0f;
    int n = 0, ax = 0, ay = 0, az = 0;
    const i64 sx = (i64)ny * nz, sy = nz;
    auto acc = [&](i64 q, int& axis) {
        if (!__ldg(obs + q)) {
            t0 += u[q];
            t1 += v[q];
            t2 += w[q];
            n += 1;
            axis = 1;
        }
    };
    if (i > 0) acc(c - sx, ax);
    if (i + 1 < nx) acc(c + sx, ax);
    if (j > 0) acc(c - sy, ay);
    if (j + 1 < ny) acc(c + sy, ay);
    if (k > 0) acc(c - 1, az);
    if (k + 1 < nz) acc(c + 1, az);
    if (n == 0) return;
    const float fn = (float)n;
    t0 = t0 / fn;
    t1 = t1 / fn;
    t2 = t2 / fn;
    const float fi = (float)i, fj = (float)j, fk = (float)k;
    float a, b, e;
    if (ax) rigid_velocity(m, (fi + 1.0f) * dx, (fj + 0.5f) * dx, (fk + 0.5f) * dx, a, b, e);
    u[c] = ax ? a : t0;
    if (ay) rigid_velocity(m, (fi + 0.5f) * dx, (fj + 1.0f) * dx, (fk + 0.5f) * dx, a, b, e);
    v[c] = ay ? b : t1;
    if (az) rigid_velocity(m, (fi + 0.5f) * dx, (fj + 0.5f) * dx, (fk + 1.0f) * dx, a, b, e);
    w[c] = az ? e : t2;
}

}  // namespace clb
