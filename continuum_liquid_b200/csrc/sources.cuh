// Particle sources on the device: the outflow removal and inflow top-up of source_particles.py:37-92
// (which the reference runs on the host with numpy between steps, after downloading every particle).
//
// Cells follow source_particles.py:21-25: clamp(floor(p / delta), 0, n - 1) per axis, the division in
// float32 as numpy evaluates a float32 array divided by a Python float. Outflow removal keeps the
// particles' order (a flag, a scan and a scatter: numpy's particles[keep]). An inflow tops every
// non-solid source cell up to its particle density; the new particles follow the cells in flat index
// order (numpy.argwhere) and each takes three consecutive doubles of the host's random stream
// (numpy.random.default_rng, a PCG64: 128-bit LCG, XSL-RR output), position = (cell + u) * delta in
// float64, stored as float32. The kernel reads the stream's state from the host and jumps to each
// particle's draws with Brown's arbitrary-stride LCG advance ("Random number generation with
// arbitrary strides", 1994); the host then advances its generator by the draws used, so the stream
// continues exactly as the host computation would.
#pragma once
#include "common.cuh"

namespace clb {

typedef unsigned __int128 u128;

constexpr u128 PCG_MULT = ((u128)0x2360ED051FC65DA4ull << 64) | (u128)0x4385DF649FCCF645ull;

__device__ __forceinline__ u128 pcg_advance(u128 state, u128 inc, unsigned long long delta) {
    u128 acc_mult = 1, acc_plus = 0, cur_mult = PCG_MULT, cur_plus = inc;
    while (delta) {
        if (delta & 1ull) {
            acc_mult *= cur_mult;
            acc_plus = acc_plus * cur_mult + cur_plus;
        }
        cur_plus = (cur_mult + 1) * cur_plus;
        cur_mult *= cur_mult;
        delta >>= 1;
    }
    return acc_mult * state + acc_plus;
}

// XSL-RR output of a state, as a double in [0, 1) the way numpy's Generator.random forms it
__device__ __forceinline__ double pcg_double(u128 state) {
    const unsigned rot = (unsigned)(state >> 122);
    const unsigned long long x = (unsigned long long)(state >> 64) ^ (unsigned long long)state;
    const unsigned long long r = (x >> rot) | (x << ((64u - rot) & 63u));
    return (double)(r >> 11) * (1.0 / 9007199254740992.0);
}

__device__ __forceinline__ int source_cell(float p, float delta, int n) {
    return clampi((int)floorf(p / delta), 0, n - 1);
}

__device__ __forceinline__ i64 particle_source_cell(const float* __restrict__ pos, i64 q, float delta, int nx, int ny,
                                                    int nz) {
    const int i = source_cell(__ldg(pos + 3 * q), delta, nx);
    const int j = source_cell(__ldg(pos + 3 * q + 1), delta, ny);
    const int k = source_cell(__ldg(pos + 3 * q + 2), delta, nz);
    return gidx(i, j, k, ny, nz);
}

// counts[cell] += particles in the cell
__global__ void __launch_bounds__(PT) k_source_cell_counts(const float* __restrict__ pos, i64 n, float delta, int nx,
                                                           int ny, int nz, int* __restrict__ counts) {
    const i64 q = (i64)blockIdx.x * PT + threadIdx.x;
    if (q < n) atomicAdd(counts + particle_source_cell(pos, q, delta, nx, ny, nz), 1);
}

// keep[q] = 1 unless the particle's cell is in the (combined) outflow mask
__global__ void __launch_bounds__(PT) k_source_keep(const float* __restrict__ pos, i64 n, float delta, int nx, int ny,
                                                    int nz, const uint8_t* __restrict__ outflow, int* __restrict__ keep) {
    const i64 q = (i64)blockIdx.x * PT + threadIdx.x;
    if (q < n) keep[q] = __ldg(outflow + particle_source_cell(pos, q, delta, nx, ny, nz)) ? 0 : 1;
}

// kept particles to their scanned slots (input order preserved)
__global__ void __launch_bounds__(PT) k_source_compact(const float* __restrict__ pos, const float* __restrict__ vel,
                                                       const int* __restrict__ keep, const int* __restrict__ slot, i64 n,
                                                       float* __restrict__ pos_out, float* __restrict__ vel_out) {
    const i64 q = (i64)blockIdx.x * PT + threadIdx.x;
    if (q >= n || !keep[q]) return;
    const i64 d = 3 * (i64)slot[q], s = 3 * q;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        pos_out[d + a] = __ldg(pos + s + a);
        vel_out[d + a] = __ldg(vel + s + a);
    }
}

// missing[c] = max(0, target - counts[c]) in non-solid source cells, 0 elsewhere
__global__ void __launch_bounds__(PT) k_source_missing(const int* __restrict__ counts, const uint8_t* __restrict__ source,
                                                       const uint8_t* __restrict__ solid, int target, i64 cells,
                                                       int* __restrict__ missing) {
    const i64 c = (i64)blockIdx.x * PT + threadIdx.x;
    if (c >= cells) return;
    const bool on = __ldg(source + c) && !(solid && __ldg(solid + c));
    missing[c] = on ? max(0, target - __ldg(counts + c)) : 0;
}

// new particles of every cell: particle g (cell order, offsets[c] + t) takes draws 3g .. 3g + 2 after
// the stream state (state, inc); pos_out/vel_out point at the first new record
__global__ void __launch_bounds__(PT) k_source_spawn(const int* __restrict__ missing, const int* __restrict__ offsets,
                                                     i64 cells, int ny, int nz, double delta, float vx, float vy,
                                                     float vz, unsigned long long state_hi,
                                                     unsigned long long state_lo, unsigned long long inc_hi,
                                                     unsigned long long inc_lo, float* __restrict__ pos_out,
                                                     float* __restrict__ vel_out) {
    const i64 c = (i64)blockIdx.x * PT + threadIdx.x;
    if (c >= cells) return;
    const int m = __ldg(missing + c);
    if (m <= 0) return;
    int i, j, k;
    gcoord(c, ny, nz, i, j, k);
    const u128 state0 = ((u128)state_hi << 64) | (u128)state_lo;
    const u128 inc = ((u128)inc_hi << 64) | (u128)inc_lo;
    const int first = __ldg(offsets + c);
    u128 st = pcg_advance(state0, inc, 3ull * (unsigned long long)first);
    for (int t = 0; t < m; ++t) {
        const i64 g = (i64)first + t;
        st = st * PCG_MULT + inc;
        const double u0 = pcg_double(st);
        st = st * PCG_MULT + inc;
        const double u1 = pcg_double(st);
        st = st * PCG_MULT + inc;
        const double u2 = pcg_double(st);
        pos_out[3 * g] = (float)(((double)i + u0) * delta);
        pos_out[3 * g + 1] = (float)(((double)j + u1) * delta);
        pos_out[3 * g + 2] = (float)(((double)k + u2) * delta);
        vel_out[3 * g] = vx;
        vel_out[3 * g + 1] = vy;
        vel_out[3 * g + 2] = vz;
    }
}

}  // namespace clb
