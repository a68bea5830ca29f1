// Multigrid pressure Poisson solve (Solver/Kernel/OpenCL/multigrid.cl, Solver/Kernel/multigrid.py,
// Solver/Kernel/pressure_solve.py).
//
// Two storage layouts are served:
//  * the reference layout (separate float32 mask/diag/wx/wy/wz arrays per level), one kernel per
//    reference kernel, used by the stage API for per-kernel parity;
//  * the product layout: level 0 keeps its operator in one byte per cell (diag 0..6 in bits 0-2,
//    wx/wy/wz in bits 3-5, fluid flag in bit 6 -- on the finest level diag is a small integer and
//    the weights are 0/1, multigrid.cl:63-88), coarse levels keep (diag, wx, wy, wz) as one float4
//    plus a one-byte mask. The Galerkin coarse operators depend only on the masks, so they are built
//    once per solve instead of on every restriction (multigrid.cl:127-179 recomputes them on every
//    visit; the values are the same).
// The arithmetic of every update keeps the reference's evaluation order, so both layouts give the
// same values as the CPU restatement.
#pragma once
#include "common.cuh"
#include <cuda_fp16.h>

namespace clb {

constexpr int MGT = 256;
constexpr int MG_MAX_LEVELS = 16;

// ------------------------------------------------------------------------------------------------
// The reference's level arrays (float32 mask, diagonal, weight_x, weight_y, weight_z per level,
// multigrid.py:18-50) converted to and from the product's level formats, so that the stage functions
// that take the reference's arrays (multigrid.w_cycle, smooth, coarse_smooth, pressure_solve) run the
// product kernels: the finest level packed into one byte per cell, a coarse level into a float4
// (diagonal, wx, wy, wz) plus a mask byte. A cell is fluid where its mask is > 0, as the reference
// tests it (multigrid.cl:38, 220, 251).
// ------------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(MGT) k_pack_finest(const float* __restrict__ mask, const float* __restrict__ diag,
                                                      const float* __restrict__ wx, const float* __restrict__ wy,
                                                      const float* __restrict__ wz, uint8_t* __restrict__ op0,
                                                      int* __restrict__ invalid, i64 C) {
    const i64 c = (i64)blockIdx.x * MGT + threadIdx.x;
    if (c >= C) return;
    const float d = __ldg(diag + c), x = __ldg(wx + c), y = __ldg(wy + c), z = __ldg(wz + c);
    // the byte holds a diagonal 0..7 and 0/1 weights, which is what build_finest_operator produces
    const bool ok = d >= 0.0f && d <= 7.0f && d == floorf(d) && (x == 0.0f || x == 1.0f) &&
                    (y == 0.0f || y == 1.0f) && (z == 0.0f || z == 1.0f);
    if (!ok) atomicAdd(invalid, 1);
    op0[c] = (uint8_t)(((uint32_t)d & 7u) | ((uint32_t)(x == 1.0f) << 3) | ((uint32_t)(y == 1.0f) << 4) |
                       ((uint32_t)(z == 1.0f) << 5) | ((uint32_t)(__ldg(mask + c) > 0.0f) << 6));
}

__global__ void __launch_bounds__(MGT) k_unpack_finest(const uint8_t* __restrict__ op0, float* __restrict__ diag,
                                                        float* __restrict__ wx, float* __restrict__ wy,
                                                        float* __restrict__ wz, i64 C) {
    const i64 c = (i64)blockIdx.x * MGT + threadIdx.x;
    if (c >= C) return;
    const uint32_t o = __ldg(op0 + c);
    diag[c] = (float)(o & 7u);
    wx[c] = (float)((o >> 3) & 1u);
    wy[c] = (float)((o >> 4) & 1u);
    wz[c] = (float)((o >> 5) & 1u);
}

__global__ void __launch_bounds__(MGT) k_pack_level(const float* __restrict__ mask, const float* __restrict__ diag,
                                                     const float* __restrict__ wx, const float* __restrict__ wy,
                                                     const float* __restrict__ wz, float4* __restrict__ op,
                                                     uint8_t* __restrict__ mask_out, i64 C) {
    const i64 c = (i64)blockIdx.x * MGT + threadIdx.x;
    if (c >= C) return;
    op[c] = make_float4(__ldg(diag + c), __ldg(wx + c), __ldg(wy + c), __ldg(wz + c));
    mask_out[c] = __ldg(mask + c) > 0.0f ? 1 : 0;
}

__global__ void __launch_bounds__(MGT) k_unpack_level(const float4* __restrict__ op, const uint8_t* __restrict__ m,
                                                       float* __restrict__ mask, float* __restrict__ diag,
                                                       float* __restrict__ wx, float* __restrict__ wy,
                                                       float* __restrict__ wz, i64 C) {
    const i64 c = (i64)blockIdx.x * MGT + threadIdx.x;
    if (c >= C) return;
    const float4 o = __ldg(op + c);
    mask[c] = __ldg(m + c) ? 1.0f : 0.0f;
    diag[c] = o.x;
    wx[c] = o.y;
    wy[c] = o.z;
    wz[c] = o.w;
}

// ------------------------------------------------------------------------------------------------
// Product layout
// ------------------------------------------------------------------------------------------------
struct Op0 {  // finest level: packed byte per cell
    const uint8_t* __restrict__ op;
    __device__ __forceinline__ uint32_t at(i64 c) const { return __ldg(op + c); }
    __device__ __forceinline__ bool fluid(i64 c) const { return (at(c) & 64u) != 0u; }
};
struct OpC {  // coarse levels: float4 (diag, wx, wy, wz) + mask byte
    const float4* __restrict__ op;
    const uint8_t* __restrict__ mask;
    __device__ __forceinline__ bool fluid(i64 c) const { return __ldg(mask + c) != 0; }
};

__device__ __forceinline__ float bitf(uint32_t v, int bit) { return (float)((v >> bit) & 1u); }

// FP16 storage of coarse levels (no counterpart in the reference): p and b as __half, the operator
// as four __half (diag, wx, wy, wz) in 8 bytes. Values on FP16 levels are scaled (see mg_half.cuh);
// all arithmetic stays FP32.
struct __align__(8) Half4 {
    __half x, y, z, w;
};
__device__ __forceinline__ float4 ld_h4(const Half4* __restrict__ op, i64 c) {
    const uint2 u = __ldg(reinterpret_cast<const uint2*>(op) + c);
    const __half2 a = *reinterpret_cast<const __half2*>(&u.x), b = *reinterpret_cast<const __half2*>(&u.y);
    return make_float4(__low2float(a), __high2float(a), __low2float(b), __high2float(b));
}
__device__ __forceinline__ float ldh(const __half* p, i64 c) { return __half2float(p[c]); }
__device__ __forceinline__ Half4 to_h4(float4 v) {
    Half4 h;
    h.x = __float2half_rn(v.x);
    h.y = __float2half_rn(v.y);
    h.z = __float2half_rn(v.z);
    h.w = __float2half_rn(v.w);
    return h;
}

// Weighted neighbour sum (multigrid.cl:7-23) for each layout, same term order.
template <typename T>
__device__ __forceinline__ T wsum0(const uint8_t* __restrict__ op, const T* p, i64 c, i64 sx, i64 sy, uint32_t self) {
    const uint32_t ox = __ldg(op + c - sx), oy = __ldg(op + c - sy), oz = __ldg(op + c - 1);
    return (T)bitf(self, 3) * p[c + sx] + (T)bitf(ox, 3) * p[c - sx] + (T)bitf(self, 4) * p[c + sy] +
           (T)bitf(oy, 4) * p[c - sy] + (T)bitf(self, 5) * p[c + 1] + (T)bitf(oz, 5) * p[c - 1];
}
__device__ __forceinline__ float wsumC(const float4* __restrict__ op, const float* p, i64 c, i64 sx, i64 sy,
                                       float4 self) {
    return self.y * p[c + sx] + __ldg(op + c - sx).y * p[c - sx] + self.z * p[c + sy] + __ldg(op + c - sy).z * p[c - sy] +
           self.w * p[c + 1] + __ldg(op + c - 1).w * p[c - 1];
}

// Fused pressure_rhs (pressure_solve.cl:3-24) + build_finest_operator (multigrid.cl:63-88) into the
// packed layout. mask is the fluid fraction, as in pressure_solve.py:299-308.
__device__ __forceinline__ void rhs_op0_at(i64 c, const float* __restrict__ u, const float* __restrict__ v,
                                                  const float* __restrict__ w, const float* __restrict__ ff,
                                                  float* __restrict__ rhs, uint8_t* __restrict__ op0,
                                                  float rho_over_dt, float inv_dx, int nx, int ny, int nz) {
    int i, j, k;
    gcoord(c, ny, nz, i, j, k);
    const i64 sx = (i64)ny * nz, sy = nz;
    if (!interior(i, j, k, nx, ny, nz) || __ldg(ff + c) <= 0.0f) {
        rhs[c] = 0.0f;
        op0[c] = 0;
        return;
    }
    const float du = __ldg(u + c) - __ldg(u + c - sx);
    const float dv = __ldg(v + c) - __ldg(v + c - sy);
    const float dw = __ldg(w + c) - __ldg(w + c - 1);
    rhs[c] = rho_over_dt * ((du + dv + dw) * inv_dx);
    uint32_t d = 6u - (i == 1) - (i == nx - 2) - (j == 1) - (j == ny - 2) - (k == 1) - (k == nz - 2);
    uint32_t bits = d | 64u;
    if (i < nx - 2 && __ldg(ff + c + sx) > 0.0f) bits |= 8u;
    if (j < ny - 2 && __ldg(ff + c + sy) > 0.0f) bits |= 16u;
    if (k < nz - 2 && __ldg(ff + c + 1) > 0.0f) bits |= 32u;
    op0[c] = (uint8_t)bits;
}

__global__ void __launch_bounds__(MGT) k_rhs_op0(const float* __restrict__ u, const float* __restrict__ v,
                                                  const float* __restrict__ w, const float* __restrict__ ff,
                                                  float* __restrict__ rhs, uint8_t* __restrict__ op0,
                                                  float rho_over_dt, float inv_dx, int nx, int ny, int nz) {
    pdl_begin();
    const i64 C = (i64)nx * ny * nz;
    const i64 c = (i64)blockIdx.x * MGT + threadIdx.x;
    if (c >= C) return;
    rhs_op0_at(c, u, v, w, ff, rhs, op0, rho_over_dt, inv_dx, nx, ny, nz);
}

// Operator part of restrict_residual (multigrid.cl:127-179) for one coarse level, from any layout:
// FS = 0 packed finest level, 1 float4 coarse level, 2 FP16 coarse level. CH = true stores the
// coarse operator in FP16 and counts entries that FP16 does not hold exactly into *inexact (the
// entries are sums of small integers, exact below 2048).
template <int FS, bool CH>
__device__ __forceinline__ void coarse_operator_at(i64 ci, const uint8_t* __restrict__ fop0,
                                                          const void* __restrict__ fopc_,
                                                          const uint8_t* __restrict__ fmask, void* __restrict__ cop_,
                                                          uint8_t* __restrict__ cmask, int* __restrict__ inexact,
                                                          int fnx, int fny, int fnz, int cnx, int cny, int cnz) {
    constexpr bool FINE0 = FS == 0;
    const float4* __restrict__ fopc = reinterpret_cast<const float4*>(fopc_);
    int I, J, K;
    gcoord(ci, cny, cnz, I, J, K);
    float dsum = 0.0f, cx = 0.0f, cy = 0.0f, cz = 0.0f;
    int active = 0;
    if (interior(I, J, K, cnx, cny, cnz)) {
        const int si = 1 + 2 * (I - 1), sj = 1 + 2 * (J - 1), sk = 1 + 2 * (K - 1);
        for (int di = 0; di < 2; ++di)
            for (int dj = 0; dj < 2; ++dj)
                for (int dk = 0; dk < 2; ++dk) {
                    const int i = si + di, j = sj + dj, k = sk + dk;
                    if (!interior(i, j, k, fnx, fny, fnz)) continue;
                    const i64 f = gidx(i, j, k, fny, fnz);
                    float d, wx, wy, wz;
                    if (FINE0) {
                        const uint32_t o = __ldg(fop0 + f);
                        if (!(o & 64u)) continue;
                        d = (float)(o & 7u);
                        wx = bitf(o, 3);
                        wy = bitf(o, 4);
                        wz = bitf(o, 5);
                    } else {
                        if (!__ldg(fmask + f)) continue;
                        const float4 o = FS == 2 ? ld_h4(reinterpret_cast<const Half4*>(fopc_), f) : __ldg(fopc + f);
                        d = o.x;
                        wx = o.y;
                        wy = o.z;
                        wz = o.w;
                    }
                    ++active;
                    dsum += d;
                    if (wx > 0.0f) {
                        if (di == 0) dsum -= 2.0f * wx;
                        else cx += wx;
                    }
                    if (wy > 0.0f) {
                        if (dj == 0) dsum -= 2.0f * wy;
                        else cy += wy;
                    }
                    if (wz > 0.0f) {
                        if (dk == 0) dsum -= 2.0f * wz;
                        else cz += wz;
                    }
                }
    }
    const float4 v = active > 0 ? make_float4(dsum, cx, cy, cz) : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    cmask[ci] = active > 0 ? 1 : 0;
    if (CH) {
        const Half4 h = to_h4(v);
        if (__half2float(h.x) != v.x || __half2float(h.y) != v.y || __half2float(h.z) != v.z ||
            __half2float(h.w) != v.w)
            atomicAdd(inexact, 1);
        reinterpret_cast<Half4*>(cop_)[ci] = h;
    } else {
        reinterpret_cast<float4*>(cop_)[ci] = v;
    }
}

template <int FS, bool CH>
__global__ void __launch_bounds__(MGT) k_coarse_operator(const uint8_t* __restrict__ fop0,
                                                          const void* __restrict__ fopc_,
                                                          const uint8_t* __restrict__ fmask, void* __restrict__ cop_,
                                                          uint8_t* __restrict__ cmask, int* __restrict__ inexact,
                                                          int fnx, int fny, int fnz, int cnx, int cny, int cnz) {
    pdl_begin();
    const i64 C = (i64)cnx * cny * cnz;
    const i64 ci = (i64)blockIdx.x * MGT + threadIdx.x;
    if (ci >= C) return;
    coarse_operator_at<FS, CH>(ci, fop0, fopc_, fmask, cop_, cmask, inexact, fnx, fny, fnz, cnx, cny, cnz);
}

// One red-black Gauss-Seidel colour (multigrid.cl:203-230) on either layout.
template <bool L0>
__device__ __forceinline__ void rbgs_at(i64 c, float* p, const float* __restrict__ b, const uint8_t* __restrict__ op0,
                                               const float4* __restrict__ opc, const uint8_t* __restrict__ mask,
                                               float delta, int parity, int nx, int ny, int nz) {
    int i, j, k;
    gcoord(c, ny, nz, i, j, k);
    const i64 sx = (i64)ny * nz, sy = nz;
    const float d2 = delta * delta;
    if (L0) {
        const uint32_t o = __ldg(op0 + c);
        const bool fluid = (o & 64u) != 0u;
        if (!interior(i, j, k, nx, ny, nz) || !fluid || ((i + j + k) & 1) != parity) {
            if (!fluid) p[c] = 0.0f;
            return;
        }
        const float d = (float)(o & 7u);
        if (d > 0.0f) p[c] = (wsum0<float>(op0, p, c, sx, sy, o) - d2 * __ldg(b + c)) / d;
    } else {
        const bool fluid = __ldg(mask + c) != 0;
        if (!interior(i, j, k, nx, ny, nz) || !fluid || ((i + j + k) & 1) != parity) {
            if (!fluid) p[c] = 0.0f;
            return;
        }
        // a fluid cell of the colour: the operator, neighbour weights, neighbours and b in one round trip
        const float4 o = __ldg(opc + c);
        const float wxm = __ldg(opc + c - sx).y, wym = __ldg(opc + c - sy).z, wzm = __ldg(opc + c - 1).w;
        const float pxp = p[c + sx], pxm = p[c - sx], pyp = p[c + sy], pym = p[c - sy], pzp = p[c + 1], pzm = p[c - 1];
        const float bc = __ldg(b + c);
        const float ws = o.y * pxp + wxm * pxm + o.z * pyp + wym * pym + o.w * pzp + wzm * pzm;
        if (o.x > 0.0f) p[c] = (ws - d2 * bc) / o.x;
    }
}

template <bool L0>
__global__ void __launch_bounds__(MGT) k_rbgs(float* p, const float* __restrict__ b, const uint8_t* __restrict__ op0,
                                               const float4* __restrict__ opc, const uint8_t* __restrict__ mask,
                                               float delta, int parity, int nx, int ny, int nz) {
    pdl_begin();
    const i64 C = (i64)nx * ny * nz;
    const i64 c = (i64)blockIdx.x * MGT + threadIdx.x;
    if (c >= C) return;
    rbgs_at<L0>(c, p, b, op0, opc, mask, delta, parity, nx, ny, nz);
}

// Residual (multigrid.cl:45-61) at one fine cell for either layout; 0 contribution when not fluid.
template <bool L0>
__device__ __forceinline__ float residual_at(const float* p, const float* __restrict__ b,
                                             const uint8_t* __restrict__ op0, const float4* __restrict__ opc,
                                             const uint8_t* __restrict__ mask, float inv_delta2, i64 f, i64 sx,
                                             i64 sy) {
    float ap;
    if (L0) {
        const uint32_t o = __ldg(op0 + f);
        ap = (wsum0<float>(op0, p, f, sx, sy, o) - (float)(o & 7u) * p[f]) * inv_delta2;
    } else {
        const float4 o = __ldg(opc + f);
        ap = (wsumC(opc, p, f, sx, sy, o) - o.x * p[f]) * inv_delta2;
    }
    return __ldg(b + f) - ap;
}

// Right-hand-side part of restrict_residual (multigrid.cl:90-180): coarse b = sum of the eight fine
// residuals in (di, dj, dk) order, coarse p = 0.
template <bool L0>
__device__ __forceinline__ void restrict_at(i64 ci, const float* __restrict__ fp, const float* __restrict__ fb,
                                                   const uint8_t* __restrict__ fop0, const float4* __restrict__ fopc,
                                                   const uint8_t* __restrict__ fmask, float* __restrict__ cp,
                                                   float* __restrict__ cb, float delta, int fnx, int fny, int fnz,
                                                   int cnx, int cny, int cnz) {
    cp[ci] = 0.0f;
    int I, J, K;
    gcoord(ci, cny, cnz, I, J, K);
    float rhs = 0.0f;
    if (interior(I, J, K, cnx, cny, cnz)) {
        const int si = 1 + 2 * (I - 1), sj = 1 + 2 * (J - 1), sk = 1 + 2 * (K - 1);
        const float inv_delta2 = 1.0f / (delta * delta);
        const i64 sx = (i64)fny * fnz, sy = fnz;
        // the eight children's fluid flags first, all loads at once; then the fluid children's
        // residuals in (di, dj, dk) order
        uint32_t flag[8];
#pragma unroll
        for (int ch = 0; ch < 8; ++ch) {
            const int i = si + (ch >> 2), j = sj + ((ch >> 1) & 1), k = sk + (ch & 1);
            const i64 f = gidx(i, j, k, fny, fnz);
            flag[ch] = !interior(i, j, k, fnx, fny, fnz) ? 0u
                       : L0 ? (uint32_t)__ldg(fop0 + f) : (__ldg(fmask + f) != 0 ? 64u : 0u);
        }
#pragma unroll
        for (int ch = 0; ch < 8; ++ch) {
            if (!(flag[ch] & 64u)) continue;
            const i64 f = gidx(si + (ch >> 2), sj + ((ch >> 1) & 1), sk + (ch & 1), fny, fnz);
            if (L0) {  // residual_at<true> with the operator byte already loaded
                const uint32_t o = flag[ch];
                const float ap = (wsum0<float>(fop0, fp, f, sx, sy, o) - (float)(o & 7u) * fp[f]) * inv_delta2;
                rhs += __ldg(fb + f) - ap;
            } else {
                rhs += residual_at<false>(fp, fb, fop0, fopc, fmask, inv_delta2, f, sx, sy);
            }
        }
    }
    cb[ci] = rhs;
}

template <bool L0>
__global__ void __launch_bounds__(MGT) k_restrict(const float* __restrict__ fp, const float* __restrict__ fb,
                                                   const uint8_t* __restrict__ fop0, const float4* __restrict__ fopc,
                                                   const uint8_t* __restrict__ fmask, float* __restrict__ cp,
                                                   float* __restrict__ cb, float delta, int fnx, int fny, int fnz,
                                                   int cnx, int cny, int cnz) {
    pdl_begin();
    const i64 C = (i64)cnx * cny * cnz;
    const i64 ci = (i64)blockIdx.x * MGT + threadIdx.x;
    if (ci >= C) return;
    restrict_at<L0>(ci, fp, fb, fop0, fopc, fmask, cp, cb, delta, fnx, fny, fnz, cnx, cny, cnz);
}

// prolongate (multigrid.cl:182-201) for either layout. w multiplies the prolonged correction (1: the
// reference's prolongation, bit for bit since 1 * e = e; see clb_mg_hierarchy.prolong_scale).
template <bool L0>
__device__ __forceinline__ void prolong_at(i64 f, const float* __restrict__ ce, float* __restrict__ fp,
                                                  const uint8_t* __restrict__ fop0, const uint8_t* __restrict__ fmask,
                                                  int cnx, int cny, int cnz, int fnx, int fny, int fnz,
                                                  float w = 1.0f) {
    int i, j, k;
    gcoord(f, fny, fnz, i, j, k);
    const bool fl = L0 ? ((__ldg(fop0 + f) & 64u) != 0u) : (__ldg(fmask + f) != 0);
    if (!interior(i, j, k, fnx, fny, fnz) || !fl) return;
    const int I = min((i - 1) / 2 + 1, cnx - 2), J = min((j - 1) / 2 + 1, cny - 2), K = min((k - 1) / 2 + 1, cnz - 2);
    fp[f] += w * __ldg(ce + gidx(I, J, K, cny, cnz));
}

template <bool L0>
__global__ void __launch_bounds__(MGT) k_prolong(const float* __restrict__ ce, float* __restrict__ fp,
                                                  const uint8_t* __restrict__ fop0, const uint8_t* __restrict__ fmask,
                                                  int cnx, int cny, int cnz, int fnx, int fny, int fnz, float w) {
    pdl_begin();
    const i64 C = (i64)fnx * fny * fnz;
    const i64 f = (i64)blockIdx.x * MGT + threadIdx.x;
    if (f >= C) return;
    prolong_at<L0>(f, ce, fp, fop0, fmask, cnx, cny, cnz, fnx, fny, fnz, w);
}

// coarse_smooth (multigrid.cl:232-264): one block runs all colour sweeps of the coarsest level,
// with the level's p, b and operator held in shared memory when they fit. Cells that are not
// interior fluid cells are never written (as in the reference).
constexpr int COARSE_THREADS = 1024;
constexpr int COARSE_SMEM_CELLS = 8192;  // 25 bytes per cell -> 200 KB

// H = true: an FP16 level (p, b, operator as __half, shared-memory path only); its scaled system uses
// kappa = scale[2] in place of delta^2 (mg_half.cuh).
template <bool SMEM, bool L0, bool H = false>
__device__ __forceinline__ void coarse_solve_block(float* p, const float* __restrict__ b,
                                                   const uint8_t* __restrict__ op0, const float4* __restrict__ opc,
                                                   const uint8_t* __restrict__ mask, float delta, int iterations,
                                                   int nx, int ny, int nz, const float* __restrict__ scale) {
    static_assert(!H || (SMEM && !L0), "FP16 levels are coarse levels solved from shared memory");
    extern __shared__ __align__(16) unsigned char smem[];
    const int C = nx * ny * nz;
    const float d2 = H ? scale[2] : delta * delta;
    const i64 sx = (i64)ny * nz, sy = nz;
    float* sp = reinterpret_cast<float*>(smem);
    float* sb = sp + C;
    float4* so = reinterpret_cast<float4*>(sb + C + ((4 - (2 * C) % 4) % 4));
    if (SMEM) {
        for (int c = threadIdx.x; c < C; c += COARSE_THREADS) {
            sp[c] = H ? ldh(reinterpret_cast<const __half*>(p), c) : p[c];
            sb[c] = H ? ldh(reinterpret_cast<const __half*>(b), c) : b[c];
            float4 o;
            if (L0) {
                const uint32_t v = op0[c];
                o = make_float4((v & 64u) ? (float)(v & 7u) : -1.0f, bitf(v, 3), bitf(v, 4), bitf(v, 5));
            } else {
                o = H ? ld_h4(reinterpret_cast<const Half4*>(opc), c) : opc[c];
                if (!mask[c]) o.x = -1.0f;  // marks "not fluid"; diag itself is never negative
            }
            so[c] = o;
        }
        __syncthreads();
    }
    for (int it = 0; it < iterations; ++it)
        for (int parity = 0; parity < 2; ++parity) {
            for (int c = threadIdx.x; c < C; c += COARSE_THREADS) {
                int i, j, k;
                gcoord(c, ny, nz, i, j, k);
                if (!interior(i, j, k, nx, ny, nz) || ((i + j + k) & 1) != parity) continue;
                if (SMEM) {
                    const float4 o = so[c];
                    if (o.x < 0.0f) continue;
                    const float ws = o.y * sp[c + sx] + so[c - sx].y * sp[c - sx] + o.z * sp[c + sy] +
                                     so[c - sy].z * sp[c - sy] + o.w * sp[c + 1] + so[c - 1].w * sp[c - 1];
                    if (o.x > 0.0f) sp[c] = (ws - d2 * sb[c]) / o.x;
                } else if (L0) {
                    const uint32_t o = op0[c];
                    if (!(o & 64u)) continue;
                    const float d = (float)(o & 7u);
                    if (d > 0.0f) p[c] = (wsum0<float>(op0, p, c, sx, sy, o) - d2 * b[c]) / d;
                } else {
                    if (!mask[c]) continue;
                    const float4 o = opc[c];
                    if (o.x > 0.0f) p[c] = (wsumC(opc, p, c, sx, sy, o) - d2 * b[c]) / o.x;
                }
            }
            __syncthreads();
        }
    if (SMEM)
        for (int c = threadIdx.x; c < C; c += COARSE_THREADS) {
            if (H) reinterpret_cast<__half*>(p)[c] = __float2half_rn(sp[c]);
            else p[c] = sp[c];
        }
}

template <bool SMEM, bool L0, bool H = false>
__global__ void __launch_bounds__(COARSE_THREADS) k_coarse_solve(float* p, const float* __restrict__ b,
                                                                  const uint8_t* __restrict__ op0,
                                                                  const float4* __restrict__ opc,
                                                                  const uint8_t* __restrict__ mask, float delta,
                                                                  int iterations, int nx, int ny, int nz,
                                                                  const float* __restrict__ scale = nullptr) {
    pdl_begin();
    coarse_solve_block<SMEM, L0, H>(p, b, op0, opc, mask, delta, iterations, nx, ny, nz, scale);
}

static inline size_t coarse_smem_bytes(int C) {
    return (size_t)C * 8 + (size_t)(((4 - (2 * C) % 4) % 4) * 4) + (size_t)C * 16;
}

// ------------------------------------------------------------------------------------------------
// FP64 residual norms and iterative refinement on the finest level (packed layout).
// ------------------------------------------------------------------------------------------------
constexpr int RN_THREADS = 256;

// FP64 residual over the finest level, one (i, j) row per warp (lanes stride along k, so there is no
// per-cell index division). Per block: sums of r^2 and b^2 over interior fluid cells, with
// r = b - A p evaluated in FP64 (A is multigrid.cl:25-43 apply_operator).
//  MODE 0 (RES_NORM): p is the float or double pressure p_in.
//  MODE 1 (RES_IR):   the refinement update fused in: p = p_in + e is formed on the fly for the cell
//                     and its neighbours and written to p_out (which must not alias p_in).
//  MODE 2 (RES_FCG):  the flexible-CG update fused in: the search direction d = e + beta d_in
//                     (rounded to float, written to d_out) and p = p_in + alpha d, with alpha and
//                     beta read from state[0] and state[1] (k_fcg_scalars).
// When r_out is given the residual is stored rounded to float at every cell (0 outside interior
// fluid cells): it is the right-hand side of the next correction solve.
// SKIP (refinement and FCG steps): cells that are not interior fluid cells are neither read nor
// written. Every value there is 0 when the caller keeps the invariant (e, d_in, p_in, and the
// outputs zeroed outside the fluid once per solve), so the outputs and sums are those of the full
// pass; the per-lane summation order over fluid cells is unchanged.
enum { RES_NORM = 0, RES_IR = 1, RES_FCG = 2 };

// Whether row `base` (nz cells of the packed finest operator) holds a fluid cell, for the whole warp:
// one 8-byte load per lane per 256 cells (when the row starts 8-byte aligned) instead of the per-cell
// byte loads a row without fluid would otherwise cost. Skipping such a row changes no sum: none of its
// cells contributes.
__device__ __forceinline__ bool row_has_fluid(const uint8_t* __restrict__ op0, i64 base, int nz, int lane) {
    bool any = false;
    if ((((uintptr_t)(op0 + base)) & 7) == 0) {
        for (int k = lane * 8; k < nz; k += 256) {
            const int n = nz - k < 8 ? nz - k : 8;
            if (n == 8) {
                const uint2 w = __ldg(reinterpret_cast<const uint2*>(op0 + base + k));
                any |= ((w.x | w.y) & 0x40404040u) != 0u;
            } else {
                for (int q = 0; q < n; ++q) any |= (__ldg(op0 + base + k + q) & 64u) != 0u;
            }
        }
    } else {
        for (int k = lane; k < nz; k += 32) any |= (__ldg(op0 + base + k) & 64u) != 0u;
    }
    return __any_sync(0xffffffffu, any);
}

// Block `blk` of `nblk` blocks sharing the rows; its partial sums go to *partial.
template <typename PT, int MODE, bool SKIP = false>
__device__ __forceinline__ void residual_rows_block(int blk, int nblk, const PT* __restrict__ p_in,
                                                    const float* __restrict__ e, double* __restrict__ p_out,
                                                    const float* __restrict__ b, const uint8_t* __restrict__ op0,
                                                    double inv_delta2, int nx, int ny, int nz,
                                                    float* __restrict__ r_out, double2* __restrict__ partial,
                                                    const float* __restrict__ d_in, float* __restrict__ d_out,
                                                    const double* __restrict__ state) {
    __shared__ double2 s_red[RN_THREADS / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int sx = ny * nz, sy = nz;
    double rr = 0.0, bb = 0.0;
    double alpha = 0.0, beta = 0.0;
    if (MODE == RES_FCG) {
        alpha = state[0];
        beta = state[1];
    }
    auto dv = [&](int q) -> float { return (float)((double)__ldg(e + q) + beta * (double)__ldg(d_in + q)); };
    auto pv = [&](int q) -> double {
        if (MODE == RES_IR) return (double)__ldg(p_in + q) + (double)__ldg(e + q);
        if (MODE == RES_FCG) return (double)__ldg(p_in + q) + alpha * (double)dv(q);
        return (double)__ldg(p_in + q);
    };
    const int rows = nx * ny;
    for (int r = blk * (RN_THREADS / 32) + warp; r < rows; r += nblk * (RN_THREADS / 32)) {
        const int i = r / ny, j = r - i * ny;
        const bool row_in = i >= 1 && i <= nx - 2 && j >= 1 && j <= ny - 2;
        const int base = r * nz;
        if (SKIP && MODE != RES_NORM && (!row_in || !row_has_fluid(op0, base, nz, lane))) continue;
        // a lane's operator bytes of 8 consecutive steps are loaded together, so a step waits on one
        // round of loads (its stencil), not two (the byte that says whether the cell is fluid first)
        for (int k0 = 0; k0 < nz; k0 += 256) {
        unsigned long long ops = 0ull;  // byte m: the operator of step m
#pragma unroll
        for (int m = 0; m < 8; ++m) {
            const int k = k0 + lane + 32 * m;
            if (k < nz) ops |= (unsigned long long)__ldg(op0 + base + k) << (8 * m);
        }
#pragma unroll 1
        for (int m = 0; m < 8; ++m) {
            const int k = k0 + lane + 32 * m;
            if (k >= nz) continue;
            const int c = base + k;
            const uint32_t o = (uint32_t)(ops >> (8 * m)) & 0xffu;
            if (SKIP && MODE != RES_NORM && !(row_in && k >= 1 && k <= nz - 2 && (o & 64u))) continue;
            const double pc = pv(c);
            if (MODE != RES_NORM) p_out[c] = pc;
            if (MODE == RES_FCG) d_out[c] = dv(c);
            float rf = 0.0f;
            if (row_in && k >= 1 && k <= nz - 2 && (o & 64u)) {
                const uint32_t ox = __ldg(op0 + c - sx), oy = __ldg(op0 + c - sy), oz = __ldg(op0 + c - 1);
                const double ws = (double)bitf(o, 3) * pv(c + sx) + (double)bitf(ox, 3) * pv(c - sx) +
                                  (double)bitf(o, 4) * pv(c + sy) + (double)bitf(oy, 4) * pv(c - sy) +
                                  (double)bitf(o, 5) * pv(c + 1) + (double)bitf(oz, 5) * pv(c - 1);
                const double bv = (double)__ldg(b + c);
                const double res = bv - (ws - (double)(o & 7u) * pc) * inv_delta2;
                rr += res * res;
                bb += bv * bv;
                rf = (float)res;
            }
            if (r_out) r_out[c] = rf;
        }
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        rr += __shfl_xor_sync(0xffffffffu, rr, o);
        bb += __shfl_xor_sync(0xffffffffu, bb, o);
    }
    if (lane == 0) s_red[warp] = make_double2(rr, bb);
    __syncthreads();
    if (threadIdx.x == 0) {
        double2 t = s_red[0];
        for (int q = 1; q < RN_THREADS / 32; ++q) {
            t.x += s_red[q].x;
            t.y += s_red[q].y;
        }
        *partial = t;
    }
}

template <typename PT, int MODE, bool SKIP = false>
__global__ void __launch_bounds__(RN_THREADS) k_residual_rows(const PT* __restrict__ p_in,
                                                               const float* __restrict__ e,
                                                               double* __restrict__ p_out,
                                                               const float* __restrict__ b,
                                                               const uint8_t* __restrict__ op0, double inv_delta2,
                                                               int nx, int ny, int nz, float* __restrict__ r_out,
                                                               double2* __restrict__ partials,
                                                               const float* __restrict__ d_in = nullptr,
                                                               float* __restrict__ d_out = nullptr,
                                                               const double* __restrict__ state = nullptr) {
    pdl_begin();
    residual_rows_block<PT, MODE, SKIP>(blockIdx.x, gridDim.x, p_in, e, p_out, b, op0, inv_delta2, nx, ny, nz, r_out,
                                  partials + blockIdx.x, d_in, d_out, state);
}

// Flexible conjugate gradients with the W-cycle as preconditioner (Notay's FCG with truncation 1;
// no counterpart in the reference, which runs W-cycles only). For the preconditioned residual
// z = e (one W-cycle on A e = r from e = 0) and the previous direction d, one block's partial sums
// over interior fluid cells of
//   x = (A z) . d     (= z . A d, the operator is symmetric)
//   y = (A z) . z,    z_ = z . r,    w = d . r
// with A z evaluated in FP64. The next direction is d' = z + beta d, beta = -(z . A d) / (d . A d),
// so d' . A d' and d' . r follow from these four sums and the previous d . A d without storing A d.
struct Sum4 {
    double x, y, z, w;
};

__device__ __forceinline__ void fcg_dots_block(int blk, int nblk, const float* __restrict__ z,
                                               const float* __restrict__ d, const float* __restrict__ r,
                                               const uint8_t* __restrict__ op0, double inv_delta2, int nx, int ny,
                                               int nz, Sum4* __restrict__ partial) {
    __shared__ Sum4 s_red[RN_THREADS / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int sx = ny * nz, sy = nz;
    Sum4 t = {0.0, 0.0, 0.0, 0.0};
    const int rows = nx * ny;
    for (int q = blk * (RN_THREADS / 32) + warp; q < rows; q += nblk * (RN_THREADS / 32)) {
        const int i = q / ny, j = q - i * ny;
        if (i < 1 || i > nx - 2 || j < 1 || j > ny - 2) continue;
        const int base = q * nz;
        if (!row_has_fluid(op0, base, nz, lane)) continue;
        for (int k = lane; k < nz; k += 32) {
            const int c = base + k;
            const uint32_t o = __ldg(op0 + c);
            if (k < 1 || k > nz - 2 || !(o & 64u)) continue;
            const uint32_t ox = __ldg(op0 + c - sx), oy = __ldg(op0 + c - sy), oz = __ldg(op0 + c - 1);
            const double zc = (double)__ldg(z + c);
            const double ws = (double)bitf(o, 3) * (double)__ldg(z + c + sx) +
                              (double)bitf(ox, 3) * (double)__ldg(z + c - sx) +
                              (double)bitf(o, 4) * (double)__ldg(z + c + sy) +
                              (double)bitf(oy, 4) * (double)__ldg(z + c - sy) +
                              (double)bitf(o, 5) * (double)__ldg(z + c + 1) +
                              (double)bitf(oz, 5) * (double)__ldg(z + c - 1);
            const double az = (ws - (double)(o & 7u) * zc) * inv_delta2;
            const double dc = (double)__ldg(d + c), rc = (double)__ldg(r + c);
            t.x += az * dc;
            t.y += az * zc;
            t.z += zc * rc;
            t.w += dc * rc;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        t.x += __shfl_xor_sync(0xffffffffu, t.x, o);
        t.y += __shfl_xor_sync(0xffffffffu, t.y, o);
        t.z += __shfl_xor_sync(0xffffffffu, t.z, o);
        t.w += __shfl_xor_sync(0xffffffffu, t.w, o);
    }
    if (lane == 0) s_red[warp] = t;
    __syncthreads();
    if (threadIdx.x == 0) {
        Sum4 a = s_red[0];
        for (int q = 1; q < RN_THREADS / 32; ++q) {
            a.x += s_red[q].x;
            a.y += s_red[q].y;
            a.z += s_red[q].z;
            a.w += s_red[q].w;
        }
        *partial = a;
    }
}

__global__ void __launch_bounds__(RN_THREADS) k_fcg_dots(const float* __restrict__ z, const float* __restrict__ d,
                                                          const float* __restrict__ r,
                                                          const uint8_t* __restrict__ op0, double inv_delta2, int nx,
                                                          int ny, int nz, Sum4* __restrict__ partials) {
    pdl_begin();
    fcg_dots_block(blockIdx.x, gridDim.x, z, d, r, op0, inv_delta2, nx, ny, nz, partials + blockIdx.x);
}

// Fixed-order sum of the k_fcg_dots partials, then the FCG scalars in
// state = {alpha, beta, d.Ad of the current direction, 1 once a direction exists}.
// The first direction is z itself (beta = 0).
__device__ __forceinline__ void fcg_scalars_block(const Sum4* __restrict__ partials, int count,
                                                  double* __restrict__ state) {
    __shared__ Sum4 s[256];
    Sum4 t = {0.0, 0.0, 0.0, 0.0};
    for (int q = threadIdx.x; q < count; q += 256) {
        t.x += partials[q].x;
        t.y += partials[q].y;
        t.z += partials[q].z;
        t.w += partials[q].w;
    }
    s[threadIdx.x] = t;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if (threadIdx.x < o) {
            s[threadIdx.x].x += s[threadIdx.x + o].x;
            s[threadIdx.x].y += s[threadIdx.x + o].y;
            s[threadIdx.x].z += s[threadIdx.x + o].z;
            s[threadIdx.x].w += s[threadIdx.x + o].w;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const Sum4 a = s[0];
        const bool has = state[3] != 0.0 && state[2] != 0.0;
        double beta = 0.0, dad = a.y, dr = a.z;
        if (has) {
            beta = -a.x / state[2];
            dad = a.y + 2.0 * beta * a.x + beta * beta * state[2];
            dr = a.z + beta * a.w;
        }
        state[0] = dad != 0.0 ? dr / dad : 0.0;
        state[1] = beta;
        state[2] = dad;
        state[3] = 1.0;
    }
}

__global__ void k_fcg_scalars(const Sum4* __restrict__ partials, int count, double* __restrict__ state) {
    pdl_begin();
    fcg_scalars_block(partials, count, state);
}

// Fixed-order reduction of the block partials (deterministic for a given grid size).
__device__ __forceinline__ void reduce_partials_block(const double2* __restrict__ partials, int count,
                                                      double2* __restrict__ out) {
    __shared__ double2 s[256];
    double2 t = make_double2(0.0, 0.0);
    for (int q = threadIdx.x; q < count; q += 256) {
        t.x += partials[q].x;
        t.y += partials[q].y;
    }
    s[threadIdx.x] = t;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if (threadIdx.x < o) {
            s[threadIdx.x].x += s[threadIdx.x + o].x;
            s[threadIdx.x].y += s[threadIdx.x + o].y;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = s[0];
}

__global__ void k_reduce_partials(const double2* __restrict__ partials, int count, double2* __restrict__ out) {
    pdl_begin();
    reduce_partials_block(partials, count, out);
}

// p64 = warm-start pressure at interior fluid cells, 0 elsewhere (cells that left the liquid since
// the previous step must not keep a stale pressure).
__device__ __forceinline__ void ir_init_at(i64 c, const float* __restrict__ p, const uint8_t* __restrict__ op0,
                                                  double* __restrict__ p64, int nx, int ny, int nz) {
    int i, j, k;
    gcoord(c, ny, nz, i, j, k);
    p64[c] = (interior(i, j, k, nx, ny, nz) && (__ldg(op0 + c) & 64u)) ? (double)__ldg(p + c) : 0.0;
}

__global__ void __launch_bounds__(MGT) k_ir_init(const float* __restrict__ p, const uint8_t* __restrict__ op0,
                                                  double* __restrict__ p64, int nx, int ny, int nz) {
    pdl_begin();
    const i64 C = (i64)nx * ny * nz;
    const i64 c = (i64)blockIdx.x * MGT + threadIdx.x;
    if (c >= C) return;
    ir_init_at(c, p, op0, p64, nx, ny, nz);
}

// The same four cells at a time (nz % 4 == 0, so the four share a row; p 16-byte and op0 4-byte
// aligned): one 16-byte load of p, one 4-byte load of operator bytes, two 16-byte stores.
__global__ void __launch_bounds__(MGT) k_ir_init4(const float* __restrict__ p, const uint8_t* __restrict__ op0,
                                                   double* __restrict__ p64, int nx, int ny, int nz) {
    pdl_begin();
    const i64 C4 = (i64)nx * ny * nz / 4;
    const i64 q = (i64)blockIdx.x * MGT + threadIdx.x;
    if (q >= C4) return;
    const i64 c = 4 * q;
    const i64 row = c / nz;
    const int k0 = (int)(c - row * nz), i = (int)(row / ny), j = (int)(row - (i64)i * ny);
    const bool row_in = i >= 1 && i <= nx - 2 && j >= 1 && j <= ny - 2;
    const float4 v = __ldg(reinterpret_cast<const float4*>(p + c));
    const uchar4 o = __ldg(reinterpret_cast<const uchar4*>(op0 + c));
    auto in = [&](int k, unsigned char b) { return row_in && k >= 1 && k <= nz - 2 && (b & 64u); };
    reinterpret_cast<double2*>(p64 + c)[0] =
        make_double2(in(k0, o.x) ? (double)v.x : 0.0, in(k0 + 1, o.y) ? (double)v.y : 0.0);
    reinterpret_cast<double2*>(p64 + c)[1] =
        make_double2(in(k0 + 2, o.z) ? (double)v.z : 0.0, in(k0 + 3, o.w) ? (double)v.w : 0.0);
}

__global__ void __launch_bounds__(MGT) k_ir_update(double* __restrict__ p64, const float* __restrict__ e, i64 C) {
    pdl_begin();
    const i64 c = (i64)blockIdx.x * MGT + threadIdx.x;
    if (c < C) p64[c] += (double)__ldg(e + c);
}

__global__ void __launch_bounds__(MGT) k_ir_store(const double* __restrict__ p64, float* __restrict__ p, i64 C) {
    pdl_begin();
    const i64 c = (i64)blockIdx.x * MGT + threadIdx.x;
    if (c < C) p[c] = (float)__ldg(p64 + c);
}

// The same four cells at a time (C4 = C / 4; p64 and p 16-byte aligned).
__global__ void __launch_bounds__(MGT) k_ir_store4(const double* __restrict__ p64, float* __restrict__ p, i64 C4) {
    pdl_begin();
    const i64 q = (i64)blockIdx.x * MGT + threadIdx.x;
    if (q >= C4) return;
    const double2 a = __ldg(reinterpret_cast<const double2*>(p64) + 2 * q);
    const double2 b = __ldg(reinterpret_cast<const double2*>(p64) + 2 * q + 1);
    reinterpret_cast<float4*>(p)[q] = make_float4((float)a.x, (float)a.y, (float)b.x, (float)b.y);
}

}  // namespace clb
