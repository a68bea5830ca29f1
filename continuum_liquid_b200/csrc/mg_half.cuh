// FP16 storage of the coarse multigrid levels (no counterpart in the reference, which is FP32
// throughout).
//
// The levels from the hierarchy's fp16_level down to the coarsest store p, b and the operator as
// __half; every update is computed in FP32 and rounded once when stored. The operator entries are
// sums of small integers and convert exactly (k_coarse_operator counts the ones that do not).
//
// p and b need scaling: a W-cycle solves A e = r for the current FP64-refined residual, whose size
// runs from the right-hand side's (about 1e6 at 256^3) down by the tolerance, far outside FP16's
// range. A W-cycle is linear in r, so the FP16 levels hold b_s = sigma_b b and p_s = sigma_p p with
// powers of two
//   sigma_b = 2^-ceil(log2 ||r||_2)  (then |b| on level l <= sqrt(8^l) ||sigma_b r||_2 <= 2^(1.5 l))
//   sigma_p = sigma_b 2^k,  2^k ~ 1 / delta^2,
// and the scaled system's smoother p_s = (sum w p_s - kappa b_s) / diag uses kappa = delta^2 2^k
// (between 0.5 and 1) in place of delta^2; residuals in scaled units are b_s - A_int(p_s) / kappa.
// Scales are applied where an FP32 level meets the first FP16 level (restriction and prolongation);
// between FP16 levels they cancel. ||r||_2^2 is the sum the residual kernels already leave in the
// hierarchy's rhs_norms, so the scales are formed on the device inside the captured W-cycle.
#pragma once
#include "multigrid.cuh"

namespace clb {

// scale = {sigma_b, 1 / sigma_p, kappa, 1 / kappa} from rhs_norms[0] = ||r||_2^2 (one thread).
__global__ void k_fp16_scale(const double* __restrict__ rhs_norms, float delta, float* __restrict__ scale) {
    pdl_begin();
    if (threadIdx.x != 0) return;
    const double nrm = sqrt(fmax(rhs_norms[0], 0.0));
    int eb = 0;
    if (nrm > 0.0 && isfinite(nrm)) frexp(nrm, &eb);  // nrm < 2^eb
    const float d2 = delta * delta;
    int ed = 0;
    frexpf(d2, &ed);  // d2 = m 2^ed, m in [0.5, 1)
    const int k = -ed;
    const float kappa = ldexpf(d2, k);  // exact: a power-of-two scaling of d2
    scale[0] = ldexpf(1.0f, -eb);
    scale[1] = ldexpf(1.0f, eb - k);
    scale[2] = kappa;
    scale[3] = 1.0f / kappa;
}

// One red-black colour (multigrid.cl:203-230) on an FP16 level, one cell per thread.
__global__ void __launch_bounds__(MGT) k_rbgs_h(__half* p, const __half* __restrict__ b, const Half4* __restrict__ op,
                                                 const uint8_t* __restrict__ mask, const float* __restrict__ scale,
                                                 int parity, int nx, int ny, int nz) {
    pdl_begin();
    const i64 C = (i64)nx * ny * nz;
    const i64 c = (i64)blockIdx.x * MGT + threadIdx.x;
    if (c >= C) return;
    int i, j, k;
    gcoord(c, ny, nz, i, j, k);
    const i64 sx = (i64)ny * nz, sy = nz;
    const bool fluid = __ldg(mask + c) != 0;
    if (!interior(i, j, k, nx, ny, nz) || !fluid || ((i + j + k) & 1) != parity) {
        if (!fluid) p[c] = __float2half_rn(0.0f);
        return;
    }
    // a fluid cell of the colour: the operator, neighbour weights, neighbours and b in one round trip
    const float4 o = ld_h4(op, c);
    const float wxm = ld_h4(op, c - sx).y, wym = ld_h4(op, c - sy).z, wzm = ld_h4(op, c - 1).w;
    const float pxp = ldh(p, c + sx), pxm = ldh(p, c - sx), pyp = ldh(p, c + sy), pym = ldh(p, c - sy);
    const float pzp = ldh(p, c + 1), pzm = ldh(p, c - 1), bc = ldh(b, c), kappa = scale[2];
    if (!(o.x > 0.0f)) return;
    const float ws = o.y * pxp + wxm * pxm + o.z * pyp + wym * pym + o.w * pzp + wzm * pzm;
    p[c] = __float2half_rn((ws - kappa * bc) / o.x);
}

// Residual at an FP16 fine cell in scaled units: b_s - (sum w p_s - diag p_s) / kappa.
__device__ __forceinline__ float residual_h(const __half* p, const __half* __restrict__ b,
                                           const Half4* __restrict__ op, float inv_kappa, i64 f, i64 sx, i64 sy) {
    const float4 o = ld_h4(op, f);
    const float ws = o.y * ldh(p, f + sx) + ld_h4(op, f - sx).y * ldh(p, f - sx) + o.z * ldh(p, f + sy) +
                     ld_h4(op, f - sy).z * ldh(p, f - sy) + o.w * ldh(p, f + 1) + ld_h4(op, f - 1).w * ldh(p, f - 1);
    return ldh(b, f) - (ws - o.x * ldh(p, f)) * inv_kappa;
}

// Restriction (multigrid.cl:90-180, right-hand-side part) into an FP16 coarse level from a fine
// level of layout FS (0 packed finest FP32, 1 FP32 coarse, 2 FP16). From an FP32 level the sum of
// the eight fine residuals is the FP32 path's, then scaled by sigma_b.
template <int FS>
__device__ __forceinline__ void restrict_h_at(i64 ci, const void* __restrict__ fp, const void* __restrict__ fb,
                                              const uint8_t* __restrict__ fop0, const void* __restrict__ fopc,
                                              const uint8_t* __restrict__ fmask, __half* __restrict__ cp,
                                              __half* __restrict__ cb, float delta, const float* __restrict__ scale,
                                              int fnx, int fny, int fnz, int cnx, int cny, int cnz) {
    cp[ci] = __float2half_rn(0.0f);
    int I, J, K;
    gcoord(ci, cny, cnz, I, J, K);
    float rhs = 0.0f;
    if (interior(I, J, K, cnx, cny, cnz)) {
        const int si = 1 + 2 * (I - 1), sj = 1 + 2 * (J - 1), sk = 1 + 2 * (K - 1);
        const float inv = FS == 2 ? scale[3] : 1.0f / (delta * delta);
        const i64 sx = (i64)fny * fnz, sy = fnz;
        for (int di = 0; di < 2; ++di)
            for (int dj = 0; dj < 2; ++dj)
                for (int dk = 0; dk < 2; ++dk) {
                    const int i = si + di, j = sj + dj, k = sk + dk;
                    if (!interior(i, j, k, fnx, fny, fnz)) continue;
                    const i64 f = gidx(i, j, k, fny, fnz);
                    const bool fl = FS == 0 ? ((__ldg(fop0 + f) & 64u) != 0u) : (__ldg(fmask + f) != 0);
                    if (!fl) continue;
                    if (FS == 2)
                        rhs += residual_h(reinterpret_cast<const __half*>(fp), reinterpret_cast<const __half*>(fb),
                                          reinterpret_cast<const Half4*>(fopc), inv, f, sx, sy);
                    else
                        rhs += residual_at<FS == 0>(reinterpret_cast<const float*>(fp),
                                                    reinterpret_cast<const float*>(fb), fop0,
                                                    reinterpret_cast<const float4*>(fopc), fmask, inv, f, sx, sy);
                }
    }
    cb[ci] = __float2half_rn(FS == 2 ? rhs : rhs * scale[0]);
}

template <int FS>
__global__ void __launch_bounds__(MGT) k_restrict_h(const void* __restrict__ fp, const void* __restrict__ fb,
                                                     const uint8_t* __restrict__ fop0, const void* __restrict__ fopc,
                                                     const uint8_t* __restrict__ fmask, __half* __restrict__ cp,
                                                     __half* __restrict__ cb, float delta,
                                                     const float* __restrict__ scale, int fnx, int fny, int fnz,
                                                     int cnx, int cny, int cnz) {
    pdl_begin();
    const i64 C = (i64)cnx * cny * cnz;
    const i64 ci = (i64)blockIdx.x * MGT + threadIdx.x;
    if (ci >= C) return;
    restrict_h_at<FS>(ci, fp, fb, fop0, fopc, fmask, cp, cb, delta, scale, fnx, fny, fnz, cnx, cny, cnz);
}

// Prolongation (multigrid.cl:182-201) from an FP16 coarse level into a fine level of layout FS; into
// an FP32 level the coarse value is unscaled by 1 / sigma_p. w multiplies the prolonged correction.
template <int FS>
__device__ __forceinline__ void prolong_h_at(i64 f, const __half* __restrict__ ce, void* __restrict__ fp,
                                             const uint8_t* __restrict__ fop0, const uint8_t* __restrict__ fmask,
                                             const float* __restrict__ scale, int cnx, int cny, int cnz, int fnx,
                                             int fny, int fnz, float w) {
    int i, j, k;
    gcoord(f, fny, fnz, i, j, k);
    const bool fl = FS == 0 ? ((__ldg(fop0 + f) & 64u) != 0u) : (__ldg(fmask + f) != 0);
    if (!interior(i, j, k, fnx, fny, fnz) || !fl) return;
    const int I = min((i - 1) / 2 + 1, cnx - 2), J = min((j - 1) / 2 + 1, cny - 2), K = min((k - 1) / 2 + 1, cnz - 2);
    const float e = ldh(ce, gidx(I, J, K, cny, cnz));
    if (FS == 2) {
        __half* p = reinterpret_cast<__half*>(fp);
        p[f] = __float2half_rn(__half2float(p[f]) + w * e);
    } else {
        reinterpret_cast<float*>(fp)[f] += w * (e * scale[1]);
    }
}

template <int FS>
__global__ void __launch_bounds__(MGT) k_prolong_h(const __half* __restrict__ ce, void* __restrict__ fp,
                                                    const uint8_t* __restrict__ fop0, const uint8_t* __restrict__ fmask,
                                                    const float* __restrict__ scale, int cnx, int cny, int cnz,
                                                    int fnx, int fny, int fnz, float w) {
    pdl_begin();
    const i64 C = (i64)fnx * fny * fnz;
    const i64 f = (i64)blockIdx.x * MGT + threadIdx.x;
    if (f >= C) return;
    prolong_h_at<FS>(f, ce, fp, fop0, fmask, scale, cnx, cny, cnz, fnx, fny, fnz, w);
}

}  // namespace clb
