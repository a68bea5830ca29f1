// 3x3x3 convolutions (padding 1, stride 1) of the learned pressure warm start as implicit GEMMs on
// the tcgen05 core (tc_gemm.cuh). Activations are channels-last BF16 volumes [B][D][H][W][C] with C a
// multiple of 8; the 27 taps are ordered (dz, dy, dx) with dx fastest, offsets -1..1.
//
//   forward   y[v][co] = act(b[co] + sum_{tap,ci} x[v + o(tap)][ci] * W[tap][ci][co])
//             GEMM: M = voxels (tiles of 128), N = Cout, K = 27 * Cin (K-major gathers of x, weights
//             pre-arranged as wf[co][tap * Cin + ci]); bias and ReLU fused in the epilogue.
//   data grad dx[v][ci] = mask(ci) * sum_{tap,co} dy[v - o(tap)][co] * W[tap][ci][co]
//             GEMM: M = voxels, N = Cin, K = 27 * Cout (wd[ci][tap * Cout + co]); the ReLU backward
//             of the layer that produced x (mask = x > 0) is fused in the epilogue.
//   weight grad dW[tap * Cin + ci][co] += sum_v x[v + o(tap)][ci] * dy[v][co]
//             GEMM: M = 27 * Cin (tiles of 128), N = Cout, K = voxels split over blocks; both
//             operands MN-major (16-byte rows of 8 consecutive channels); FP32 atomics in the
//             epilogue accumulate the blocks' partial sums.
#pragma once
#include "tc_gemm.cuh"

namespace clb {
namespace conv {

using tc::TC_KC;
using tc::TC_M;
using tc::TC_THREADS;

struct Vol {
    int B, D, H, W;
    __device__ __forceinline__ int voxels() const { return B * D * H * W; }
};

// neighbour of voxel (b, z, y, x) at tap t, or -1 outside the volume
__device__ __forceinline__ int tap_neighbour(const Vol& g, int b, int z, int y, int x, int tap, int sign) {
    const int dz = tap / 9 - 1, dy = (tap / 3) % 3 - 1, dx = tap % 3 - 1;
    const int zz = z + sign * dz, yy = y + sign * dy, xx = x + sign * dx;
    if (zz < 0 || zz >= g.D || yy < 0 || yy >= g.H || xx < 0 || xx >= g.W) return -1;
    return ((b * g.D + zz) * g.H + yy) * g.W + xx;
}

__device__ __forceinline__ void decode(const Vol& g, int v, int& b, int& z, int& y, int& x) {
    x = v % g.W;
    int r = v / g.W;
    y = r % g.H;
    r /= g.H;
    z = r % g.D;
    b = r / g.D;
}

__device__ __forceinline__ uint32_t pack_bf16x2(float a, float b) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<const uint32_t*>(&h);
}

// ---- forward and data gradient: A = gathered activations (K-major), B = arranged weights ----------
template <int N, bool DGRAD>
struct ConvRows {
    static constexpr bool A_MN = false, B_MN = false;
    const __nv_bfloat16* src;  // forward: x [V][Cs]; data grad: dy [V][Cs]
    const __nv_bfloat16* wmat;  // [N][Kpad] bf16
    const float* bias;          // forward only (nullable)
    const __nv_bfloat16* mask_src;  // data grad: x [V][N] for the ReLU mask (nullable)
    __nv_bfloat16* out;         // [V][N]
    Vol g;
    int Cs, K, Kpad, chunks, m0, relu;
    int vb, vz, vy, vx;  // this thread's row voxel (row = threadIdx.x)
    bool valid;
    __device__ void setup() {
        const int v = m0 + threadIdx.x;
        valid = v < g.voxels();
        if (valid) decode(g, v, vb, vz, vy, vx);
    }
    __device__ void gather_a(uint8_t* st, int chunk) const {
        const int row = threadIdx.x;
#pragma unroll
        for (int kv = 0; kv < TC_KC / 8; ++kv) {
            const int k = chunk * TC_KC + kv * 8;
            uint4 val = make_uint4(0, 0, 0, 0);
            if (valid && k < K) {
                const int tap = k / Cs, c = k - tap * Cs;
                const int nb = tap_neighbour(g, vb, vz, vy, vx, tap, DGRAD ? -1 : 1);
                if (nb >= 0) val = __ldg(reinterpret_cast<const uint4*>(src + (i64)nb * Cs + c));
            }
            *reinterpret_cast<uint4*>(st + tc::kmajor_off(row, kv)) = val;
        }
    }
    __device__ void gather_b(uint8_t* st, int chunk) const {
        for (int t = threadIdx.x; t < N * (TC_KC / 8); t += TC_THREADS) {
            const int row = t / (TC_KC / 8), kv = t % (TC_KC / 8);
            const uint4 val = __ldg(reinterpret_cast<const uint4*>(wmat + (i64)row * Kpad + chunk * TC_KC + kv * 8));
            *reinterpret_cast<uint4*>(st + tc::kmajor_off(row, kv)) = val;
        }
    }
    __device__ void epilogue(int row, const float* acc, int col0) const {
        const int v = m0 + row;
        if (v >= g.voxels()) return;
        float r[16];
#pragma unroll
        for (int q = 0; q < 16; ++q) {
            float a = acc[q];
            if (!DGRAD) {
                if (bias) a += __ldg(bias + col0 + q);
                if (relu) a = fmaxf(a, 0.0f);
            }
            r[q] = a;
        }
        if (DGRAD && mask_src) {
            const uint4* m4 = reinterpret_cast<const uint4*>(mask_src + (i64)v * N + col0);
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const uint4 mv = __ldg(m4 + h);
                const __nv_bfloat16* mb = reinterpret_cast<const __nv_bfloat16*>(&mv);
#pragma unroll
                for (int q = 0; q < 8; ++q)
                    if (!(__bfloat162float(mb[q]) > 0.0f)) r[8 * h + q] = 0.0f;
            }
        }
        uint4* o4 = reinterpret_cast<uint4*>(out + (i64)v * N + col0);
        o4[0] = make_uint4(pack_bf16x2(r[0], r[1]), pack_bf16x2(r[2], r[3]), pack_bf16x2(r[4], r[5]),
                           pack_bf16x2(r[6], r[7]));
        o4[1] = make_uint4(pack_bf16x2(r[8], r[9]), pack_bf16x2(r[10], r[11]), pack_bf16x2(r[12], r[13]),
                           pack_bf16x2(r[14], r[15]));
    }
};

template <int N, bool DGRAD>
__global__ void __launch_bounds__(TC_THREADS) k_conv_rows(const __nv_bfloat16* src, const __nv_bfloat16* wmat,
                                                           const float* bias, const __nv_bfloat16* mask_src,
                                                           __nv_bfloat16* out, Vol g, int Cs, int Kpad, int relu) {
    extern __shared__ __align__(1024) uint8_t smem[];
    ConvRows<N, DGRAD> op;
    op.src = src;
    op.wmat = wmat;
    op.bias = bias;
    op.mask_src = mask_src;
    op.out = out;
    op.g = g;
    op.Cs = Cs;
    op.K = 27 * Cs;
    op.Kpad = Kpad;
    op.chunks = Kpad / TC_KC;
    op.m0 = blockIdx.x * TC_M;
    op.relu = relu;
    op.setup();
    tc::tile_gemm<ConvRows<N, DGRAD>, N>(op, smem);
}

// ---- weight gradient: A = x at tap offsets (MN-major over (tap, ci)), B = dy (MN-major over co) ---
template <int N>
struct ConvWgrad {
    static constexpr bool A_MN = true, B_MN = true;
    const __nv_bfloat16* x;   // [V][Cin]
    const __nv_bfloat16* dy;  // [V][N]
    float* dw;                // [27 * Cin][N], accumulated
    Vol g;
    int Cin, Mrows, m0, chunk0, chunks;
    __device__ void gather_a(uint8_t* st, int chunk) const {
        const int kk = threadIdx.x & (TC_KC - 1);
        const int v = (chunk0 + chunk) * TC_KC + kk;
        int b = 0, z = 0, y = 0, xx = 0;
        const bool valid = v < g.voxels();
        if (valid) decode(g, v, b, z, y, xx);
        for (int mv = threadIdx.x / TC_KC; mv < TC_M / 8; mv += TC_THREADS / TC_KC) {
            const int m = m0 + mv * 8;
            uint4 val = make_uint4(0, 0, 0, 0);
            if (valid && m < Mrows) {
                const int tap = m / Cin, c = m - tap * Cin;
                const int nb = tap_neighbour(g, b, z, y, xx, tap, 1);
                if (nb >= 0) val = __ldg(reinterpret_cast<const uint4*>(x + (i64)nb * Cin + c));
            }
            *reinterpret_cast<uint4*>(st + tc::mnmajor_off(mv, kk)) = val;
        }
    }
    __device__ void gather_b(uint8_t* st, int chunk) const {
        const int kk = threadIdx.x & (TC_KC - 1);
        const int v = (chunk0 + chunk) * TC_KC + kk;
        const bool valid = v < g.voxels();
        for (int nv = threadIdx.x / TC_KC; nv < N / 8; nv += TC_THREADS / TC_KC) {
            uint4 val = make_uint4(0, 0, 0, 0);
            if (valid) val = __ldg(reinterpret_cast<const uint4*>(dy + (i64)v * N + nv * 8));
            *reinterpret_cast<uint4*>(st + tc::mnmajor_off(nv, kk)) = val;
        }
    }
    __device__ void epilogue(int row, const float* acc, int col0) const {
        const int m = m0 + row;
        if (m >= Mrows) return;
#pragma unroll
        for (int q = 0; q < 16; ++q) atomicAdd(dw + (i64)m * N + col0 + q, acc[q]);
    }
};

template <int N>
__global__ void __launch_bounds__(TC_THREADS) k_conv_wgrad(const __nv_bfloat16* x, const __nv_bfloat16* dy,
                                                            float* dw, Vol g, int Cin, int chunks_per_block) {
    extern __shared__ __align__(1024) uint8_t smem[];
    ConvWgrad<N> op;
    op.x = x;
    op.dy = dy;
    op.dw = dw;
    op.g = g;
    op.Cin = Cin;
    op.Mrows = 27 * Cin;
    op.m0 = blockIdx.x * TC_M;
    const int total_chunks = (g.B * g.D * g.H * g.W + TC_KC - 1) / TC_KC;
    op.chunk0 = blockIdx.y * chunks_per_block;
    op.chunks = max(0, min(chunks_per_block, total_chunks - op.chunk0));
    tc::tile_gemm<ConvWgrad<N>, N>(op, smem);
}

// ---- elementwise pieces of the network ------------------------------------------------------------
constexpr int EW = 256;

// master weights [27 * Cin][Cout] (fp32) -> forward matrix wf[Cout][Kpad] and data-grad matrix
// wd[Cin][Kpad2] (bf16, zero-padded along K to multiples of 64)
__global__ void k_arrange_weights(const float* __restrict__ w, __nv_bfloat16* __restrict__ wf,
                                  __nv_bfloat16* __restrict__ wd, int Cin, int Cout, int Kpad, int Kpad2) {
    const int total = Cout * Kpad + (wd ? Cin * Kpad2 : 0);
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
        if (t < Cout * Kpad) {
            const int co = t / Kpad, k = t % Kpad;
            wf[t] = __float2bfloat16_rn(k < 27 * Cin ? w[(i64)k * Cout + co] : 0.0f);
        } else {
            const int u = t - Cout * Kpad;
            const int ci = u / Kpad2, k = u % Kpad2;
            float val = 0.0f;
            if (k < 27 * Cout) {
                const int tap = k / Cout, co = k % Cout;
                val = w[((i64)tap * Cin + ci) * Cout + co];
            }
            wd[u] = __float2bfloat16_rn(val);
        }
    }
}

// Eight BF16 channels (16 bytes) to and from FP32.
__device__ __forceinline__ void unpack8(const uint4 u, float* f) {
    const __nv_bfloat162* h = reinterpret_cast<const __nv_bfloat162*>(&u);
#pragma unroll
    for (int e = 0; e < 4; ++e) {
        const float2 t = __bfloat1622float2(h[e]);
        f[2 * e] = t.x;
        f[2 * e + 1] = t.y;
    }
}
__device__ __forceinline__ uint4 pack8(const float* f) {
    return make_uint4(pack_bf16x2(f[0], f[1]), pack_bf16x2(f[2], f[3]), pack_bf16x2(f[4], f[5]),
                      pack_bf16x2(f[6], f[7]));
}
__device__ __forceinline__ void decode_vox(i64 v, int D, int H, int W, int& b, int& z, int& y, int& x) {
    x = (int)(v % W);
    v /= W;
    y = (int)(v % H);
    v /= H;
    z = (int)(v % D);
    b = (int)(v / D);
}

// 2x2x2 average pooling of a channels-last volume (D, H, W even); one thread per coarse voxel and
// group of 8 channels
__global__ void k_avgpool2(const __nv_bfloat16* __restrict__ x, __nv_bfloat16* __restrict__ y, Vol fine, int C) {
    const int G = C / 8, cD = fine.D / 2, cH = fine.H / 2, cW = fine.W / 2;
    const i64 total = (i64)fine.B * cD * cH * cW * G;
    for (i64 t = (i64)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (i64)gridDim.x * blockDim.x) {
        const int grp = (int)(t % G);
        int b, Z, Y, X;
        decode_vox(t / G, cD, cH, cW, b, Z, Y, X);
        float s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        for (int d = 0; d < 8; ++d) {
            const int z = 2 * Z + (d >> 2), y2 = 2 * Y + ((d >> 1) & 1), x2 = 2 * X + (d & 1);
            float f[8];
            unpack8(__ldg(reinterpret_cast<const uint4*>(x + ((((i64)b * fine.D + z) * fine.H + y2) * fine.W + x2) * C) + grp), f);
#pragma unroll
            for (int e = 0; e < 8; ++e) s[e] += f[e];
        }
#pragma unroll
        for (int e = 0; e < 8; ++e) s[e] *= 0.125f;
        reinterpret_cast<uint4*>(y)[t] = pack8(s);
    }
}

// nearest 2x upsampling of `coarse` (C1 channels) written into channels [0, C1) of `out`, and a copy
// of `skip` (C2 channels) into channels [C1, C1 + C2): the decoder's concatenated input. One thread
// per fine voxel and group of 8 channels.
__global__ void k_upsample_concat(const __nv_bfloat16* __restrict__ coarse, const __nv_bfloat16* __restrict__ skip,
                                  __nv_bfloat16* __restrict__ out, Vol fine, int C1, int C2) {
    const int G1 = C1 / 8, G = (C1 + C2) / 8;
    const i64 total = (i64)fine.B * fine.D * fine.H * fine.W * G;
    for (i64 t = (i64)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (i64)gridDim.x * blockDim.x) {
        const int grp = (int)(t % G);
        const i64 v = t / G;
        uint4 val;
        if (grp < G1) {
            int b, z, y, x;
            decode_vox(v, fine.D, fine.H, fine.W, b, z, y, x);
            const i64 cv = (((i64)b * (fine.D / 2) + z / 2) * (fine.H / 2) + y / 2) * (fine.W / 2) + x / 2;
            val = __ldg(reinterpret_cast<const uint4*>(coarse + cv * C1) + grp);
        } else {
            val = __ldg(reinterpret_cast<const uint4*>(skip + v * C2) + (grp - G1));
        }
        reinterpret_cast<uint4*>(out)[t] = val;
    }
}

// backward of k_upsample_concat: d coarse = sum over the 8 children (into FP32 then BF16), d skip +=
// the copied channels (added to an existing gradient, as the skip tensor also feeds the encoder)
__global__ void k_upsample_concat_backward(const __nv_bfloat16* __restrict__ dout, __nv_bfloat16* __restrict__ dcoarse,
                                           __nv_bfloat16* __restrict__ dskip, Vol fine, int C1, int C2) {
    const int C = C1 + C2, G1 = C1 / 8, G2 = C2 / 8, cD = fine.D / 2, cH = fine.H / 2, cW = fine.W / 2;
    const i64 coarse_total = (i64)fine.B * cD * cH * cW * G1;
    const i64 skip_total = (i64)fine.B * fine.D * fine.H * fine.W * G2;
    for (i64 t = (i64)blockIdx.x * blockDim.x + threadIdx.x; t < coarse_total + skip_total;
         t += (i64)gridDim.x * blockDim.x) {
        if (t < coarse_total) {
            const int grp = (int)(t % G1);
            int b, Z, Y, X;
            decode_vox(t / G1, cD, cH, cW, b, Z, Y, X);
            float s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
            for (int d = 0; d < 8; ++d) {
                const int z = 2 * Z + (d >> 2), y = 2 * Y + ((d >> 1) & 1), x = 2 * X + (d & 1);
                float f[8];
                unpack8(__ldg(reinterpret_cast<const uint4*>(dout + ((((i64)b * fine.D + z) * fine.H + y) * fine.W + x) * C) + grp), f);
#pragma unroll
                for (int e = 0; e < 8; ++e) s[e] += f[e];
            }
            reinterpret_cast<uint4*>(dcoarse)[t] = pack8(s);
        } else {
            const i64 u = t - coarse_total;
            const int grp = (int)(u % G2);
            const i64 v = u / G2;
            float a[8], f[8];
            unpack8(reinterpret_cast<const uint4*>(dskip)[u], a);
            unpack8(__ldg(reinterpret_cast<const uint4*>(dout + v * C + C1) + grp), f);
#pragma unroll
            for (int e = 0; e < 8; ++e) a[e] += f[e];
            reinterpret_cast<uint4*>(dskip)[u] = pack8(a);
        }
    }
}

// backward of 2x2x2 average pooling: each fine voxel gets 1/8 of its parent's gradient, added to an
// existing gradient and masked by the ReLU of the pooled activation's producer (x > 0)
__global__ void k_avgpool2_backward(const __nv_bfloat16* __restrict__ dy, const __nv_bfloat16* __restrict__ x,
                                    __nv_bfloat16* __restrict__ dx, Vol fine, int C) {
    const int G = C / 8;
    const i64 total = (i64)fine.B * fine.D * fine.H * fine.W * G;
    for (i64 t = (i64)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (i64)gridDim.x * blockDim.x) {
        const int grp = (int)(t % G);
        int b, z, y, xx;
        decode_vox(t / G, fine.D, fine.H, fine.W, b, z, y, xx);
        const i64 cv = (((i64)b * (fine.D / 2) + z / 2) * (fine.H / 2) + y / 2) * (fine.W / 2) + xx / 2;
        float a[8], p[8], xv[8];
        unpack8(reinterpret_cast<const uint4*>(dx)[t], a);
        unpack8(__ldg(reinterpret_cast<const uint4*>(dy + cv * C) + grp), p);
        unpack8(__ldg(reinterpret_cast<const uint4*>(x) + t), xv);
#pragma unroll
        for (int e = 0; e < 8; ++e) a[e] = xv[e] > 0.0f ? a[e] + 0.125f * p[e] : 0.0f;
        reinterpret_cast<uint4*>(dx)[t] = pack8(a);
    }
}

// 1x1x1 head (C = 16 channels): out[v] = bias + sum_c h[v][c] w[c]
__global__ void k_head_forward(const __nv_bfloat16* __restrict__ h, const float* __restrict__ w, const float* bias,
                               float* __restrict__ out, int V, int C) {
    float wr[16];
#pragma unroll
    for (int c = 0; c < 16; ++c) wr[c] = c < C ? __ldg(w + c) : 0.0f;
    const float b0 = __ldg(bias);
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
        const uint4* hv = reinterpret_cast<const uint4*>(h + (i64)v * C);
        float f[16];
        unpack8(__ldg(hv), f);
        unpack8(__ldg(hv + 1), f + 8);
        float s = b0;
#pragma unroll
        for (int c = 0; c < 16; ++c) s += f[c] * wr[c];
        out[v] = s;
    }
}

// dh[v][c] = dout[v] * w[c] masked by (h > 0); dw[c] += sum_v dout[v] h[v][c]; db += sum dout (C = 16)
__global__ void k_head_backward(const __nv_bfloat16* __restrict__ h, const float* __restrict__ w,
                                const float* __restrict__ dout, __nv_bfloat16* __restrict__ dh, float* dw, float* db,
                                int V, int C) {
    __shared__ float s_dw[17];
    if (threadIdx.x < 17) s_dw[threadIdx.x] = 0.0f;
    __syncthreads();
    float wr[16], ldw[16];
#pragma unroll
    for (int c = 0; c < 16; ++c) {
        wr[c] = __ldg(w + c);
        ldw[c] = 0.0f;
    }
    float ldb = 0.0f;
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
        const float g = __ldg(dout + v);
        ldb += g;
        const uint4* hv = reinterpret_cast<const uint4*>(h + (i64)v * C);
        float f[16], o[16];
        unpack8(__ldg(hv), f);
        unpack8(__ldg(hv + 1), f + 8);
#pragma unroll
        for (int c = 0; c < 16; ++c) {
            ldw[c] += g * f[c];
            o[c] = f[c] > 0.0f ? g * wr[c] : 0.0f;
        }
        uint4* dv = reinterpret_cast<uint4*>(dh + (i64)v * C);
        dv[0] = pack8(o);
        dv[1] = pack8(o + 8);
    }
#pragma unroll
    for (int c = 0; c < 16; ++c) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) ldw[c] += __shfl_xor_sync(0xffffffffu, ldw[c], o);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) ldb += __shfl_xor_sync(0xffffffffu, ldb, o);
    if ((threadIdx.x & 31) == 0) {
#pragma unroll
        for (int c = 0; c < 16; ++c) atomicAdd(&s_dw[c], ldw[c]);
        atomicAdd(&s_dw[16], ldb);
    }
    __syncthreads();
    if (threadIdx.x < 16) atomicAdd(dw + threadIdx.x, s_dw[threadIdx.x]);
    if (threadIdx.x == 16) atomicAdd(db, s_dw[16]);
}

// bias gradient of a conv: db[co] += sum_v dy[v][co]. Thread t of a block sums channel group
// t % G (8 channels) over voxels t / G, t / G + stride, ... (blockDim is a multiple of G).
__global__ void k_bias_grad(const __nv_bfloat16* __restrict__ dy, float* db, int V, int C) {
    __shared__ float s[256];
    const int G = C / 8;
    for (int c = threadIdx.x; c < C; c += blockDim.x) s[c] = 0.0f;
    __syncthreads();
    const int per_block = blockDim.x / G;
    const int grp = threadIdx.x % G, slot = threadIdx.x / G;
    float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    if (slot < per_block)
        for (i64 v = (i64)blockIdx.x * per_block + slot; v < V; v += (i64)gridDim.x * per_block) {
            float f[8];
            unpack8(__ldg(reinterpret_cast<const uint4*>(dy + v * C) + grp), f);
#pragma unroll
            for (int e = 0; e < 8; ++e) acc[e] += f[e];
        }
    if (slot < per_block)
#pragma unroll
        for (int e = 0; e < 8; ++e) atomicAdd(&s[grp * 8 + e], acc[e]);
    __syncthreads();
    for (int c = threadIdx.x; c < C; c += blockDim.x) atomicAdd(db + c, s[c]);
}

// Adam step (Kingma & Ba) on FP32 master parameters
__global__ void k_adam(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, i64 n, float lr, float beta1, float beta2, float eps, float bc1,
                       float bc2) {
    for (i64 t = (i64)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (i64)gridDim.x * blockDim.x) {
        const float gt = g[t];
        const float mt = beta1 * m[t] + (1.0f - beta1) * gt;
        const float vt = beta2 * v[t] + (1.0f - beta2) * gt * gt;
        m[t] = mt;
        v[t] = vt;
        p[t] -= lr * (mt / bc1) / (sqrtf(vt / bc2) + eps);
    }
}

// Network input from the solver's finest level: channels (b * scale_b, fluid, solid, p * inv_s,
// 0, 0, 0, 0) of grid cell (oi + z, oj + y, ok + x) into voxel (z, y, x) of batch slot `slot` of a
// [B][D][H][W][8] volume; cells outside the grid are 0.
__global__ void k_pack_input(const float* __restrict__ b, const uint8_t* __restrict__ op0,
                             const uint8_t* __restrict__ solid, const float* __restrict__ p, float scale_b,
                             float inv_s, int nx, int ny, int nz, int oi, int oj, int ok, __nv_bfloat16* __restrict__ x0,
                             int slot, int D, int H, int W) {
    const i64 V = (i64)D * H * W;
    for (i64 v = (i64)blockIdx.x * blockDim.x + threadIdx.x; v < V; v += (i64)gridDim.x * blockDim.x) {
        const int xx = (int)(v % W), y = (int)((v / W) % H), z = (int)(v / ((i64)W * H));
        const int i = oi + z, j = oj + y, k = ok + xx;
        float c0 = 0.0f, c1 = 0.0f, c2 = 0.0f, c3 = 0.0f;
        if (i >= 0 && i < nx && j >= 0 && j < ny && k >= 0 && k < nz) {
            const i64 c = ((i64)i * ny + j) * nz + k;
            const bool fl = (__ldg(op0 + c) & 64u) != 0u;
            c0 = fl ? __ldg(b + c) * scale_b : 0.0f;
            c1 = fl ? 1.0f : 0.0f;
            c2 = (solid && __ldg(solid + c)) ? 1.0f : 0.0f;
            c3 = fl ? __ldg(p + c) * inv_s : 0.0f;
        }
        uint4* dst = reinterpret_cast<uint4*>(x0 + ((i64)slot * V + v) * 8);
        *dst = make_uint4(pack_bf16x2(c0, c1), pack_bf16x2(c2, c3), 0u, 0u);
    }
}

// Training target and loss weight of one batch slot: t = (p - p_prev) * inv_s and m = 1 at fluid
// cells (the network predicts the change of the pressure since the previous step).
__global__ void k_pack_target(const float* __restrict__ p, const float* __restrict__ p_prev,
                              const uint8_t* __restrict__ op0, float inv_s, int nx, int ny, int nz, int oi, int oj,
                              int ok, float* __restrict__ t, float* __restrict__ m, int slot, int D, int H, int W) {
    const i64 V = (i64)D * H * W;
    for (i64 v = (i64)blockIdx.x * blockDim.x + threadIdx.x; v < V; v += (i64)gridDim.x * blockDim.x) {
        const int xx = (int)(v % W), y = (int)((v / W) % H), z = (int)(v / ((i64)W * H));
        const int i = oi + z, j = oj + y, k = ok + xx;
        float tv = 0.0f, mv = 0.0f;
        if (i >= 0 && i < nx && j >= 0 && j < ny && k >= 0 && k < nz) {
            const i64 c = ((i64)i * ny + j) * nz + k;
            if (__ldg(op0 + c) & 64u) {
                tv = (__ldg(p + c) - __ldg(p_prev + c)) * inv_s;
                mv = 1.0f;
            }
        }
        t[(i64)slot * V + v] = tv;
        m[(i64)slot * V + v] = mv;
    }
}

// Network output of voxel (i, j, k) (batch slot 0) back to the grid: p = p_prev + out * s at fluid
// cells (in FP32, so the previous pressure keeps its precision), 0 elsewhere.
__global__ void k_unpack_output(const float* __restrict__ out, const float* __restrict__ p_prev,
                                const uint8_t* __restrict__ op0, float s, float* __restrict__ p, int nx, int ny, int nz,
                                int D, int H, int W) {
    const i64 C = (i64)nx * ny * nz;
    for (i64 c = (i64)blockIdx.x * blockDim.x + threadIdx.x; c < C; c += (i64)gridDim.x * blockDim.x) {
        const int k = (int)(c % nz), j = (int)((c / nz) % ny), i = (int)(c / ((i64)ny * nz));
        const bool fl = (__ldg(op0 + c) & 64u) != 0u;
        p[c] = fl ? __ldg(p_prev + c) + __ldg(out + ((i64)i * H + j) * W + k) * s : 0.0f;
    }
}

// Masked mean squared error: dout = 2 m (out - t) / count, loss += sum m (out - t)^2 / count.
__global__ void k_mse(const float* __restrict__ out, const float* __restrict__ t, const float* __restrict__ m,
                      float* __restrict__ dout, float* loss, i64 n, float inv_count) {
    float acc = 0.0f;
    for (i64 v = (i64)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (i64)gridDim.x * blockDim.x) {
        const float d = (out[v] - t[v]) * m[v];
        dout[v] = 2.0f * d * inv_count;
        acc += d * d * inv_count;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(loss, acc);
}

}  // namespace conv
}  // namespace clb
