// Bottom of the W-cycle in one launch.
//
// With L levels the second-coarsest level A = L-2 is visited 2^(L-2) times per W-cycle, and each
// visit runs (multigrid.py:53-187) pre-smoothing of A, restriction to the coarsest level B, two
// coarse solves of B (multigrid.py:127-170, 2 + 64 red-black iterations each), prolongation and
// post-smoothing of A: about 280 dependent red-black phases on a few thousand cells. As separate
// launches these are bound by launch latency; here one block of 512 threads runs the whole visit
// with both levels in shared memory and block barriers between phases.
//
// Each thread owns a fixed set of A cells and B cells of either colour (colour slots, below); the
// cell index, diagonal and delta^2 * b of each owned cell stay in registers across all sweeps (the
// neighbour weights of A cells are read from shared memory, those of B cells are registers too). The
// update formula and every summation order are those of multigrid.cl (rbgs_step, restrict_residual,
// prolongate), so the result is identical to the launch-per-kernel W-cycle.
#pragma once
#include "multigrid.cuh"

namespace clb {

constexpr int BOTTOM_THREADS = 512;
constexpr int BOTTOM_MAX_A = 8;  // A slots of each colour per thread
constexpr int BOTTOM_MAX_B = 4;  // B slots of each colour per B thread

static inline size_t bottom_smem_bytes(int ca, int cb) {
    // A: p, b, op(float4); B: p, op(float4); the fluid-cell lists of both colours of both levels and
    // their four counts; each region padded to 16 bytes
    auto pad = [](size_t x) { return (x + 15) & ~(size_t)15; };
    return pad((size_t)ca * 4) * 2 + (size_t)ca * 16 + pad((size_t)cb * 4) + (size_t)cb * 16 +
           pad((size_t)(ca + cb + 8) * 4);
}

// Cells of one colour are numbered by slots: the interior rows (i, j) in index order, ceil(mz / 2)
// slots per row, slot s of a row being its (s+1)-th cell of the colour, k = k0 + 2 s with k0 the
// row's first such k (1 or 2). With an odd interior extent along k the last slot of every other row
// is empty. A colour phase updates cells of one colour only, and those are independent of each other,
// so any assignment of cells to threads gives the same result; numbering by colour keeps every lane
// of a warp busy in every phase.
__host__ __device__ __forceinline__ int colour_slots(int nx, int ny, int nz) {
    return (nx - 2) * (ny - 2) * ((nz - 1) / 2);
}

// smem / grid index of slot r of colour `colour`, or -1 for an empty slot or r past the last slot
__device__ __forceinline__ int colour_cell(int r, int colour, int nx, int ny, int nz) {
    const int half = (nz - 1) / 2, my = ny - 2;
    const int row = r / half, s = r - row * half;
    const int i = 1 + row / my, j = 1 + row % my;
    const int k = 1 + 2 * s + ((i + j + 1 + colour) & 1);
    if (i > nx - 2 || k > nz - 2) return -1;
    return (i * ny + j) * nz + k;
}

// Constants of one owned cell of the second-coarsest level: smem index, diagonal (<= 0: not updated;
// -1 marks cells that are not fluid or slots without a cell) and delta^2 * b.
struct OwnedCell {
    int c;
    float d;
    float d2b;
};

// Owned coarsest-level cell with its neighbour weights in registers (constant for the whole visit).
struct OwnedCellW {
    int c;
    float d, d2b;
    float wxp, wxm, wyp, wym, wzp, wzm;
};

__device__ __forceinline__ void relax_w(const OwnedCellW& o, float* sp, int sx, int sy) {
    const int c = o.c;
    const float ws = o.wxp * sp[c + sx] + o.wxm * sp[c - sx] + o.wyp * sp[c + sy] + o.wym * sp[c - sy] +
                     o.wzp * sp[c + 1] + o.wzm * sp[c - 1];
    sp[c] = (ws - o.d2b) / o.d;
}

// One red-black update of an owned cell (multigrid.cl:225-229), p and weights in shared memory.
__device__ __forceinline__ void relax(const OwnedCell& o, float* sp, const float4* so, int sx, int sy) {
    const int c = o.c;
    const float4 self = so[c];
    const float ws = self.y * sp[c + sx] + so[c - sx].y * sp[c - sx] + self.z * sp[c + sy] + so[c - sy].z * sp[c - sy] +
                     self.w * sp[c + 1] + so[c - 1].w * sp[c - 1];
    sp[c] = (ws - o.d2b) / o.d;
}

// The coarsest level B runs on BOTTOM_BTHREADS threads (8 warps) that synchronise with a named
// barrier; each owns slots r = thread, thread + 256, ... of both colours, so every thread updates
// its cells of one colour per phase.
constexpr int BOTTOM_BTHREADS = 256;

__device__ __forceinline__ void bar_b() { asm volatile("bar.sync 1, 256;" ::: "memory"); }

// Shared-memory arrays of a bottom visit: A's p, b and operator (float4, diagonal -1 where not
// fluid), B's p and operator, and the fluid cells of each colour of both levels; each region padded to
// 16 bytes (bottom_smem_bytes).
struct BottomSmem {
    float* spa;
    float* sba;
    float4* soa;
    float* spb;
    float4* sob;
    int* count;   // fluid cells: A colour 0, A colour 1, B colour 0, B colour 1
    int* list_a;  // two lists of CA / 2 + 1 entries
    int* list_b;  // two lists of CB / 2 + 1 entries
};

__device__ __forceinline__ BottomSmem bottom_smem(unsigned char* base, int CA, int CB) {
    auto pad = [](int x) { return (x + 3) & ~3; };  // in floats
    BottomSmem S;
    S.spa = reinterpret_cast<float*>(base);
    S.sba = S.spa + pad(CA);
    S.soa = reinterpret_cast<float4*>(S.sba + pad(CA));
    S.spb = reinterpret_cast<float*>(S.soa + CA);
    S.sob = reinterpret_cast<float4*>(S.spb + pad(CB));
    S.count = reinterpret_cast<int*>(S.sob + CB);
    S.list_a = S.count + 4;
    S.list_b = S.list_a + 2 * (CA / 2 + 1);
    return S;
}

// Lists the fluid interior cells of each colour of both levels (after the operators are staged and
// the block has synchronised). Their order is arbitrary -- cells of one colour are independent -- and
// the threads take them in turn, so a warp's owned cells are fluid but for the last ones and the empty
// slots beyond the count are empty in whole warps: a phase costs what the fluid needs, not what the
// level's size does.
__device__ __forceinline__ void bottom_lists(const BottomSmem& S, int anx, int any, int anz, int bnx, int bny,
                                             int bnz) {
    const int CA = anx * any * anz, CB = bnx * bny * bnz;
    const int la = CA / 2 + 1, lb = CB / 2 + 1;
    if (threadIdx.x < 4) S.count[threadIdx.x] = 0;
    __syncthreads();
    const int sa = colour_slots(anx, any, anz), sb = colour_slots(bnx, bny, bnz);
    for (int colour = 0; colour < 2; ++colour) {
        for (int r = threadIdx.x; r < sa; r += BOTTOM_THREADS) {
            const int c = colour_cell(r, colour, anx, any, anz);
            if (c >= 0 && S.soa[c].x >= 0.0f) S.list_a[colour * la + atomicAdd(S.count + colour, 1)] = c;
        }
        for (int r = threadIdx.x; r < sb; r += BOTTOM_THREADS) {
            const int c = colour_cell(r, colour, bnx, bny, bnz);
            if (c >= 0 && S.sob[c].x >= 0.0f) S.list_b[colour * lb + atomicAdd(S.count + 2 + colour, 1)] = c;
        }
    }
    __syncthreads();
}

// Staging of the operators of both levels and, when pa / ba are given, of A's p and b (FP16 levels
// are converted to FP32). Four cells per thread and round, all loads issued before the stores.
template <bool H>
__device__ __forceinline__ void bottom_stage(const BottomSmem& S, const float* __restrict__ pa,
                                             const float* __restrict__ ba, const float4* __restrict__ opa,
                                             const uint8_t* __restrict__ ma, int CA, const float4* __restrict__ opb,
                                             const uint8_t* __restrict__ mb, int CB) {
    auto ld = [&](const float* a, int c) -> float {
        return H ? ldh(reinterpret_cast<const __half*>(a), c) : a[c];
    };
    auto ld4 = [&](const float4* a, int c) -> float4 {
        return H ? ld_h4(reinterpret_cast<const Half4*>(a), c) : a[c];
    };
    constexpr int U = 4;
    for (int c0 = threadIdx.x; c0 < CA; c0 += U * BOTTOM_THREADS) {
        float pv[U], bv[U];
        float4 ov[U];
        uint8_t mv[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int c = c0 + u * BOTTOM_THREADS;
            if (c < CA) {
                pv[u] = pa ? ld(pa, c) : 0.0f;
                bv[u] = ba ? ld(ba, c) : 0.0f;
                ov[u] = ld4(opa, c);
                mv[u] = ma[c];
            }
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int c = c0 + u * BOTTOM_THREADS;
            if (c < CA) {
                if (pa) S.spa[c] = pv[u];
                if (ba) S.sba[c] = bv[u];
                float4 o = ov[u];
                if (!mv[u]) o.x = -1.0f;
                S.soa[c] = o;
            }
        }
    }
    for (int c0 = threadIdx.x; c0 < CB; c0 += U * BOTTOM_THREADS) {
        float4 ov[U];
        uint8_t mv[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int c = c0 + u * BOTTOM_THREADS;
            if (c < CB) {
                ov[u] = ld4(opb, c);
                mv[u] = mb[c];
            }
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int c = c0 + u * BOTTOM_THREADS;
            if (c < CB) {
                float4 o = ov[u];
                if (!mv[u]) o.x = -1.0f;
                S.sob[c] = o;
            }
        }
    }
}

// The cells a thread owns in a bottom visit: A cells of each colour (index, diagonal, delta^2 * b) and
// B cells of each colour with their neighbour weights. Index, diagonal and weights depend on the
// operators only, so a launch that visits A several times sets them once (bottom_cells); A's delta^2 * b
// is set again whenever A's right-hand side changes (bottom_rhs).
template <int KA, int KB>
struct BottomCells {
    OwnedCell A[2][KA];   // [colour][m]: the thread's fluid cells (bottom_lists)
    OwnedCellW B[2][KB];  // [colour][m]
};

// After the lists are built and the block has synchronised.
template <int KA, int KB>
__device__ __forceinline__ void bottom_cells(const BottomSmem& S, BottomCells<KA, KB>& R, int anx, int any, int anz,
                                             int bnx, int bny, int bnz) {
    const int la = (anx * any * anz) / 2 + 1, lb = (bnx * bny * bnz) / 2 + 1;
    const int bsx = bny * bnz, bsy = bnz;
#pragma unroll
    for (int colour = 0; colour < 2; ++colour)
#pragma unroll
        for (int m = 0; m < KA; ++m) {
            const int r = threadIdx.x + m * BOTTOM_THREADS;
            const int c = r < S.count[colour] ? S.list_a[colour * la + r] : -1;
            OwnedCell& o = R.A[colour][m];
            o.c = c < 0 ? 0 : c;
            o.d = c < 0 ? -1.0f : S.soa[c].x;  // fluid: >= 0
            o.d2b = 0.0f;
        }
    const bool btile = threadIdx.x < BOTTOM_BTHREADS;
#pragma unroll
    for (int colour = 0; colour < 2; ++colour)
#pragma unroll
        for (int m = 0; m < KB; ++m) {
            const int r = threadIdx.x + m * BOTTOM_BTHREADS;
            const int c = btile && r < S.count[2 + colour] ? S.list_b[colour * lb + r] : -1;
            OwnedCellW& o = R.B[colour][m];
            o.d2b = 0.0f;
            o.c = 0;
            o.d = -1.0f;
            o.wxp = o.wxm = o.wyp = o.wym = o.wzp = o.wzm = 0.0f;
            if (c >= 0) {
                const float4 self = S.sob[c];
                o.c = c;
                o.d = self.x;
                o.wxp = self.y;
                o.wyp = self.z;
                o.wzp = self.w;
                o.wxm = S.sob[c - bsx].y;
                o.wym = S.sob[c - bsy].z;
                o.wzm = S.sob[c - 1].w;
            }
        }
}

// A's delta^2 * b of the owned cells, after A's right-hand side is in shared memory and visible.
template <int KA, int KB>
__device__ __forceinline__ void bottom_rhs(const BottomSmem& S, BottomCells<KA, KB>& R, float d2) {
#pragma unroll
    for (int colour = 0; colour < 2; ++colour)
#pragma unroll
        for (int m = 0; m < KA; ++m) {
            OwnedCell& o = R.A[colour][m];
            o.d2b = o.d < 0.0f ? 0.0f : d2 * S.sba[o.c];
        }
}

// One visit of A from staged shared memory with the owned cells set (bottom_cells, bottom_rhs):
// pre-smoothing of A, restriction into B (B's p zeroed, multigrid.cl:114), the two coarse solves of B,
// prolongation, post-smoothing of A. bb (nullable): B's right-hand side is stored there (FP16 when H).
// KA: A slots of each colour per thread (of BOTTOM_THREADS); KB: B slots of each colour per B thread.
template <int KA, int KB, bool H>
__device__ __forceinline__ void bottom_core(const BottomSmem& S, BottomCells<KA, KB>& R, int anx, int any, int anz,
                                            int bnx, int bny, int bnz, float d2, float inv_delta2, int pre, int post,
                                            int coarse_iters, float* __restrict__ bb, int b_solves = 2,
                                            float w = 1.0f) {
    float* spa = S.spa;
    const float* sba = S.sba;
    const float4* soa = S.soa;
    float* spb = S.spb;
    const int CB = bnx * bny * bnz;
    auto st = [&](float* a, int c, float v) {
        if (H) reinterpret_cast<__half*>(a)[c] = __float2half_rn(v);
        else a[c] = v;
    };
    const int asx = any * anz, asy = anz, bsx = bny * bnz, bsy = bnz;
    const int lb = CB / 2 + 1;
    OwnedCell (&A)[2][KA] = R.A;
    OwnedCellW (&B)[2][KB] = R.B;
    const bool btile = threadIdx.x < BOTTOM_BTHREADS;

    auto smooth_a = [&](int iterations) {
        for (int it = 0; it < iterations; ++it)
#pragma unroll
            for (int colour = 0; colour < 2; ++colour) {
#pragma unroll
                for (int m = 0; m < KA; ++m)
                    if (A[colour][m].d > 0.0f) relax(A[colour][m], spa, soa, asx, asy);
                __syncthreads();
            }
    };

    __syncthreads();  // staging and the caller's writes to shared memory are complete
    smooth_a(pre);
    // restriction of the residual (multigrid.cl:90-180, right-hand-side part) of B's fluid cells (both
    // lists), one thread per coarse cell: the residuals of the eight children l = 4 di + 2 dj + dk are
    // formed independently (interior fluid children only) and added in that order, as the reference's
    // loop over di, dj, dk adds them. The sums go to B's p (free until the coarse solves), from which B's
    // owners take them.
    {
        const int n0 = S.count[2], nb = n0 + S.count[3];
        for (int g = threadIdx.x; g < nb; g += BOTTOM_THREADS) {
            const int cb = g < n0 ? S.list_b[g] : S.list_b[lb + g - n0];
            const int I = cb / bsx, J = (cb / bsy) % bny, K = cb % bnz;
            float r[8];
            bool present[8];
#pragma unroll
            for (int l = 0; l < 8; ++l) {
                const int i = 2 * I - 1 + (l >> 2), j = 2 * J - 1 + ((l >> 1) & 1), k = 2 * K - 1 + (l & 1);
                r[l] = 0.0f;
                present[l] = false;
                if (interior(i, j, k, anx, any, anz)) {
                    const int f = (i * any + j) * anz + k;
                    const float4 o = soa[f];
                    if (o.x >= 0.0f) {
                        const float ws = o.y * spa[f + asx] + soa[f - asx].y * spa[f - asx] + o.z * spa[f + asy] +
                                         soa[f - asy].z * spa[f - asy] + o.w * spa[f + 1] + soa[f - 1].w * spa[f - 1];
                        r[l] = sba[f] - (ws - o.x * spa[f]) * inv_delta2;
                        present[l] = true;
                    }
                }
            }
            float rhs = 0.0f;
#pragma unroll
            for (int l = 0; l < 8; ++l)
                if (present[l]) rhs += r[l];
            spb[cb] = rhs;
        }
    }
    __syncthreads();
    float bvals[2][KB];
#pragma unroll
    for (int colour = 0; colour < 2; ++colour)
#pragma unroll
        for (int m = 0; m < KB; ++m) {
            // a fluid cell (slots without a cell and air cells hold -1)
            const float rhs = B[colour][m].d >= 0.0f ? spb[B[colour][m].c] : 0.0f;
            bvals[colour][m] = rhs;
            B[colour][m].d2b = d2 * rhs;
        }
    __syncthreads();
    for (int c = threadIdx.x; c < CB; c += BOTTOM_THREADS) spb[c] = 0.0f;  // multigrid.cl:114
    __syncthreads();
    if (btile) {
        // two coarse solves of the W (multigrid.py:127-170; b_solves: one when the coarsest level is
        // visited once), pre + coarse_iters iterations each
        const int iterations = b_solves * (pre + coarse_iters);
        for (int it = 0; it < iterations; ++it)
#pragma unroll
            for (int colour = 0; colour < 2; ++colour) {
#pragma unroll
                for (int m = 0; m < KB; ++m)
                    if (B[colour][m].d > 0.0f) relax_w(B[colour][m], spb, bsx, bsy);
                bar_b();
            }
    }
    __syncthreads();
    // prolongation (multigrid.cl:182-201)
#pragma unroll
    for (int colour = 0; colour < 2; ++colour)
#pragma unroll
        for (int m = 0; m < KA; ++m) {
            if (A[colour][m].d < 0.0f) continue;  // interior fluid cells only
            const int c = A[colour][m].c;
            const int i = c / asx, j = (c / asy) % any, k = c % anz;
            const int I = min((i - 1) / 2 + 1, bnx - 2), J = min((j - 1) / 2 + 1, bny - 2),
                      K = min((k - 1) / 2 + 1, bnz - 2);
            spa[c] += w * spb[(I * bny + J) * bnz + K];
        }
    __syncthreads();
    smooth_a(post);
    if (bb) {
#pragma unroll
        for (int colour = 0; colour < 2; ++colour)
#pragma unroll
            for (int m = 0; m < KB; ++m)
                if (B[colour][m].d >= 0.0f) st(bb, B[colour][m].c, bvals[colour][m]);  // fluid cells
    }
}

// H = true: both levels are stored in FP16 (p, b and operator as __half, scaled values); the visit
// computes in FP32 in shared memory with kappa = scale[2] in place of delta^2 (mg_half.cuh).
template <int KA, int KB, bool H = false>
__device__ __forceinline__ void bottom_visit_block(float* __restrict__ pa, const float* __restrict__ ba,
                                                   const float4* __restrict__ opa, const uint8_t* __restrict__ ma,
                                                   int anx, int any, int anz, float* __restrict__ pb,
                                                   float* __restrict__ bb, const float4* __restrict__ opb,
                                                   const uint8_t* __restrict__ mb, int bnx, int bny, int bnz,
                                                   float delta, int pre, int post, int coarse_iters,
                                                   const float* __restrict__ scale, int b_solves = 2,
                                                   float w = 1.0f) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int CA = anx * any * anz, CB = bnx * bny * bnz;
    const BottomSmem S = bottom_smem(smem, CA, CB);
    const float d2 = H ? scale[2] : delta * delta;
    const float inv_delta2 = H ? scale[3] : 1.0f / (delta * delta);
    auto st = [&](float* a, int c, float v) {
        if (H) reinterpret_cast<__half*>(a)[c] = __float2half_rn(v);
        else a[c] = v;
    };
    bottom_stage<H>(S, pa, ba, opa, ma, CA, opb, mb, CB);
    bottom_lists(S, anx, any, anz, bnx, bny, bnz);
    BottomCells<KA, KB> R;
    bottom_cells(S, R, anx, any, anz, bnx, bny, bnz);
    bottom_rhs(S, R, d2);
    bottom_core<KA, KB, H>(S, R, anx, any, anz, bnx, bny, bnz, d2, inv_delta2, pre, post, coarse_iters, bb, b_solves,
                           w);
    const int bsx = bny * bnz, bsy = bnz;
    for (int c = threadIdx.x; c < CA; c += BOTTOM_THREADS) st(pa, c, S.spa[c]);
    for (int c = threadIdx.x; c < CB; c += BOTTOM_THREADS) {
        st(pb, c, S.spb[c]);
        const int I = c / bsx, J = (c / bsy) % bny, K = c % bnz;
        // multigrid.cl:115 zeroes b off the interior; cells that are not fluid restrict to 0
        if (!interior(I, J, K, bnx, bny, bnz) || S.sob[c].x < 0.0f) st(bb, c, 0.0f);
    }
}

template <int KA, int KB, bool H = false>
__global__ void __launch_bounds__(BOTTOM_THREADS, 1)
    k_bottom_visit(float* __restrict__ pa, const float* __restrict__ ba, const float4* __restrict__ opa,
                   const uint8_t* __restrict__ ma, int anx, int any, int anz, float* __restrict__ pb,
                   float* __restrict__ bb, const float4* __restrict__ opb, const uint8_t* __restrict__ mb, int bnx,
                   int bny, int bnz, float delta, int pre, int post, int coarse_iters,
                   const float* __restrict__ scale, int b_solves, float w) {
    pdl_begin();
    bottom_visit_block<KA, KB, H>(pa, ba, opa, ma, anx, any, anz, pb, bb, opb, mb, bnx, bny, bnz, delta, pre, post,
                                  coarse_iters, scale, b_solves, w);
}

}  // namespace clb
