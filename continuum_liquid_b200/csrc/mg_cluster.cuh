// One visit of the third-coarsest level C = L-3 together with both visits of the level below it
// (its two bottom visits, mg_bottom.cuh), as one launch of a thread-block cluster; or the two visits
// of C that the level above makes back to back, in one launch (`visits` = 2). `a_visits` and
// `b_solves` (2 in the reference's W-cycle, 1 for a level visited once per parent visit) are the
// visits of A per visit of C and the coarse solves of B per visit of A.
//
// A W-cycle visits C 2^(L-3) times, and each visit (multigrid.py:53-187) is pre-smoothing of C,
// restriction to A = C+1, two visits of A (each: smoothing, restriction to B, two coarse solves,
// prolongation, smoothing), prolongation and post-smoothing of C. Launched per step this is ~16
// small launches, each at the ~2 us floor of a dependent launch, while the work per launch is a few
// thousand cells. Here the C-level phases run on CS slab CTAs of a cluster that synchronise with the
// hardware cluster barrier (~0.25 us), and the two A visits run on the cluster's first CTA from its
// shared memory, with A's right-hand side written there by the restriction through distributed
// shared memory.
//
// Layout. C's interior planes are grouped in pairs (the fine planes of one coarse plane of A); slab
// CTA s owns pairs [s P / CS, (s+1) P / CS) and keeps its planes plus one ghost plane on either side
// in shared memory (p, b, and the operator with diagonal -1 where not fluid). After every C phase a
// slab CTA copies its first and last owned planes into its neighbours' ghost planes (remote stores),
// then the cluster barrier makes them visible. The first CTA holds A and B as the bottom visit does.
//
// Every update, restriction sum and prolongation uses the reference's formula and term order; with
// FP16 storage (H) each C-level update is rounded to FP16 as the per-cell FP16 sweep stores it, A's
// right-hand side as the FP16 restriction stores it, and A's p between and after its two visits as
// the bottom visit stores it, so the result equals the launch-per-kernel path bit for bit.
// Nothing waits on a flag: the only waits are cluster and block barriers, which every thread of
// every CTA passes the same number of times.
#pragma once
#include <cooperative_groups.h>

#include "mg_bottom.cuh"
#include "mg_sweep.cuh"

namespace clb {

constexpr int CLUSTER_MAX = 16;  // CTAs per cluster (non-portable size, allowed on sm_100)

__device__ __forceinline__ void cluster_barrier() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

// Planes [i_lo, i_hi) of C owned by slab s of cs (global plane indices; interior planes 1..nx-2),
// the pairs [p0, p1) they form (pair p: planes 2p+1, 2p+2, the fine planes of A's plane p+1).
struct Slab {
    int i_lo, i_hi, p0, p1;
};

__host__ __device__ __forceinline__ Slab cluster_slab(int s, int cs, int nx) {
    const int pairs = (nx - 1) / 2;  // ceil((nx - 2) / 2)
    Slab r;
    r.p0 = (int)((long long)s * pairs / cs);
    r.p1 = (int)((long long)(s + 1) * pairs / cs);
    r.i_lo = 2 * r.p0 + 1;
    r.i_hi = 2 * r.p1 + 1 < nx - 1 ? 2 * r.p1 + 1 : nx - 1;
    return r;
}

// Most planes a slab owns, and the byte offsets of its arrays (the same in every slab CTA, so a
// neighbour's ghost plane is at the same offset in its shared memory).
struct ClusterLayout {
    int own_max;     // owned planes of the largest slab
    size_t op_off;   // operator: (own_max + 2) planes
    size_t p_off;    // p: (own_max + 2) planes
    size_t b_off;    // b: own_max planes
    size_t list_off; // fluid cells of each colour: list_len ints each, then two counts
    int list_len;
    size_t slab_bytes;
};

__host__ __device__ __forceinline__ ClusterLayout cluster_layout(int cs, int nx, int ny, int nz, bool half) {
    const int pairs = (nx - 1) / 2;
    const int pairs_max = (pairs + cs - 1) / cs;
    ClusterLayout L;
    L.own_max = 2 * pairs_max;
    const size_t plane = (size_t)ny * nz;
    const size_t op_bytes = half ? 8 : 16;
    auto pad = [](size_t x) { return (x + 15) & ~(size_t)15; };
    L.op_off = 0;
    L.p_off = pad((size_t)(L.own_max + 2) * plane * op_bytes);
    L.b_off = L.p_off + pad((size_t)(L.own_max + 2) * plane * 4);
    L.list_off = L.b_off + pad((size_t)L.own_max * plane * 4);
    L.list_len = (int)((size_t)L.own_max * plane / 2 + 1);
    L.slab_bytes = L.list_off + pad((size_t)(2 * L.list_len + 2) * 4);
    return L;
}

// Fluid-cell lists of a cluster launch in global memory (clb_mg_hierarchy.cluster_lists), built once
// per solve by k_cluster_lists: first the first CTA's count and list arrays as they lie in its shared
// memory (BottomSmem from `count` on: four counts, A's two lists of CA / 2 + 1 entries, B's two of
// CB / 2 + 1), then per slab its two lists of list_len entries and its two counts (the slab's list
// region); each part padded to a multiple of four entries.
__host__ __device__ __forceinline__ long long cluster_lists_bottom_ints(int CA, int CB) {
    return (4LL + 2 * (CA / 2 + 1) + 2 * (CB / 2 + 1) + 3) & ~3LL;
}
__host__ __device__ __forceinline__ long long cluster_lists_slab_ints(const ClusterLayout& L) {
    return (2LL * L.list_len + 2 + 3) & ~3LL;
}

// Owned C cell: local shared-memory index, diagonal (-1: not updated) and delta^2 * b.
struct SlabCell {
    int c;
    float d;
    float d2b;
};

// glist (nullable): the slab's part of the lists built by k_cluster_lists.
template <int NS, bool H>
__device__ void cluster_slab_path(int s, int cs, const float* __restrict__ pc, float* __restrict__ pc_out,
                                  const float* __restrict__ bc, const void* __restrict__ opc_,
                                  const uint8_t* __restrict__ mc, int nx, int ny, int nz, int anx, int any, int anz,
                                  float d2, float inv_delta2, int pre, int post, int visits,
                                  const int* __restrict__ glist, float w) {
    namespace cgx = cooperative_groups;
    extern __shared__ __align__(16) unsigned char smem[];
    using OpT = typename std::conditional<H, uint2, float4>::type;
    const ClusterLayout L = cluster_layout(cs, nx, ny, nz, H);
    const Slab sl = cluster_slab(s, cs, nx);
    const int own = sl.i_hi - sl.i_lo, np = own + 2;
    const int PL = ny * nz;
    OpT* sop = reinterpret_cast<OpT*>(smem + L.op_off);
    float* sp = reinterpret_cast<float*>(smem + L.p_off);
    float* sb = reinterpret_cast<float*>(smem + L.b_off);
    const OpT* gop = reinterpret_cast<const OpT*>(opc_);
    auto op4 = [&](int q) -> float4 {
        if constexpr (H) return h4_to_f4(sop[q]);
        else return sop[q];
    };
    auto stored = [](float x) { return H ? __half2float(__float2half_rn(x)) : x; };  // as C's p holds it

    // staging: planes i_lo - 1 .. i_hi of p and the operator, the owned planes of b
    const size_t g0 = (size_t)(sl.i_lo - 1) * PL;
    for (int q = threadIdx.x; q < np * PL; q += BOTTOM_THREADS) {
        const size_t g = g0 + q;
        const bool fluid = __ldg(mc + g) != 0;
        const float p = H ? __half2float(reinterpret_cast<const __half*>(pc)[g]) : __ldg(pc + g);
        OpT o = __ldg(gop + g);
        if (!fluid) {
            if constexpr (H) o.x = (o.x & 0xFFFF0000u) | 0xBC00u;  // half -1 in the diagonal's slot
            else o.x = -1.0f;
        }
        sp[q] = fluid ? p : 0.0f;
        sop[q] = o;
    }
    for (int q = threadIdx.x; q < own * PL; q += BOTTOM_THREADS) {
        const size_t g = g0 + PL + q;
        sb[q] = H ? __half2float(reinterpret_cast<const __half*>(bc)[g]) : __ldg(bc + g);
    }
    __syncthreads();

    // owned cells: the slab's fluid cells of each colour (the slab seen as a level of np planes; the
    // local plane il is global plane il + i_lo - 1), taken in turn by the threads, so only a warp's last
    // owned slots can be empty (bottom_lists). From glist when given (k_cluster_lists, in slot order),
    // otherwise listed here in arbitrary order; cells of one colour are independent, so the order does
    // not change any value.
    int* list = reinterpret_cast<int*>(smem + L.list_off);
    const int* src = glist;
    if (!glist) {
        const int flip = (sl.i_lo - 1) & 1;
        int* count = list + 2 * L.list_len;
        if (threadIdx.x < 2) count[threadIdx.x] = 0;
        __syncthreads();
        const int slots = colour_slots(np, ny, nz);
        for (int colour = 0; colour < 2; ++colour)
            for (int r = threadIdx.x; r < slots; r += BOTTOM_THREADS) {
                const int c = colour_cell(r, colour ^ flip, np, ny, nz);
                if (c >= 0 && op4(c).x >= 0.0f) list[colour * L.list_len + atomicAdd(count + colour, 1)] = c;
            }
        src = list;
    }
    __syncthreads();
    const int counts[2] = {src[2 * L.list_len], src[2 * L.list_len + 1]};
    SlabCell C[2][NS];
#pragma unroll
    for (int colour = 0; colour < 2; ++colour)
#pragma unroll
        for (int m = 0; m < NS; ++m) {
            const int r = threadIdx.x + m * BOTTOM_THREADS;
            const int c = r < counts[colour] ? src[colour * L.list_len + r] : -1;
            SlabCell& o = C[colour][m];
            o.c = c < 0 ? 0 : c;
            o.d = c < 0 ? -1.0f : op4(c).x;
            o.d2b = c < 0 ? 0.0f : d2 * sb[c - PL];
        }

    // neighbours' ghost planes: the left slab's top ghost, the right slab's bottom ghost
    cgx::cluster_group cluster = cgx::this_cluster();
    float* left_ghost = nullptr;
    float* right_ghost = nullptr;
    if (s > 0) {
        const Slab ls = cluster_slab(s - 1, cs, nx);
        float* lp = cluster.map_shared_rank(sp, (unsigned)s);  // rank s hosts slab s - 1
        left_ghost = lp + (size_t)(ls.i_hi - ls.i_lo + 1) * PL;
    }
    if (s + 1 < cs) right_ghost = cluster.map_shared_rank(sp, (unsigned)(s + 2));
    auto push = [&]() {
        __syncthreads();
        if (left_ghost)
            for (int q = threadIdx.x; q < PL; q += BOTTOM_THREADS) left_ghost[q] = sp[PL + q];
        if (right_ghost)
            for (int q = threadIdx.x; q < PL; q += BOTTOM_THREADS) right_ghost[q] = sp[own * PL + q];
        cluster_barrier();
    };
    auto phase = [&](int colour) {
#pragma unroll
        for (int m = 0; m < NS; ++m) {
            const SlabCell& o = C[colour][m];
            if (!(o.d > 0.0f)) continue;
            const int c = o.c;
            const float4 self = op4(c);
            const float ws = self.y * sp[c + PL] + op4(c - PL).y * sp[c - PL] + self.z * sp[c + nz] +
                             op4(c - nz).z * sp[c - nz] + self.w * sp[c + 1] + op4(c - 1).w * sp[c - 1];
            sp[c] = stored((ws - o.d2b) / o.d);
        }
        push();
    };

    // consecutive visits of C (the two a W-cycle makes from the level above) keep C's planes, lists and
    // operands in shared memory: a visit starts from the p the previous one left, exactly as a
    // separate launch that staged it again would
    for (int visit = 0; visit < visits; ++visit) {
    cluster_barrier();  // every CTA staged (the first CTA zeroed A's p and b)
    for (int it = 0; it < pre; ++it) {
        phase(0);
        phase(1);
    }

    // restriction of the residual into A's b in the first CTA (multigrid.cl:90-180; FP16:
    // k_restrict_h<2>, rounded to FP16 as stored there). The residuals of the eight children
    // l = 4 di + 2 dj + dk are formed independently (interior fluid children only) and added in that
    // order, as the reference's loop over di, dj, dk adds them.
    {
        const int CA = anx * any * anz;
        const BottomSmem S = bottom_smem(cluster.map_shared_rank(smem, 0u), CA, 1);
        const int I0 = sl.p0 + 1, I1 = sl.p1 + 1;  // A's planes of the owned pairs
        const int my = any - 2, mz = anz - 2;
        for (int t = threadIdx.x; t < (I1 - I0) * my * mz; t += BOTTOM_THREADS) {
            const int I = I0 + t / (my * mz), r = t % (my * mz), J = 1 + r / mz, K = 1 + r % mz;
            if (I <= anx - 2) {
                float res[8];
                bool present[8];
#pragma unroll
                for (int l = 0; l < 8; ++l) {
                    const int i = 2 * I - 1 + (l >> 2), j = 2 * J - 1 + ((l >> 1) & 1), k = 2 * K - 1 + (l & 1);
                    res[l] = 0.0f;
                    present[l] = false;
                    if (interior(i, j, k, nx, ny, nz)) {
                        const int f = ((i - sl.i_lo + 1) * ny + j) * nz + k;
                        const float4 o = op4(f);
                        if (o.x >= 0.0f) {  // fluid
                            const float ws = o.y * sp[f + PL] + op4(f - PL).y * sp[f - PL] + o.z * sp[f + nz] +
                                             op4(f - nz).z * sp[f - nz] + o.w * sp[f + 1] + op4(f - 1).w * sp[f - 1];
                            res[l] = sb[f - PL] - (ws - o.x * sp[f]) * inv_delta2;
                            present[l] = true;
                        }
                    }
                }
                float rhs = 0.0f;
#pragma unroll
                for (int l = 0; l < 8; ++l)
                    if (present[l]) rhs += res[l];
                S.sba[(I * any + J) * anz + K] = stored(rhs);
            }
        }
    }
    cluster_barrier();  // A's right-hand side is complete
    cluster_barrier();  // the first CTA finished both visits of A

    // prolongation (multigrid.cl:182-201) from A's p in the first CTA. The owned planes' parents lie in
    // A's planes [I_lo, I_hi]; they are first copied into the list region (free once the owned cells
    // are in registers) with every remote load of a thread issued before its stores, so each owned cell
    // then reads its parent from this CTA's shared memory instead of waiting on a remote load.
    {
        const int CA = anx * any * anz, APL = any * anz;
        const float* spa = bottom_smem(cluster.map_shared_rank(smem, 0u), CA, 1).spa;
        const int I_lo = min(sl.p0 + 1, anx - 2), I_hi = min(sl.p1, anx - 2);
        const int n_a = (I_hi - I_lo + 1) * APL;
        const bool local = n_a > 0 && n_a <= 2 * L.list_len;  // uniform over the CTA
        const float* parent = spa;
        int base = 0;
        if (local) {
            float* sa = reinterpret_cast<float*>(list);
            const float* src = spa + (size_t)I_lo * APL;
            constexpr int U = 4;
            for (int q0 = threadIdx.x; q0 < n_a; q0 += U * BOTTOM_THREADS) {
                float v[U];
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const int q = q0 + u * BOTTOM_THREADS;
                    v[u] = q < n_a ? src[q] : 0.0f;
                }
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const int q = q0 + u * BOTTOM_THREADS;
                    if (q < n_a) sa[q] = v[u];
                }
            }
            __syncthreads();
            parent = sa;
            base = I_lo * APL;
        }
#pragma unroll
        for (int colour = 0; colour < 2; ++colour)
#pragma unroll
            for (int m = 0; m < NS; ++m) {
                const SlabCell& o = C[colour][m];
                if (o.d < 0.0f) continue;  // interior fluid cells only
                const int c = o.c;
                const int il = c / PL, j = (c / nz) % ny, k = c % nz;
                const int i = il + sl.i_lo - 1;
                const int I = min((i - 1) / 2 + 1, anx - 2), J = min((j - 1) / 2 + 1, any - 2),
                          K = min((k - 1) / 2 + 1, anz - 2);
                sp[c] = stored(sp[c] + w * parent[(I * any + J) * anz + K - base]);
            }
    }
    push();
    for (int it = 0; it < post; ++it) {
        phase(0);
        phase(1);
    }
    }  // visits

    // the owned planes back to C's p
    for (int q = threadIdx.x; q < own * PL; q += BOTTOM_THREADS) {
        const size_t g = g0 + PL + q;
        if (H) reinterpret_cast<__half*>(pc_out)[g] = __float2half_rn(sp[PL + q]);
        else pc_out[g] = sp[PL + q];
    }
}

template <int KA, int KB, bool H>
__device__ void cluster_bottom_path(float* __restrict__ pa, const float4* __restrict__ opa,
                                    const uint8_t* __restrict__ ma, int anx, int any, int anz,
                                    const float4* __restrict__ opb, const uint8_t* __restrict__ mb, int bnx, int bny,
                                    int bnz, float d2, float inv_delta2, int pre, int post, int coarse_iters,
                                    int visits, int a_visits, int b_solves, const int* __restrict__ glist, float w) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int CA = anx * any * anz, CB = bnx * bny * bnz;
    const BottomSmem S = bottom_smem(smem, CA, CB);
    bottom_stage<H>(S, nullptr, nullptr, opa, ma, CA, opb, mb, CB);
    if (glist) {
        // the counts and lists as k_cluster_lists built them (16-byte aligned at both ends; the padded
        // length fits the shared list region, bottom_smem_bytes)
        const int n4 = (int)(cluster_lists_bottom_ints(CA, CB) / 4);
        const int4* from = reinterpret_cast<const int4*>(glist);
        int4* to = reinterpret_cast<int4*>(S.count);
        for (int q = threadIdx.x; q < n4; q += BOTTOM_THREADS) to[q] = from[q];
        __syncthreads();
    } else {
        bottom_lists(S, anx, any, anz, bnx, bny, bnz);
    }
    BottomCells<KA, KB> R;  // the owned cells and B's weights, set once for every visit of A
    bottom_cells(S, R, anx, any, anz, bnx, bny, bnz);
    // the restriction zeroes the coarse pressure (multigrid.cl:114) before every visit of A's parent;
    // cells of b that the restriction does not write (not interior) hold 0, and the slabs write every
    // interior cell of b in each visit of C, so b is zeroed once
    for (int c = threadIdx.x; c < CA; c += BOTTOM_THREADS) {
        S.spa[c] = 0.0f;
        S.sba[c] = 0.0f;
    }
    for (int visit_c = 0; visit_c < visits; ++visit_c) {
    cluster_barrier();  // staged (for a later visit of C: A's p zeroed after the slabs read it)
    for (int it = 0; it < 2 * pre; ++it) cluster_barrier();  // the C-level pre-smoothing phases
    cluster_barrier();  // A's right-hand side is complete
    bottom_rhs(S, R, d2);
    for (int visit = 0; visit < a_visits; ++visit) {  // two, or one when A is visited once
        bottom_core<KA, KB, H>(S, R, anx, any, anz, bnx, bny, bnz, d2, inv_delta2, pre, post, coarse_iters,
                               nullptr, b_solves, w);
        __syncthreads();
        if (H)  // A's p as the bottom visit stores it (FP16) before it is read again
            for (int c = threadIdx.x; c < CA; c += BOTTOM_THREADS) S.spa[c] = __half2float(__float2half_rn(S.spa[c]));
        __syncthreads();
    }
    cluster_barrier();  // both visits done; the slabs read A's p next
    cluster_barrier();  // prolongation done
    if (visit_c + 1 < visits)  // the next visit's zero p, while the slabs post-smooth
        for (int c = threadIdx.x; c < CA; c += BOTTOM_THREADS) S.spa[c] = 0.0f;
    for (int it = 0; it < 2 * post; ++it) cluster_barrier();  // the C-level post-smoothing phases
    }  // visits of C
    for (int c = threadIdx.x; c < CA; c += BOTTOM_THREADS) {
        if (H) reinterpret_cast<__half*>(pa)[c] = __float2half_rn(S.spa[c]);
        else pa[c] = S.spa[c];
    }
}

// The cluster's CTA 0 runs the A/B visits; CTAs 1.. are the C-level slabs (cs = cluster size - 1).
template <int NS, int KA, int KB, bool H>
__global__ void __launch_bounds__(BOTTOM_THREADS, 1)
    k_cluster_visit(float* __restrict__ pc, const float* __restrict__ bc, const void* __restrict__ opc,
                    const uint8_t* __restrict__ mc, int nx, int ny, int nz, float* __restrict__ pa,
                    const float4* __restrict__ opa, const uint8_t* __restrict__ ma, int anx, int any, int anz,
                    const float4* __restrict__ opb, const uint8_t* __restrict__ mb, int bnx, int bny, int bnz,
                    float delta, int pre, int post, int coarse_iters, const float* __restrict__ scale,
                    int visits, int a_visits, int b_solves, const int* __restrict__ lists, float w) {
    pdl_begin();
    const float d2 = H ? scale[2] : delta * delta;
    const float inv_delta2 = H ? scale[3] : 1.0f / (delta * delta);
    const unsigned rank = cooperative_groups::this_cluster().block_rank();
    const int cs = (int)cooperative_groups::this_cluster().num_blocks() - 1;
    if (rank == 0)
        cluster_bottom_path<KA, KB, H>(pa, opa, ma, anx, any, anz, opb, mb, bnx, bny, bnz, d2, inv_delta2, pre, post,
                                       coarse_iters, visits, a_visits, b_solves, lists, w);
    else
        cluster_slab_path<NS, H>((int)rank - 1, cs, pc, pc, bc, opc, mc, nx, ny, nz, anx, any, anz, d2, inv_delta2,
                                 pre, post, visits,
                                 lists ? lists + cluster_lists_bottom_ints(anx * any * anz, bnx * bny * bnz) +
                                             (rank - 1) * cluster_lists_slab_ints(cluster_layout(cs, nx, ny, nz, H))
                                       : nullptr,
                                 w);
}

// Lists the fluid cells that the CTAs of a cluster launch own, as the launch would list them but in
// slot order: block 0 those of A and B (bottom_lists), block s + 1 those of slab s (the launch's
// per-slab lists). Once per solve, after the coarse operators are built; a cell is listed when the
// diagonal the launch stages for it (-1 where not fluid) is not negative, the launch's own test.
template <bool H>
__global__ void __launch_bounds__(BOTTOM_THREADS)
    k_cluster_lists(int* __restrict__ lists, const void* __restrict__ opc, const uint8_t* __restrict__ mc, int nx,
                    int ny, int nz, const void* __restrict__ opa, const uint8_t* __restrict__ ma, int anx, int any,
                    int anz, const void* __restrict__ opb, const uint8_t* __restrict__ mb, int bnx, int bny, int bnz,
                    int cs) {
    pdl_begin();
    __shared__ int warp_n[BOTTOM_THREADS / 32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    // appends the cells cell(r) >= 0 of slots r < slots to out in slot order; returns how many
    auto compact = [&](int slots, auto cell, int* out) -> int {
        int base = 0;
        for (int r0 = 0; r0 < slots; r0 += BOTTOM_THREADS) {  // the same trip count in every thread
            const int r = r0 + (int)threadIdx.x;
            const int c = r < slots ? cell(r) : -1;
            const unsigned ballot = __ballot_sync(0xffffffffu, c >= 0);
            if (lane == 0) warp_n[w] = __popc(ballot);
            __syncthreads();
            int before = 0, all = 0;
            for (int q = 0; q < BOTTOM_THREADS / 32; ++q) {
                const int v = warp_n[q];
                before += q < w ? v : 0;
                all += v;
            }
            if (c >= 0) out[base + before + __popc(ballot & ((1u << lane) - 1u))] = c;
            __syncthreads();
            base += all;
        }
        return base;
    };
    auto diag = [](const void* op, const uint8_t* m, long long g) -> float {
        if (!m[g]) return -1.0f;
        if constexpr (H) return h4_to_f4(reinterpret_cast<const uint2*>(op)[g]).x;
        else return reinterpret_cast<const float4*>(op)[g].x;
    };
    if (blockIdx.x == 0) {
        const int CA = anx * any * anz, CB = bnx * bny * bnz, la = CA / 2 + 1, lb = CB / 2 + 1;
        int* list_a = lists + 4;
        int* list_b = list_a + 2 * la;
        const int sa = colour_slots(anx, any, anz), sb = colour_slots(bnx, bny, bnz);
        int n[4];
#pragma unroll
        for (int colour = 0; colour < 2; ++colour) {
            n[colour] = compact(sa, [&](int r) {
                const int c = colour_cell(r, colour, anx, any, anz);
                return c >= 0 && diag(opa, ma, c) >= 0.0f ? c : -1;
            }, list_a + colour * la);
            n[2 + colour] = compact(sb, [&](int r) {
                const int c = colour_cell(r, colour, bnx, bny, bnz);
                return c >= 0 && diag(opb, mb, c) >= 0.0f ? c : -1;
            }, list_b + colour * lb);
        }
        if (threadIdx.x == 0) {
            lists[0] = n[0];
            lists[1] = n[1];
            lists[2] = n[2];
            lists[3] = n[3];
        }
    } else {
        const int s = (int)blockIdx.x - 1;
        const ClusterLayout L = cluster_layout(cs, nx, ny, nz, H);
        const Slab sl = cluster_slab(s, cs, nx);
        const int np = sl.i_hi - sl.i_lo + 2, flip = (sl.i_lo - 1) & 1;
        const long long g0 = (long long)(sl.i_lo - 1) * ny * nz;
        int* list = lists + cluster_lists_bottom_ints(anx * any * anz, bnx * bny * bnz) +
                    (long long)s * cluster_lists_slab_ints(L);
        const int slots = colour_slots(np, ny, nz);
        int n[2];
#pragma unroll
        for (int colour = 0; colour < 2; ++colour)
            n[colour] = compact(slots, [&](int r) {
                const int c = colour_cell(r, colour ^ flip, np, ny, nz);
                return c >= 0 && diag(opc, mc, g0 + c) >= 0.0f ? c : -1;
            }, list + colour * L.list_len);
        if (threadIdx.x == 0) {
            list[2 * L.list_len] = n[0];
            list[2 * L.list_len + 1] = n[1];
        }
    }
}

}  // namespace clb
