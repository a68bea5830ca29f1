// Particle binning: bin keys, per-cell counts, exclusive scan, deterministic stable counting sort,
// and the per-cell P2G gather (Solver/Kernel/OpenCL/particles.cl, Solver/Kernel/particles.py).
#pragma once
#include "common.cuh"

namespace clb {

// ------------------------------------------------------------------------------------------------
// Particle loads: a block stages its particles' (N,3) float32 records through shared memory with
// 16-byte vector loads, so each warp issues full 128-byte requests instead of 12-byte-strided ones.
// ------------------------------------------------------------------------------------------------
constexpr int PT = 256;  // particles (threads) per block for particle-wide kernels

__device__ __forceinline__ void stage_particles(const float* __restrict__ src, i64 first, i64 n, float* sm) {
    const i64 count = (n - first) < PT ? (n - first) : PT;
    const float* base = src + 3 * first;
    if (count == PT && (((uintptr_t)base) & 15) == 0) {
        const float4* b4 = reinterpret_cast<const float4*>(base);
        float4* s4 = reinterpret_cast<float4*>(sm);
        for (int t = threadIdx.x; t < 3 * PT / 4; t += blockDim.x) s4[t] = __ldg(b4 + t);
    } else {
        for (int t = threadIdx.x; t < 3 * count; t += blockDim.x) sm[t] = __ldg(base + t);
    }
}

__device__ __forceinline__ void unstage_particles(float* __restrict__ dst, i64 first, i64 n, const float* sm) {
    const i64 count = (n - first) < PT ? (n - first) : PT;
    float* base = dst + 3 * first;
    if (count == PT && (((uintptr_t)base) & 15) == 0) {
        float4* b4 = reinterpret_cast<float4*>(base);
        const float4* s4 = reinterpret_cast<const float4*>(sm);
        for (int t = threadIdx.x; t < 3 * PT / 4; t += blockDim.x) b4[t] = s4[t];
    } else {
        for (int t = threadIdx.x; t < 3 * count; t += blockDim.x) base[t] = sm[t];
    }
}

// particles.cl:3-6 interpolation_base + helper.cl:4-6: flat bin key of a position.
__device__ __forceinline__ int bin_key(float px, float py, float pz, float inv_dx, int nx, int ny, int nz) {
    const float x = px * inv_dx - 0.5f;
    const float y = py * inv_dx - 0.5f;
    const float z = pz * inv_dx - 0.5f;
    const int bx = clampi((int)floorf(x), 0, nx - 2);
    const int by = clampi((int)floorf(y), 0, ny - 2);
    const int bz = clampi((int)floorf(z), 0, nz - 2);
    return (int)gidx(bx, by, bz, ny, nz);
}

// particles.cl:44-59 count_particles_per_cell, warp-aggregated: lanes with equal keys are grouped by
// __match_any_sync and their leader issues one atomicAdd for the group. Each particle also gets its
// key and a rank within its bin (unique, but ordered by atomic arrival; k_stable_gather makes the
// final order deterministic).
__global__ void __launch_bounds__(PT) k_bin_count(const float* __restrict__ pos, i64 n, float inv_dx, int nx, int ny,
                                                   int nz, int* __restrict__ counts, int* __restrict__ keys,
                                                   int* __restrict__ ranks) {
    __shared__ __align__(16) float sm[3 * PT];
    const i64 first = (i64)blockIdx.x * PT;
    stage_particles(pos, first, n, sm);
    __syncthreads();
    const i64 p = first + threadIdx.x;
    int key = -1;
    if (p < n) key = bin_key(sm[3 * threadIdx.x], sm[3 * threadIdx.x + 1], sm[3 * threadIdx.x + 2], inv_dx, nx, ny, nz);
    const unsigned peers = __match_any_sync(0xffffffffu, key);
    if (key >= 0) {
        const int lane = threadIdx.x & 31;
        const int leader = __ffs(peers) - 1;
        int base = 0;
        if (lane == leader) base = atomicAdd(counts + key, __popc(peers));
        base = __shfl_sync(peers, base, leader);
        if (keys) keys[p] = key;
        if (ranks) ranks[p] = base + __popc(peers & ((1u << lane) - 1u));
    }
}

// ------------------------------------------------------------------------------------------------
// Exclusive scan (replaces particles.py:39-70 exclusive_prefix_sum and particles.cl:61-108): one
// pass with decoupled look-back. Tiles are claimed in launch order from a ticket counter, so a tile
// only ever waits on tiles whose blocks are already running. Every wait is bounded; when it runs out
// the kernel records error code 1 and carries on, so the launch always terminates.
// Scratch layout: [ticket u32, pad u32][status u64 x tiles]; it must start zeroed (the launcher
// clears it on the stream before each scan).
// ------------------------------------------------------------------------------------------------
constexpr int SCAN_THREADS = 256;
constexpr int SCAN_ITEMS = 16;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;
constexpr unsigned long long SCAN_FLAG_AGG = 1ull << 32;
constexpr unsigned long long SCAN_FLAG_INC = 2ull << 32;
constexpr int SCAN_SPIN_LIMIT = 1 << 20;

__device__ __forceinline__ unsigned long long ld_volatile_u64(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_volatile_u64(unsigned long long* p, unsigned long long v) {
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__global__ void __launch_bounds__(SCAN_THREADS) k_scan_lookback(const int* __restrict__ in, int* __restrict__ out,
                                                                  i64 count, unsigned int* ticket,
                                                                  unsigned long long* status, int* total, int tiles) {
    __shared__ int s_tile;
    __shared__ int s_warp[SCAN_THREADS / 32];
    __shared__ int s_prefix;
    if (threadIdx.x == 0) s_tile = (int)atomicAdd(ticket, 1u);
    __syncthreads();
    const int tile = s_tile;
    const i64 base = (i64)tile * SCAN_TILE + (i64)threadIdx.x * SCAN_ITEMS;
    int v[SCAN_ITEMS];
    if (base + SCAN_ITEMS <= count && (((uintptr_t)(in + base)) & 15) == 0) {
        const int4* p4 = reinterpret_cast<const int4*>(in + base);
#pragma unroll
        for (int q = 0; q < SCAN_ITEMS / 4; ++q) {
            const int4 t = __ldg(p4 + q);
            v[4 * q] = t.x;
            v[4 * q + 1] = t.y;
            v[4 * q + 2] = t.z;
            v[4 * q + 3] = t.w;
        }
    } else {
#pragma unroll
        for (int q = 0; q < SCAN_ITEMS; ++q) v[q] = (base + q < count) ? __ldg(in + base + q) : 0;
    }
    int run = 0;
#pragma unroll
    for (int q = 0; q < SCAN_ITEMS; ++q) {
        const int x = v[q];
        v[q] = run;  // exclusive within the thread
        run += x;
    }
    // block-wide exclusive scan of the per-thread totals
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int inc = run;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += y;
    }
    if (lane == 31) s_warp[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        int w = lane < SCAN_THREADS / 32 ? s_warp[lane] : 0;
        int wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi += y;
        }
        if (lane < SCAN_THREADS / 32) s_warp[lane] = wi - w;  // exclusive warp offsets
        const int aggregate = __shfl_sync(0xffffffffu, wi, SCAN_THREADS / 32 - 1);
        // decoupled look-back
        int prefix = 0;
        if (tile == 0) {
            if (lane == 0) st_volatile_u64(status, SCAN_FLAG_INC | (unsigned int)aggregate);
        } else {
            if (lane == 0) st_volatile_u64(status + tile, SCAN_FLAG_AGG | (unsigned int)aggregate);
            int idx = tile - 1;
            bool done = false;
            while (!done) {
                const int mine = idx - lane;
                unsigned long long s = SCAN_FLAG_INC;  // lanes before tile 0 contribute nothing
                if (mine >= 0) {
                    int spins = 0;
                    s = ld_volatile_u64(status + mine);
                    while ((s >> 32) == 0ull) {
                        if (++spins > SCAN_SPIN_LIMIT) {
                            raise_device_error(1u);
                            s = SCAN_FLAG_INC;
                            break;
                        }
                        __nanosleep(32);
                        s = ld_volatile_u64(status + mine);
                    }
                }
                const unsigned inc_mask = __ballot_sync(0xffffffffu, (s >> 32) == 2ull);
                const int stop = inc_mask ? (__ffs(inc_mask) - 1) : 32;
                int contrib = (lane <= stop && lane < 32 && mine >= 0) ? (int)(unsigned int)(s & 0xffffffffull) : 0;
                if (lane > stop) contrib = 0;
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) contrib += __shfl_xor_sync(0xffffffffu, contrib, o);
                prefix += contrib;
                if (inc_mask) done = true;
                idx -= 32;
            }
            if (lane == 0) st_volatile_u64(status + tile, SCAN_FLAG_INC | (unsigned int)(prefix + aggregate));
        }
        if (lane == 0) {
            s_prefix = prefix;
            if (tile == tiles - 1 && total) *total = prefix + aggregate;
        }
    }
    __syncthreads();
    const int offset = s_prefix + s_warp[warp] + (inc - run);
    if (base + SCAN_ITEMS <= count && (((uintptr_t)(out + base)) & 15) == 0) {
        int4* o4 = reinterpret_cast<int4*>(out + base);
#pragma unroll
        for (int q = 0; q < SCAN_ITEMS / 4; ++q)
            o4[q] = make_int4(v[4 * q] + offset, v[4 * q + 1] + offset, v[4 * q + 2] + offset, v[4 * q + 3] + offset);
    } else {
#pragma unroll
        for (int q = 0; q < SCAN_ITEMS; ++q)
            if (base + q < count) out[base + q] = v[q] + offset;
    }
}

static inline i64 scan_tiles(i64 count) { return (count + SCAN_TILE - 1) / SCAN_TILE; }
static inline i64 scan_scratch_bytes(i64 count) { return 16 + 8 * (scan_tiles(count) > 0 ? scan_tiles(count) : 1); }

static inline int launch_scan(const int* in, int* out, i64 count, void* scratch, i64 scratch_bytes, int* total,
                              cudaStream_t s) {
    if (count <= 0) {
        if (total) return check_call(cudaMemsetAsync(total, 0, sizeof(int), s), "scan total");
        return 0;
    }
    CLB_REQUIRE(scratch != nullptr && scratch_bytes >= scan_scratch_bytes(count),
                "exclusive_prefix_sum: scratch of %lld bytes is below the %lld bytes needed", (long long)scratch_bytes,
                (long long)scan_scratch_bytes(count));
    CLB_REQUIRE((((uintptr_t)scratch) & 15) == 0, "exclusive_prefix_sum: scratch must be 16-byte aligned");
    const i64 tiles = scan_tiles(count);
    CLB_REQUIRE(tiles < (1ll << 31), "exclusive_prefix_sum: count too large");
    if (check_call(cudaMemsetAsync(scratch, 0, (size_t)scan_scratch_bytes(count), s), "scan scratch clear")) return 1;
    unsigned int* ticket = reinterpret_cast<unsigned int*>(scratch);
    unsigned long long* status = reinterpret_cast<unsigned long long*>(reinterpret_cast<char*>(scratch) + 16);
    k_scan_lookback<<<(unsigned)tiles, SCAN_THREADS, 0, s>>>(in, out, count, ticket, status, total, (int)tiles);
    CLB_LAUNCH_CHECK("k_scan_lookback");
    return 0;
}

// ------------------------------------------------------------------------------------------------
// Stable counting-sort scatter (replaces particles.cl:110-133 sort_particles). The reference's
// atomic cursor leaves the order within a bin unspecified; here the final order is ascending by the
// particle's index in the unsorted array, which is the order a serial run of the reference gives.
// Pass 1 places each particle's index at offsets[key] + rank (rank from the count pass).
// Pass 2 (one thread per slot) counts the smaller indices in its bin's slot range to get the
// stable position, and moves the position and velocity records there.
// ------------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(PT) k_scatter_perm(const int* __restrict__ keys, const int* __restrict__ ranks,
                                                      const int* __restrict__ offsets, i64 n, int* __restrict__ perm,
                                                      int* __restrict__ slot_keys) {
    const i64 p = (i64)blockIdx.x * PT + threadIdx.x;
    if (p >= n) return;
    const int key = keys[p];
    const i64 slot = (i64)offsets[key] + ranks[p];
    perm[slot] = (int)p;
    slot_keys[slot] = key;
}

__global__ void __launch_bounds__(PT) k_stable_gather(const int* __restrict__ perm, const int* __restrict__ slot_keys,
                                                       const int* __restrict__ offsets, const int* __restrict__ counts,
                                                       const float* __restrict__ pos, const float* __restrict__ vel,
                                                       i64 n, float* __restrict__ pos_sorted,
                                                       float* __restrict__ vel_sorted) {
    const i64 j = (i64)blockIdx.x * PT + threadIdx.x;
    if (j >= n) return;
    const int key = slot_keys[j];
    const int begin = offsets[key];
    const int cnt = counts[key];
    const int me = perm[j];
    int rank = 0;
    for (int t = 0; t < cnt; ++t) rank += (__ldg(perm + begin + t) < me) ? 1 : 0;
    const i64 dst = 3 * ((i64)begin + rank);
    const i64 src = 3 * (i64)me;
    pos_sorted[dst] = __ldg(pos + src);
    pos_sorted[dst + 1] = __ldg(pos + src + 1);
    pos_sorted[dst + 2] = __ldg(pos + src + 2);
    vel_sorted[dst] = __ldg(vel + src);
    vel_sorted[dst + 1] = __ldg(vel + src + 1);
    vel_sorted[dst + 2] = __ldg(vel + src + 2);
}

// ------------------------------------------------------------------------------------------------
// particles.cl:135-227 particle_to_grid_gather. Eight lanes per cell, exactly as the reference's
// work-group of GATHER_THREADS_PER_CELL=8: lane l visits neighbour bins l, l+8, l+16, l+24 in that
// order and the particles of each bin in sorted order; the partial sums are reduced with offsets
// 4, 2, 1. Using the reference's summation order makes the result bit-identical to the CPU
// restatement for the same sorted particle order.
//
// Bins whose every term is exactly zero are skipped: a particle in bin b has s = p/dx in
// [b + 0.5, b + 1.5) on each axis (for clamped bins, farther away), so for the u face of cell c (at
// c + (1, 0.5, 0.5)) the y and z weights vanish when the bin is one above the cell (o_y = +1 or
// o_z = +1), likewise for v and w, and the inside count needs o <= 0 on all axes: a bin with two or
// more +1 offsets contributes nothing. Adding an exactly-zero term does not change a sum (up to the
// sign of a zero sum), so the result keeps the reference's values.
// ------------------------------------------------------------------------------------------------
constexpr int P2G_LANES = 8;
constexpr int P2G_THREADS = 256;

__device__ __forceinline__ float tent(float s, float f) { return fmaxf(0.0f, 1.0f - fabsf(s - f)); }

// Cell `index` of the grid (nothing to do when index >= nx*ny*nz) by lane `lane` of its eight-lane
// group; every lane of the warp must call it (the partial sums are combined with shuffles).
__device__ __forceinline__ void p2g_cell(i64 index, int lane, const float* __restrict__ pos,
                                         const float* __restrict__ vel, const int* __restrict__ offsets,
                                         const int* __restrict__ counts, float* __restrict__ u, float* __restrict__ v,
                                         float* __restrict__ w, float* __restrict__ ff, float inv_dx, float inv_ppc,
                                         int nx, int ny, int nz) {
    const i64 C = (i64)nx * ny * nz;
    float vs0 = 0.0f, vs1 = 0.0f, vs2 = 0.0f, ws0 = 0.0f, ws1 = 0.0f, ws2 = 0.0f;
    int inside = 0;
    int ci = 0, cj = 0, ck = 0;
    if (index < C) {
        gcoord(index, ny, nz, ci, cj, ck);
        const float gx = (float)ci, gy = (float)cj, gz = (float)ck;
        const float ux = gx + 1.0f, uy = gy + 0.5f, uz = gz + 0.5f;
        const float vx = gx + 0.5f, vy = gy + 1.0f, vz = gz + 0.5f;
        const float wx = gx + 0.5f, wy = gy + 0.5f, wz = gz + 1.0f;
        for (int nb = lane; nb < 27; nb += P2G_LANES) {
            const int ox = nb / 9 - 1, oy = (nb / 3) % 3 - 1, oz = nb % 3 - 1;
            const int bx = ci + ox;
            if (bx < 0 || bx >= nx - 1) continue;
            const int by = cj + oy;
            if (by < 0 || by >= ny - 1) continue;
            const int bz = ck + oz;
            if (bz < 0 || bz >= nz - 1) continue;
            if ((ox > 0) + (oy > 0) + (oz > 0) >= 2) continue;  // every weight of this bin is zero
            const i64 bin = gidx(bx, by, bz, ny, nz);
            const int begin = __ldg(offsets + bin);
            const int end = begin + __ldg(counts + bin);
            for (int q = begin; q < end; ++q) {
                const float* P = pos + 3 * (i64)q;
                const float* V = vel + 3 * (i64)q;
                const float s0 = __ldg(P) * inv_dx, s1 = __ldg(P + 1) * inv_dx, s2 = __ldg(P + 2) * inv_dx;
                const int pc0 = clampi((int)s0, 1, nx - 2);
                const int pc1 = clampi((int)s1, 1, ny - 2);
                const int pc2 = clampi((int)s2, 1, nz - 2);
                inside += (pc0 == ci && pc1 == cj && pc2 == ck) ? 1 : 0;
                const float wu = tent(s0, ux) * tent(s1, uy) * tent(s2, uz);
                const float wv = tent(s0, vx) * tent(s1, vy) * tent(s2, vz);
                const float ww = tent(s0, wx) * tent(s1, wy) * tent(s2, wz);
                vs0 += wu * __ldg(V);
                vs1 += wv * __ldg(V + 1);
                vs2 += ww * __ldg(V + 2);
                ws0 += wu;
                ws1 += wv;
                ws2 += ww;
            }
        }
    }
#pragma unroll
    for (int o = P2G_LANES / 2; o > 0; o >>= 1) {
        vs0 += __shfl_down_sync(0xffffffffu, vs0, o, P2G_LANES);
        vs1 += __shfl_down_sync(0xffffffffu, vs1, o, P2G_LANES);
        vs2 += __shfl_down_sync(0xffffffffu, vs2, o, P2G_LANES);
        ws0 += __shfl_down_sync(0xffffffffu, ws0, o, P2G_LANES);
        ws1 += __shfl_down_sync(0xffffffffu, ws1, o, P2G_LANES);
        ws2 += __shfl_down_sync(0xffffffffu, ws2, o, P2G_LANES);
        inside += __shfl_down_sync(0xffffffffu, inside, o, P2G_LANES);
    }
    if (lane == 0 && index < C) {
        u[index] = ws0 > 0.0f ? vs0 / ws0 : 0.0f;
        v[index] = ws1 > 0.0f ? vs1 / ws1 : 0.0f;
        w[index] = ws2 > 0.0f ? vs2 / ws2 : 0.0f;
        ff[index] = (float)inside * inv_ppc;
    }
}

// The same gather with the lanes laid out by warp: block b handles cells 32 b .. 32 b + 31, warp w
// is lane w of all 32 cells (thread t of the warp: cell 32 b + t). The warp's threads then visit bins
// with the same offset at the same time, so the exact-zero cases above are uniform across the warp:
// a bin one above the cell on exactly one axis feeds only that axis's face component and never the
// inside count, and it skips the other two components' weights and the count. Each lane still
// visits bins w, w+8, w+16, w+24 and their particles in order and accumulates as above; the eight
// partial sums of a cell are combined in shared memory in the order of the offset-4, 2, 1 tree
// ((l0 + l4) + (l2 + l6)) + ((l1 + l5) + (l3 + l7)), so the values are the same as p2g_cell's.
__global__ void __launch_bounds__(P2G_THREADS) k_p2g_gather(const float* __restrict__ pos, const float* __restrict__ vel,
                                                             const int* __restrict__ offsets,
                                                             const int* __restrict__ counts, float* __restrict__ u,
                                                             float* __restrict__ v, float* __restrict__ w,
                                                             float* __restrict__ ff, float inv_dx, float inv_ppc,
                                                             int nx, int ny, int nz) {
    __shared__ float s_sum[6][P2G_LANES][32];
    __shared__ int s_inside[P2G_LANES][32];
    const i64 C = (i64)nx * ny * nz;
    const int lane = threadIdx.x >> 5, t = threadIdx.x & 31;
    const i64 index = (i64)blockIdx.x * 32 + t;
    float vs0 = 0.0f, vs1 = 0.0f, vs2 = 0.0f, ws0 = 0.0f, ws1 = 0.0f, ws2 = 0.0f;
    int inside = 0;
    if (index < C) {
        int ci, cj, ck;
        gcoord(index, ny, nz, ci, cj, ck);
        const float gx = (float)ci, gy = (float)cj, gz = (float)ck;
        const float x1 = gx + 1.0f, xh = gx + 0.5f, y1 = gy + 1.0f, yh = gy + 0.5f, z1 = gz + 1.0f, zh = gz + 0.5f;
        for (int nb = lane; nb < 27; nb += P2G_LANES) {  // the same nb in the whole warp
            const int ox = nb / 9 - 1, oy = (nb / 3) % 3 - 1, oz = nb % 3 - 1;
            const int up = (ox > 0) + (oy > 0) + (oz > 0);
            if (up >= 2) continue;  // every weight of this bin is zero
            const bool du = oy <= 0 && oz <= 0, dv = ox <= 0 && oz <= 0, dw = ox <= 0 && oy <= 0, din = up == 0;
            const int bx = ci + ox, by = cj + oy, bz = ck + oz;
            if (bx < 0 || bx >= nx - 1 || by < 0 || by >= ny - 1 || bz < 0 || bz >= nz - 1) continue;
            const i64 bin = gidx(bx, by, bz, ny, nz);
            const int begin = __ldg(offsets + bin);
            const int end = begin + __ldg(counts + bin);
            for (int q = begin; q < end; ++q) {
                const float* P = pos + 3 * (i64)q;
                const float* V = vel + 3 * (i64)q;
                const float s0 = __ldg(P) * inv_dx, s1 = __ldg(P + 1) * inv_dx, s2 = __ldg(P + 2) * inv_dx;
                if (din) {
                    const int pc0 = clampi((int)s0, 1, nx - 2);
                    const int pc1 = clampi((int)s1, 1, ny - 2);
                    const int pc2 = clampi((int)s2, 1, nz - 2);
                    inside += (pc0 == ci && pc1 == cj && pc2 == ck) ? 1 : 0;
                }
                if (du) {
                    const float wu = tent(s0, x1) * tent(s1, yh) * tent(s2, zh);
                    vs0 += wu * __ldg(V);
                    ws0 += wu;
                }
                if (dv) {
                    const float wv = tent(s0, xh) * tent(s1, y1) * tent(s2, zh);
                    vs1 += wv * __ldg(V + 1);
                    ws1 += wv;
                }
                if (dw) {
                    const float ww = tent(s0, xh) * tent(s1, yh) * tent(s2, z1);
                    vs2 += ww * __ldg(V + 2);
                    ws2 += ww;
                }
            }
        }
    }
    s_sum[0][lane][t] = vs0;
    s_sum[1][lane][t] = vs1;
    s_sum[2][lane][t] = vs2;
    s_sum[3][lane][t] = ws0;
    s_sum[4][lane][t] = ws1;
    s_sum[5][lane][t] = ws2;
    s_inside[lane][t] = inside;
    __syncthreads();
    if (lane == 0 && index < C) {
        float r[6];
#pragma unroll
        for (int a = 0; a < 6; ++a) {
            const float* l = &s_sum[a][0][t];
            r[a] = ((l[0] + l[4 * 32]) + (l[2 * 32] + l[6 * 32])) + ((l[1 * 32] + l[5 * 32]) + (l[3 * 32] + l[7 * 32]));
        }
        int n = 0;
#pragma unroll
        for (int q = 0; q < P2G_LANES; ++q) n += s_inside[q][t];
        u[index] = r[3] > 0.0f ? r[0] / r[3] : 0.0f;
        v[index] = r[4] > 0.0f ? r[1] / r[4] : 0.0f;
        w[index] = r[5] > 0.0f ? r[2] / r[5] : 0.0f;
        ff[index] = (float)n * inv_ppc;
    }
}

}  // namespace clb
