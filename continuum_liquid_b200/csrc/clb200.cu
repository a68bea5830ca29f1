// libclb200.so: C ABI entry points (include/clb200.h). Unity build: the kernels live in the headers
// included below; this file validates arguments, picks launch shapes and enqueues the kernels.
#include "../../include/clb200.h"
#include "binning.cuh"
#include "p2g_tiled.cuh"
#include "particles.cuh"
#include "g2p_tiled.cuh"
#include "grid.cuh"
#include "multigrid.cuh"
#include "mg_bottom.cuh"
#include "mg_sweep.cuh"
#include "mg_half.cuh"
#include "mg_cluster.cuh"
#include "mg_tiles.cuh"
#include "mg_level0.cuh"
#include "batch.cuh"
#include "sources.cuh"
#include "voxelise.cuh"
#include "tc_gemm.cuh"
#include "conv3d.cuh"
#include "conv_win.cuh"

#include <mutex>

using namespace clb;

#define CLB_STREAM(s) (reinterpret_cast<cudaStream_t>(s))
#define CLB_GRID_ARGS_OK(nx, ny, nz)                                                                   \
    CLB_REQUIRE((nx) >= 3 && (ny) >= 3 && (nz) >= 3, "grid %dx%dx%d: every dimension must be >= 3", (nx), (ny), \
                (nz));                                                                                 \
    CLB_REQUIRE((i64)(nx) * (ny) * (nz) < (1ll << 31), "grid %dx%dx%d has more than 2^31 cells", (nx), (ny), (nz))

static const int kAbiVersion = 8;
static const size_t kBottomSmemLimit = 220 * 1024;
static bool g_use_bottom = true;  // clb_mg_set_option(0, ...) switches the single-block bottom visit off
static bool g_use_cluster = true;  // clb_mg_set_option(2, ...) switches the cluster visit off
static int g_single_from = 0;      // clb_mg_set_option(4, l): levels >= l (> 0) are visited once per parent visit

// Visits of `level` per visit of the level above: the reference's two, or one from the single-visit level on.
static inline int visits_of(int level) { return g_single_from > 0 && level >= g_single_from ? 1 : 2; }
static bool g_skip_air = true;     // clb_mg_set_option(3, ...): refinement/FCG steps skip cells without fluid

template <bool L0, bool H, int TI, int TJ, int T>
static cudaError_t rbgs_iter_attr_one() {
    return cudaFuncSetAttribute(k_rbgs_iter<L0, H, TI, TJ, 32, T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)SweepTile<L0, H, TI, TJ, 32, T>::smem());
}
// every tile and iteration count dispatched for one level kind (FP32 coarse levels have no
// two-iteration 8 x 8 x 32 tile: its staged operator would exceed the shared memory)
template <bool L0, bool H>
static cudaError_t rbgs_iter_attr() {
    cudaError_t e = rbgs_iter_attr_one<L0, H, 4, 4, 1>();
    e = e != cudaSuccess ? e : rbgs_iter_attr_one<L0, H, 4, 4, 2>();
    e = e != cudaSuccess ? e : rbgs_iter_attr_one<L0, H, 8, 8, 1>();
    if (L0 || H) e = e != cudaSuccess ? e : rbgs_iter_attr_one<L0, H, 8, 8, (L0 || H) ? 2 : 1>();
    return e;
}

template <int NS, int KA, int KB, bool H>
static cudaError_t cluster_visit_attr_one() {
    cudaError_t e = cudaFuncSetAttribute(k_cluster_visit<NS, KA, KB, H>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)kBottomSmemLimit);
    return e != cudaSuccess ? e
                            : cudaFuncSetAttribute(k_cluster_visit<NS, KA, KB, H>,
                                                   cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
}
template <bool H>
static cudaError_t cluster_visit_attr() {
    cudaError_t e = cluster_visit_attr_one<2, 4, 1, H>();
    e = e != cudaSuccess ? e : cluster_visit_attr_one<4, 4, 1, H>();
    e = e != cudaSuccess ? e : cluster_visit_attr_one<8, 4, 1, H>();
    e = e != cudaSuccess ? e : cluster_visit_attr_one<4, 2, 1, H>();
    return e;
}

template <int N, bool DG>
static cudaError_t conv_win_attr() {
    return cudaFuncSetAttribute(conv::k_conv_win<N, DG>, cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024);
}
template <int N>
static cudaError_t conv_wgrad_attr() {
    return cudaFuncSetAttribute(conv::k_conv_wgrad<N>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)tc::tile_smem_bytes<N>());
}
static int conv_set_attributes() {
    cudaError_t e = cudaSuccess;
    e = e != cudaSuccess ? e : conv_win_attr<16, false>();
    e = e != cudaSuccess ? e : conv_win_attr<32, false>();
    e = e != cudaSuccess ? e : conv_win_attr<64, false>();
    e = e != cudaSuccess ? e : conv_win_attr<16, true>();
    e = e != cudaSuccess ? e : conv_win_attr<32, true>();
    e = e != cudaSuccess ? e : conv_win_attr<48, true>();
    e = e != cudaSuccess ? e : conv_win_attr<64, true>();
    e = e != cudaSuccess ? e : conv_win_attr<96, true>();
    e = e != cudaSuccess ? e : conv_wgrad_attr<16>();
    e = e != cudaSuccess ? e : conv_wgrad_attr<32>();
    e = e != cudaSuccess ? e : conv_wgrad_attr<64>();
    return check_call(e, "convolution attributes");
}

extern "C" {

int clb_abi_version(void) { return kAbiVersion; }

int64_t clb_launch_count(void) { return (int64_t)g_launches.load(std::memory_order_relaxed); }

const char* clb_last_error(void) { return t_last_error; }

int clb_init(int device) {
    int count = 0;
    if (check_call(cudaGetDeviceCount(&count), "cudaGetDeviceCount")) return 1;
    CLB_REQUIRE(device >= 0 && device < count, "device %d not present (%d CUDA devices)", device, count);
    if (check_call(cudaSetDevice(device), "cudaSetDevice")) return 1;
    cudaDeviceProp prop;
    if (check_call(cudaGetDeviceProperties(&prop, device), "cudaGetDeviceProperties")) return 1;
    CLB_REQUIRE(prop.major == 10 && prop.minor == 0,
                "device %d is sm_%d%d; this library is built for sm_100a (B200) only", device, prop.major, prop.minor);
    g_sm_count = prop.multiProcessorCount;
    const int smem_max = (int)coarse_smem_bytes(COARSE_SMEM_CELLS);
    if (check_call(cudaFuncSetAttribute(k_coarse_solve<true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        smem_max),
                   "coarse solve attribute"))
        return 1;
    if (check_call(cudaFuncSetAttribute(k_coarse_solve<true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        smem_max),
                   "coarse solve attribute"))
        return 1;
    if (check_call(cudaFuncSetAttribute(k_coarse_solve<true, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        smem_max),
                   "coarse solve attribute"))
        return 1;
    const int bottom_max = (int)kBottomSmemLimit;
    cudaError_t e = cudaSuccess;
    // the fused sweeps stage more than the default 48 KB of shared memory
    e = e != cudaSuccess ? e : rbgs_iter_attr<true, false>();
    e = e != cudaSuccess ? e : rbgs_iter_attr<false, false>();
    e = e != cudaSuccess ? e : rbgs_iter_attr<false, true>();
    e = e != cudaSuccess ? e : cluster_visit_attr<false>();
    e = e != cudaSuccess ? e : cluster_visit_attr<true>();
    e = e != cudaSuccess ? e : cudaFuncSetAttribute(k_bottom_visit<1, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, bottom_max);
    e = e != cudaSuccess ? e : cudaFuncSetAttribute(k_bottom_visit<2, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, bottom_max);
    e = e != cudaSuccess ? e : cudaFuncSetAttribute(k_bottom_visit<4, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, bottom_max);
    e = e != cudaSuccess ? e : cudaFuncSetAttribute(k_bottom_visit<4, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, bottom_max);
    e = e != cudaSuccess ? e : cudaFuncSetAttribute(k_bottom_visit<8, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, bottom_max);
    e = e != cudaSuccess ? e : cudaFuncSetAttribute(k_bottom_visit<1, 1, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, bottom_max);
    e = e != cudaSuccess ? e : cudaFuncSetAttribute(k_bottom_visit<2, 1, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, bottom_max);
    e = e != cudaSuccess ? e : cudaFuncSetAttribute(k_bottom_visit<4, 1, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, bottom_max);
    e = e != cudaSuccess ? e : cudaFuncSetAttribute(k_bottom_visit<4, 2, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, bottom_max);
    e = e != cudaSuccess ? e : cudaFuncSetAttribute(k_bottom_visit<8, 4, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, bottom_max);
    e = e != cudaSuccess ? e : cudaFuncSetAttribute(kb_bottom_visit<1, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, bottom_max);
    e = e != cudaSuccess ? e : cudaFuncSetAttribute(kb_bottom_visit<2, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, bottom_max);
    e = e != cudaSuccess ? e : cudaFuncSetAttribute(kb_bottom_visit<4, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, bottom_max);
    e = e != cudaSuccess ? e : cudaFuncSetAttribute(kb_bottom_visit<4, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, bottom_max);
    e = e != cudaSuccess ? e : cudaFuncSetAttribute(kb_bottom_visit<8, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, bottom_max);
    e = e != cudaSuccess ? e : cudaFuncSetAttribute(kb_coarse_solve, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_max);
    if (check_call(e, "bottom visit attribute")) return 1;
    if (check_call(cudaFuncSetAttribute(k_p2g_tiled, cudaFuncAttributeMaxDynamicSharedMemorySize, P2GT_SMEM),
                   "tiled P2G attribute") ||
        check_call(cudaFuncSetAttribute(kb_p2g_tiled, cudaFuncAttributeMaxDynamicSharedMemorySize, P2GT_SMEM),
                   "batched tiled P2G attribute") ||
        check_call(cudaFuncSetAttribute(k_particle_update_tiled<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        PUT_SMEM),
                   "tiled particle update attribute") ||
        check_call(cudaFuncSetAttribute(k_particle_update_tiled<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        PUT_SMEM),
                   "tiled particle update attribute"))
        return 1;
    e = cudaFuncSetAttribute(k_l0_iter_tiles<L0F_ZERO | L0F_RESTRICT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)L0Region<3>::smem());
    e = e != cudaSuccess ? e : cudaFuncSetAttribute(k_l0_iter_tiles<L0F_RESTRICT>,
                                                    cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                    (int)L0Region<3>::smem());
    e = e != cudaSuccess ? e : cudaFuncSetAttribute(k_l0_iter_tiles<L0F_ZERO>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                    (int)L0Region<2>::smem());
    e = e != cudaSuccess ? e : cudaFuncSetAttribute(k_l0_iter_tiles<0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                    (int)L0Region<2>::smem());
    e = e != cudaSuccess ? e : cudaFuncSetAttribute(k_l0_iter_tiles<L0F_PROLONG>,
                                                    cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                    (int)L0Region<2>::smem());
    if (check_call(e, "level-0 fused iteration attribute")) return 1;
    if (conv_set_attributes()) return 1;
    return 0;
}

int clb_device_error(uint32_t* code) {
    CLB_REQUIRE(code != nullptr, "clb_device_error: null output");
    unsigned int v = 0, zero = 0;
    if (check_call(cudaMemcpyFromSymbol(&v, g_device_error, sizeof(v)), "read device error")) return 1;
    if (check_call(cudaMemcpyToSymbol(g_device_error, &zero, sizeof(zero)), "clear device error")) return 1;
    *code = v;
    return 0;
}

// ---- particles --------------------------------------------------------------------------------

int clb_count_particles_per_cell(const float* particles, int32_t* bin_counts, int32_t* keys, int32_t* ranks,
                                 int64_t n, float inv_dx, int nx, int ny, int nz, void* stream) {
    CLB_GRID_ARGS_OK(nx, ny, nz);
    CLB_REQUIRE(n >= 0 && n < (1ll << 31), "count_particles_per_cell: n=%lld out of range", (long long)n);
    if (n == 0) return 0;
    CLB_REQUIRE(particles && bin_counts, "count_particles_per_cell: null pointer");
    k_bin_count<<<blocks_for(n, PT), PT, 0, CLB_STREAM(stream)>>>(particles, n, inv_dx, nx, ny, nz, bin_counts, keys,
                                                                   ranks);
    CLB_LAUNCH_CHECK("k_bin_count");
    return 0;
}

int64_t clb_scan_scratch_bytes(int64_t count) { return scan_scratch_bytes(count); }

int clb_exclusive_prefix_sum(const int32_t* values, int32_t* output, int32_t* total, int64_t count, void* scratch,
                             int64_t scratch_bytes, void* stream) {
    CLB_REQUIRE(count >= 0, "exclusive_prefix_sum: negative count");
    CLB_REQUIRE(count == 0 || (values && output), "exclusive_prefix_sum: null pointer");
    return launch_scan(values, output, count, scratch, scratch_bytes, total, CLB_STREAM(stream));
}

// ---- exclusive scan with library-owned scratch --------------------------------------------------
// Some callers cannot allocate device memory: a host application that has handed the whole device
// memory budget to its own pool, or code that must not add the device-wide synchronisation that
// cudaMalloc/cudaFree imply in the middle of asynchronous work. For them this variant keeps the
// scan's look-back state (a 16-byte ticket header and one 8-byte status word per 4096-element tile)
// in a fixed array compiled into the library, sized for CLB_SCAN_STATIC_MAX_COUNT elements:
// 16 + 8 * 16384 bytes, held on every GPU that loads the library until the process exits.
//
// In host code the array's name only stands for it; its device address is obtained once per device
// with cudaGetSymbolAddress, on the first call made while that device is current, and kept for the
// life of the process (a device reset would invalidate it; the header tells callers not to reset).
static constexpr i64 kScanStaticTiles = (CLB_SCAN_STATIC_MAX_COUNT + SCAN_TILE - 1) / SCAN_TILE;
static __device__ __align__(256) unsigned char g_scan_static_scratch[16 + 8 * kScanStaticTiles];
static std::mutex g_scan_static_mutex;
static void* g_scan_static_address[256] = {};  // per device ordinal

int clb_exclusive_prefix_sum_static(const int32_t* values, int32_t* output, int32_t* total, int64_t count,
                                    void* stream) {
    CLB_REQUIRE(count >= 0, "exclusive_prefix_sum_static: negative count");
    CLB_REQUIRE(count <= CLB_SCAN_STATIC_MAX_COUNT,
                "exclusive_prefix_sum_static: %lld elements exceed the fixed scratch limit of %lld elements; "
                "use clb_exclusive_prefix_sum with caller-provided scratch",
                (long long)count, (long long)CLB_SCAN_STATIC_MAX_COUNT);
    CLB_REQUIRE(count == 0 || (values && output), "exclusive_prefix_sum_static: null pointer");
    int device = 0;
    if (check_call(cudaGetDevice(&device), "exclusive_prefix_sum_static: cudaGetDevice")) return 1;
    CLB_REQUIRE(device >= 0 && device < 256, "exclusive_prefix_sum_static: device ordinal %d out of range", device);
    void* scratch = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_scan_static_mutex);
        if (g_scan_static_address[device] == nullptr) {
            void* address = nullptr;
            if (check_call(cudaGetSymbolAddress(&address, g_scan_static_scratch),
                           "exclusive_prefix_sum_static: cudaGetSymbolAddress"))
                return 1;
            g_scan_static_address[device] = address;
        }
        scratch = g_scan_static_address[device];
    }
    // launch_scan clears the ticket and the status words this count uses before the scan runs
    return launch_scan(values, output, count, scratch, (i64)sizeof(g_scan_static_scratch), total,
                       CLB_STREAM(stream));
}

int clb_sort_particles(const float* particles, const float* velocity, float* particles_sorted, float* velocity_sorted,
                       const int32_t* bin_offsets, const int32_t* bin_counts, const int32_t* keys,
                       const int32_t* ranks, int32_t* perm, int32_t* slot_keys, int64_t n, void* stream) {
    CLB_REQUIRE(n >= 0 && n < (1ll << 31), "sort_particles: n=%lld out of range", (long long)n);
    if (n == 0) return 0;
    CLB_REQUIRE(particles && velocity && particles_sorted && velocity_sorted && bin_offsets && bin_counts && keys &&
                    ranks && perm && slot_keys,
                "sort_particles: null pointer");
    cudaStream_t s = CLB_STREAM(stream);
    k_scatter_perm<<<blocks_for(n, PT), PT, 0, s>>>(keys, ranks, bin_offsets, n, perm, slot_keys);
    CLB_LAUNCH_CHECK("k_scatter_perm");
    k_stable_gather<<<blocks_for(n, PT), PT, 0, s>>>(perm, slot_keys, bin_offsets, bin_counts, particles, velocity, n,
                                                      particles_sorted, velocity_sorted);
    CLB_LAUNCH_CHECK("k_stable_gather");
    return 0;
}

int clb_particle_to_grid_gather(const float* particles, const float* velocity, const int32_t* bin_offsets,
                                const int32_t* bin_counts, float* u, float* v, float* w, float* fluid_fraction,
                                float inv_dx, float inv_particles_per_cell, int nx, int ny, int nz, void* stream) {
    CLB_GRID_ARGS_OK(nx, ny, nz);
    CLB_REQUIRE(bin_offsets && bin_counts && u && v && w && fluid_fraction, "particle_to_grid_gather: null pointer");
    const i64 C = (i64)nx * ny * nz;
    k_p2g_gather<<<blocks_for(C * P2G_LANES, P2G_THREADS), P2G_THREADS, 0, CLB_STREAM(stream)>>>(
        particles, velocity, bin_offsets, bin_counts, u, v, w, fluid_fraction, inv_dx, inv_particles_per_cell, nx, ny,
        nz);
    CLB_LAUNCH_CHECK("k_p2g_gather");
    return 0;
}

int clb_particle_to_grid_gather_tiled(const float* particles, const float* velocity, const int32_t* bin_offsets,
                                      const int32_t* bin_counts, float* u, float* v, float* w, float* fluid_fraction,
                                      float inv_dx, float inv_particles_per_cell, int nx, int ny, int nz,
                                      void* stream) {
    CLB_GRID_ARGS_OK(nx, ny, nz);
    CLB_REQUIRE(bin_offsets && bin_counts && u && v && w && fluid_fraction,
                "particle_to_grid_gather_tiled: null pointer");
    int tiles_j = 0, tiles_k = 0;
    const int tiles = p2g_tiled_tiles(nx, ny, nz, &tiles_j, &tiles_k);
    k_p2g_tiled<<<tiles, P2GT_THREADS, P2GT_SMEM, CLB_STREAM(stream)>>>(particles, velocity, bin_offsets, bin_counts,
                                                                          u, v, w, fluid_fraction, inv_dx,
                                                                          inv_particles_per_cell, nx, ny, nz, tiles_j,
                                                                          tiles_k);
    CLB_LAUNCH_CHECK("k_p2g_tiled");
    return 0;
}

static int particle_to_grid_impl(const float* particles, const float* velocity, float* particles_work,
                                 float* velocity_work, float* u, float* v, float* w, float* fluid_fraction,
                                 int32_t* bin_counts, int32_t* bin_offsets, int32_t* keys, int32_t* ranks,
                                 int32_t* perm, int32_t* slot_keys, void* scan_scratch, int64_t scan_scratch_bytes_,
                                 int64_t n, float inv_dx, float inv_ppc, int nx, int ny, int nz, void* stream,
                                 bool tiled) {
    CLB_GRID_ARGS_OK(nx, ny, nz);
    CLB_REQUIRE(inv_dx > 0.0f && inv_ppc > 0.0f, "particle_to_grid: inv_dx and inv_particles_per_cell must be > 0");
    CLB_REQUIRE(n >= 0 && n < (1ll << 31), "particle_to_grid: n=%lld out of range", (long long)n);
    cudaStream_t s = CLB_STREAM(stream);
    const i64 C = (i64)nx * ny * nz;
    if (check_call(cudaMemsetAsync(bin_counts, 0, sizeof(int32_t) * C, s), "zero bin_counts")) return 1;
    if (clb_count_particles_per_cell(particles, bin_counts, keys, ranks, n, inv_dx, nx, ny, nz, stream)) return 1;
    if (clb_exclusive_prefix_sum(bin_counts, bin_offsets, nullptr, C, scan_scratch, scan_scratch_bytes_, stream))
        return 1;
    if (clb_sort_particles(particles, velocity, particles_work, velocity_work, bin_offsets, bin_counts, keys, ranks,
                           perm, slot_keys, n, stream))
        return 1;
    if (tiled)
        return clb_particle_to_grid_gather_tiled(particles_work, velocity_work, bin_offsets, bin_counts, u, v, w,
                                                 fluid_fraction, inv_dx, inv_ppc, nx, ny, nz, stream);
    return clb_particle_to_grid_gather(particles_work, velocity_work, bin_offsets, bin_counts, u, v, w, fluid_fraction,
                                       inv_dx, inv_ppc, nx, ny, nz, stream);
}

int clb_particle_to_grid(const float* particles, const float* velocity, float* particles_work, float* velocity_work,
                         float* u, float* v, float* w, float* fluid_fraction, int32_t* bin_counts,
                         int32_t* bin_offsets, int32_t* keys, int32_t* ranks, int32_t* perm, int32_t* slot_keys,
                         void* scan_scratch, int64_t scan_scratch_bytes_, int64_t n, float inv_dx,
                         float inv_ppc, int nx, int ny, int nz, void* stream) {
    return particle_to_grid_impl(particles, velocity, particles_work, velocity_work, u, v, w, fluid_fraction,
                                 bin_counts, bin_offsets, keys, ranks, perm, slot_keys, scan_scratch,
                                 scan_scratch_bytes_, n, inv_dx, inv_ppc, nx, ny, nz, stream, false);
}

int clb_particle_to_grid_tiled(const float* particles, const float* velocity, float* particles_work,
                               float* velocity_work, float* u, float* v, float* w, float* fluid_fraction,
                               int32_t* bin_counts, int32_t* bin_offsets, int32_t* keys, int32_t* ranks,
                               int32_t* perm, int32_t* slot_keys, void* scan_scratch, int64_t scan_scratch_bytes_,
                               int64_t n, float inv_dx, float inv_ppc, int nx, int ny, int nz, void* stream) {
    return particle_to_grid_impl(particles, velocity, particles_work, velocity_work, u, v, w, fluid_fraction,
                                 bin_counts, bin_offsets, keys, ranks, perm, slot_keys, scan_scratch,
                                 scan_scratch_bytes_, n, inv_dx, inv_ppc, nx, ny, nz, stream, true);
}

int clb_grid_to_particle(float* velocity, const float* particles, const float* u, const float* v, const float* w,
                         const float* u_old, const float* v_old, const float* w_old, int64_t n, float inv_dx, int nx,
                         int ny, int nz, float flip_ratio, void* stream) {
    CLB_GRID_ARGS_OK(nx, ny, nz);
    CLB_REQUIRE(n >= 0, "grid_to_particle: negative n");
    if (n == 0) return 0;
    CLB_REQUIRE(velocity && particles && u && v && w && u_old && v_old && w_old, "grid_to_particle: null pointer");
    k_grid_to_particle<<<blocks_for(n, PT), PT, 0, CLB_STREAM(stream)>>>(velocity, particles, u, v, w, u_old, v_old,
                                                                          w_old, n, inv_dx, nx, ny, nz, flip_ratio);
    CLB_LAUNCH_CHECK("k_grid_to_particle");
    return 0;
}

int clb_advect_particles(float* particles, const float* velocity, int64_t n, float dt, void* stream) {
    CLB_REQUIRE(n >= 0, "advect_particles: negative n");
    if (n == 0) return 0;
    CLB_REQUIRE(particles && velocity, "advect_particles: null pointer");
    k_advect<<<blocks_for(3 * n, PT), PT, 0, CLB_STREAM(stream)>>>(particles, velocity, 3 * n, dt);
    CLB_LAUNCH_CHECK("k_advect");
    return 0;
}

int clb_particle_domain_bc(float* particles, float* velocity, int64_t n, float lower, float upper_x, float upper_y,
                           float upper_z, void* stream) {
    CLB_REQUIRE(n >= 0, "particle_domain_bc: negative n");
    if (n == 0) return 0;
    CLB_REQUIRE(particles && velocity, "particle_domain_bc: null pointer");
    k_particle_domain_bc<<<blocks_for(n, PT), PT, 0, CLB_STREAM(stream)>>>(particles, velocity, n, lower, upper_x,
                                                                            upper_y, upper_z);
    CLB_LAUNCH_CHECK("k_particle_domain_bc");
    return 0;
}

int clb_particle_obstacle_bc(float* particles, const float* previous, float* velocity, const uint8_t* obstacle,
                             int64_t n, float inv_dx, int nx, int ny, int nz, void* stream) {
    CLB_GRID_ARGS_OK(nx, ny, nz);
    CLB_REQUIRE(n >= 0, "particle_obstacle_bc: negative n");
    if (n == 0) return 0;
    CLB_REQUIRE(particles && previous && velocity && obstacle, "particle_obstacle_bc: null pointer");
    k_particle_obstacle_bc<false><<<blocks_for(n, PT), PT, 0, CLB_STREAM(stream)>>>(particles, previous, velocity, obstacle, n,
                                                                              inv_dx, nx, ny, nz);
    CLB_LAUNCH_CHECK("k_particle_obstacle_bc");
    return 0;
}

int clb_particle_update(float* particles, float* velocity, float* previous_out, const float* u, const float* v,
                        const float* w, const float* u_old, const float* v_old, const float* w_old,
                        const uint8_t* obstacle, int64_t n, float inv_dx, int nx, int ny, int nz, float flip_ratio,
                        float dt, float lower, float upper_x, float upper_y, float upper_z, void* stream) {
    CLB_GRID_ARGS_OK(nx, ny, nz);
    CLB_REQUIRE(n >= 0, "particle_update: negative n");
    if (n == 0) return 0;
    CLB_REQUIRE(particles && velocity && u && v && w && u_old && v_old && w_old, "particle_update: null pointer");
    k_particle_update<false><<<blocks_for(n, PT), PT, 0, CLB_STREAM(stream)>>>(
        particles, velocity, previous_out, u, v, w, u_old, v_old, w_old, obstacle, n, inv_dx, nx, ny, nz, flip_ratio,
        dt, lower, upper_x, upper_y, upper_z);
    CLB_LAUNCH_CHECK("k_particle_update");
    return 0;
}

static RigidMotion motion_of(const float* m) {
    return RigidMotion{m[0], m[1], m[2], m[3], m[4], m[5], m[6], m[7], m[8]};
}

int clb_particle_update_tiled(float* particles, float* velocity, float* previous_out, const float* u, const float* v,
                              const float* w, const float* u_old, const float* v_old, const float* w_old,
                              const uint8_t* obstacle, const int32_t* bin_offsets, const int32_t* bin_counts,
                              int64_t n, float inv_dx, int nx, int ny, int nz, float flip_ratio, float dt, float lower,
                              float upper_x, float upper_y, float upper_z, const float* motion, void* stream) {
    CLB_GRID_ARGS_OK(nx, ny, nz);
    CLB_REQUIRE(n >= 0 && n < (1ll << 31), "particle_update_tiled: n=%lld out of range", (long long)n);
    if (n == 0) return 0;
    CLB_REQUIRE(particles && velocity && u && v && w && u_old && v_old && w_old && bin_offsets && bin_counts,
                "particle_update_tiled: null pointer");
    CLB_REQUIRE(motion == nullptr || obstacle != nullptr, "particle_update_tiled: a motion needs an obstacle");
    int tiles_j = 0, tiles_k = 0;
    const int tiles = particle_update_tiles(nx, ny, nz, &tiles_j, &tiles_k);
    if (motion)
        k_particle_update_tiled<true><<<tiles, PUT_THREADS, PUT_SMEM, CLB_STREAM(stream)>>>(
            particles, velocity, previous_out, u, v, w, u_old, v_old, w_old, obstacle, bin_offsets, bin_counts, inv_dx,
            nx, ny, nz, flip_ratio, dt, lower, upper_x, upper_y, upper_z, tiles_j, tiles_k, motion_of(motion));
    else
        k_particle_update_tiled<false><<<tiles, PUT_THREADS, PUT_SMEM, CLB_STREAM(stream)>>>(
            particles, velocity, previous_out, u, v, w, u_old, v_old, w_old, obstacle, bin_offsets, bin_counts, inv_dx,
            nx, ny, nz, flip_ratio, dt, lower, upper_x, upper_y, upper_z, tiles_j, tiles_k, RigidMotion{});
    CLB_LAUNCH_CHECK("k_particle_update_tiled");
    return 0;
}

// ---- moving colliders (no counterpart in the reference) ------------------------------------------

int clb_particle_obstacle_bc_moving(float* particles, const float* previous, float* velocity,
                                    const uint8_t* obstacle, int64_t n, float inv_dx, int nx, int ny, int nz,
                                    const float* motion, void* stream) {
    CLB_GRID_ARGS_OK(nx, ny, nz);
    CLB_REQUIRE(n >= 0, "particle_obstacle_bc_moving: negative n");
    CLB_REQUIRE(motion != nullptr, "particle_obstacle_bc_moving: null motion");
    if (n == 0) return 0;
    CLB_REQUIRE(particles && previous && velocity && obstacle, "particle_obstacle_bc_moving: null pointer");
    k_particle_obstacle_bc<true><<<blocks_for(n, PT), PT, 0, CLB_STREAM(stream)>>>(
        particles, previous, velocity, obstacle, n, inv_dx, nx, ny, nz, motion_of(motion));
    CLB_LAUNCH_CHECK("k_particle_obstacle_bc");
    return 0;
}

int clb_particle_update_moving(float* particles, float* velocity, float* previous_out, const float* u, const float* v,
                               const float* w, const float* u_old, const float* v_old, const float* w_old,
                               const uint8_t* obstacle, int64_t n, float inv_dx, int nx, int ny, int nz,
                               float flip_ratio, float dt, float lower, float upper_x, float upper_y, float upper_z,
                               const float* motion, void* stream) {
    CLB_GRID_ARGS_OK(nx, ny, nz);
    CLB_REQUIRE(n >= 0, "particle_update_moving: negative n");
    CLB_REQUIRE(motion != nullptr && obstacle != nullptr, "particle_update_moving: null motion or obstacle");
    if (n == 0) return 0;
    CLB_REQUIRE(particles && velocity && u && v && w && u_old && v_old && w_old, "particle_update_moving: null pointer");
    k_particle_update<true><<<blocks_for(n, PT), PT, 0, CLB_STREAM(stream)>>>(
        particles, velocity, previous_out, u, v, w, u_old, v_old, w_old, obstacle, n, inv_dx, nx, ny, nz, flip_ratio,
        dt, lower, upper_x, upper_y, upper_z, motion_of(motion));
    CLB_LAUNCH_CHECK("k_particle_update");
    return 0;
}

int clb_grid_obstacle_bc_moving(float* u, float* v, float* w, float* fluid_fraction, const uint8_t* obstacle, int nx,
                                int ny, int nz, const float* motion, float dx, void* stream) {
    CLB_GRID_ARGS_OK(nx, ny, nz);
    CLB_REQUIRE(u && v && w && fluid_fraction && obstacle && motion, "grid_obstacle_bc_moving: null pointer");
    const i64 C = (i64)nx * ny * nz;
    cudaStream_t s = CLB_STREAM(stream);
    const RigidMotion m = motion_of(motion);
    k_grid_obstacle_bc_moving<<<blocks_for(C, 256), 256, 0, s>>>(u, v, w, fluid_fraction, obstacle, nx, ny, nz, m, dx);
    CLB_LAUNCH_CHECK("k_grid_obstacle_bc_moving");
    k_extrapolate_obstacle_velocity_moving<<<blocks_for(C, 256), 256, 0, s>>>(u, v, w, obstacle, nx, ny, nz, m, dx);
    CLB_LAUNCH_CHECK("k_extrapolate_obstacle_velocity_moving");
    return 0;
}

// ---- grid -------------------------------------------------------------------------------------

int clb_update_velocity(const float* u, const float* v, const float* w, float* result_u, float* result_v,
                        float* result_w, const float* fluid_fraction, float gravity_x, float gravity_y,
                        float gravity_z, float force_x, float force_y, float force_z, float rho, float nu,
                        float inv_dx2, float dt, int nx, int ny, int nz, void* stream) {
    CLB_GRID_ARGS_OK(nx, ny, nz);
    CLB_REQUIRE(u && v && w && result_u && result_v && result_w && fluid_fraction, "update_velocity: null pointer");
    const i64 C = (i64)nx * ny * nz;
    k_update_velocity<<<blocks_for(C, GT), GT, 0, CLB_STREAM(stream)>>>(u, v, w, result_u, result_v, result_w,
                                                                         fluid_fraction, gravity_x, gravity_y,
                                                                         gravity_z, force_x, force_y, force_z, rho, nu,
                                                                         inv_dx2, dt, nx, ny, nz);
    CLB_LAUNCH_CHECK("k_update_velocity");
    return 0;
}

int clb_grid_domain_bc(float* u, float* v, float* w, int nx, int ny, int nz, void* stream) {
    CLB_GRID_ARGS_OK(nx, ny, nz);
    CLB_REQUIRE(u && v && w, "grid_domain_bc: null pointer");
    const i64 C = (i64)nx * ny * nz;
    if (nx >= 3 && ny >= 3 && nz >= 3)  // the shell of cells the conditions change
        k_grid_domain_bc_shell<<<blocks_for(shell_cells(nx, ny, nz, 1, 2), GT), GT, 0, CLB_STREAM(stream)>>>(
            u, v, w, nx, ny, nz);
    else
        k_grid_domain_bc<<<blocks_for(C, GT), GT, 0, CLB_STREAM(stream)>>>(u, v, w, nx, ny, nz);
    CLB_LAUNCH_CHECK("k_grid_domain_bc");
    return 0;
}

int clb_grid_obstacle_bc(float* u, float* v, float* w, float* fluid_fraction, const uint8_t* obstacle, int nx, int ny,
                         int nz, void* stream) {
    CLB_GRID_ARGS_OK(nx, ny, nz);
    CLB_REQUIRE(u && v && w && fluid_fraction && obstacle, "grid_obstacle_bc: null pointer");
    const i64 C = (i64)nx * ny * nz;
    cudaStream_t s = CLB_STREAM(stream);
    k_grid_obstacle_bc<<<blocks_for(C, GT), GT, 0, s>>>(u, v, w, fluid_fraction, obstacle, nx, ny, nz);
    CLB_LAUNCH_CHECK("k_grid_obstacle_bc");
    k_extrapolate_obstacle_velocity<<<blocks_for(C, GT), GT, 0, s>>>(u, v, w, obstacle, nx, ny, nz);
    CLB_LAUNCH_CHECK("k_extrapolate_obstacle_velocity");
    return 0;
}

int clb_pressure_rhs(const float* u, const float* v, const float* w, const float* fluid_fraction, float* rhs,
                     float rho_over_dt, float inv_dx, int nx, int ny, int nz, void* stream) {
    CLB_GRID_ARGS_OK(nx, ny, nz);
    CLB_REQUIRE(u && v && w && fluid_fraction && rhs, "pressure_rhs: null pointer");
    const i64 C = (i64)nx * ny * nz;
    k_pressure_rhs<<<blocks_for(C, GT), GT, 0, CLB_STREAM(stream)>>>(u, v, w, fluid_fraction, rhs, rho_over_dt, inv_dx,
                                                                      nx, ny, nz);
    CLB_LAUNCH_CHECK("k_pressure_rhs");
    return 0;
}

extern "C++" {
template <typename PT>
static int pressure_correction_impl(float* u, float* v, float* w, const PT* pressure, float dt_over_rho,
                                    float inv_dx, int nx, int ny, int nz, void* stream) {
    CLB_GRID_ARGS_OK(nx, ny, nz);
    CLB_REQUIRE(u && v && w && pressure, "pressure_correction: null pointer");
    const i64 C = (i64)nx * ny * nz;
    launch(blocks_for(C, GT), GT, 0, CLB_STREAM(stream))(k_pressure_correction<PT>, u, v, w, pressure, dt_over_rho,
                                                         inv_dx, nx, ny, nz);
    CLB_LAUNCH_CHECK("k_pressure_correction");
    return 0;
}

template <typename PT>
static int neumann_domain_bc_impl(PT* pressure, int nx, int ny, int nz, void* stream) {
    CLB_GRID_ARGS_OK(nx, ny, nz);
    CLB_REQUIRE(pressure, "neumann_domain_bc: null pointer");
    const i64 C = (i64)nx * ny * nz;
    if (nx >= 2 && ny >= 2 && nz >= 2)  // the shell of non-interior cells
        launch(blocks_for(shell_cells(nx, ny, nz, 1, 1), GT), GT, 0, CLB_STREAM(stream))(
            k_neumann_domain_bc_shell<PT>, pressure, nx, ny, nz);
    else
        launch(blocks_for(C, GT), GT, 0, CLB_STREAM(stream))(k_neumann_domain_bc<PT>, pressure, nx, ny, nz);
    CLB_LAUNCH_CHECK("k_neumann_domain_bc");
    return 0;
}
}  // extern "C++"

int clb_pressure_correction(float* u, float* v, float* w, const float* pressure, float dt_over_rho, float inv_dx,
                            int nx, int ny, int nz, void* stream) {
    return pressure_correction_impl<float>(u, v, w, pressure, dt_over_rho, inv_dx, nx, ny, nz, stream);
}

int clb_pressure_correction_f64(float* u, float* v, float* w, const double* pressure, float dt_over_rho,
                                float inv_dx, int nx, int ny, int nz, void* stream) {
    return pressure_correction_impl<double>(u, v, w, pressure, dt_over_rho, inv_dx, nx, ny, nz, stream);
}

int clb_neumann_domain_bc(float* pressure, int nx, int ny, int nz, void* stream) {
    return neumann_domain_bc_impl<float>(pressure, nx, ny, nz, stream);
}

int clb_neumann_domain_bc_f64(double* pressure, int nx, int ny, int nz, void* stream) {
    return neumann_domain_bc_impl<double>(pressure, nx, ny, nz, stream);
}

// ---- multigrid: the reference's level arrays through the product kernels -----------------------

int clb_mg_pack_finest(const float* mask, const float* diagonal, const float* weight_x, const float* weight_y,
                       const float* weight_z, uint8_t* op0, int32_t* invalid, int nx, int ny, int nz, void* stream) {
    CLB_GRID_ARGS_OK(nx, ny, nz);
    CLB_REQUIRE(mask && diagonal && weight_x && weight_y && weight_z && op0 && invalid, "mg_pack_finest: null pointer");
    const i64 C = (i64)nx * ny * nz;
    k_pack_finest<<<blocks_for(C, MGT), MGT, 0, CLB_STREAM(stream)>>>(mask, diagonal, weight_x, weight_y, weight_z,
                                                                        op0, invalid, C);
    CLB_LAUNCH_CHECK("k_pack_finest");
    return 0;
}

int clb_mg_unpack_finest(const uint8_t* op0, float* diagonal, float* weight_x, float* weight_y, float* weight_z,
                         int nx, int ny, int nz, void* stream) {
    CLB_GRID_ARGS_OK(nx, ny, nz);
    CLB_REQUIRE(op0 && diagonal && weight_x && weight_y && weight_z, "mg_unpack_finest: null pointer");
    const i64 C = (i64)nx * ny * nz;
    k_unpack_finest<<<blocks_for(C, MGT), MGT, 0, CLB_STREAM(stream)>>>(op0, diagonal, weight_x, weight_y, weight_z, C);
    CLB_LAUNCH_CHECK("k_unpack_finest");
    return 0;
}

int clb_mg_pack_level(const float* mask, const float* diagonal, const float* weight_x, const float* weight_y,
                      const float* weight_z, float* op4, uint8_t* mask_out, int nx, int ny, int nz, void* stream) {
    CLB_GRID_ARGS_OK(nx, ny, nz);
    CLB_REQUIRE(mask && diagonal && weight_x && weight_y && weight_z && op4 && mask_out, "mg_pack_level: null pointer");
    CLB_REQUIRE((((uintptr_t)op4) & 15) == 0, "mg_pack_level: op4 must be 16-byte aligned");
    const i64 C = (i64)nx * ny * nz;
    k_pack_level<<<blocks_for(C, MGT), MGT, 0, CLB_STREAM(stream)>>>(mask, diagonal, weight_x, weight_y, weight_z,
                                                                       reinterpret_cast<float4*>(op4), mask_out, C);
    CLB_LAUNCH_CHECK("k_pack_level");
    return 0;
}

int clb_mg_unpack_level(const float* op4, const uint8_t* mask_in, float* mask, float* diagonal, float* weight_x,
                        float* weight_y, float* weight_z, int nx, int ny, int nz, void* stream) {
    CLB_GRID_ARGS_OK(nx, ny, nz);
    CLB_REQUIRE(op4 && mask_in && mask && diagonal && weight_x && weight_y && weight_z, "mg_unpack_level: null pointer");
    CLB_REQUIRE((((uintptr_t)op4) & 15) == 0, "mg_unpack_level: op4 must be 16-byte aligned");
    const i64 C = (i64)nx * ny * nz;
    k_unpack_level<<<blocks_for(C, MGT), MGT, 0, CLB_STREAM(stream)>>>(reinterpret_cast<const float4*>(op4), mask_in,
                                                                         mask, diagonal, weight_x, weight_y, weight_z,
                                                                         C);
    CLB_LAUNCH_CHECK("k_unpack_level");
    return 0;
}

int clb_mg_smooth_level(float* p, const float* b, const float* op4, const uint8_t* mask, float delta, int iterations,
                        int nx, int ny, int nz, void* stream) {
    CLB_GRID_ARGS_OK(nx, ny, nz);
    CLB_REQUIRE(iterations >= 0, "mg_smooth_level: negative iterations");
    CLB_REQUIRE(p && b && op4 && mask, "mg_smooth_level: null pointer");
    CLB_REQUIRE((((uintptr_t)op4) & 15) == 0, "mg_smooth_level: op4 must be 16-byte aligned");
    const i64 C = (i64)nx * ny * nz;
    const float4* opc = reinterpret_cast<const float4*>(op4);
    cudaStream_t s = CLB_STREAM(stream);
    for (int it = 0; it < iterations; ++it)
        for (int parity = 0; parity < 2; ++parity) {
            launch(blocks_for(C, MGT), MGT, 0, s)(k_rbgs<false>, p, b, (const uint8_t*)nullptr, opc, mask, delta,
                                                  parity, nx, ny, nz);
            CLB_LAUNCH_CHECK("k_rbgs");
        }
    return 0;
}

int clb_mg_coarse_solve_level(float* p, const float* b, const float* op4, const uint8_t* mask, float delta,
                              int iterations, int nx, int ny, int nz, void* stream) {
    CLB_GRID_ARGS_OK(nx, ny, nz);
    CLB_REQUIRE(iterations >= 0, "mg_coarse_solve_level: negative iterations");
    CLB_REQUIRE(p && b && op4 && mask, "mg_coarse_solve_level: null pointer");
    CLB_REQUIRE((((uintptr_t)op4) & 15) == 0, "mg_coarse_solve_level: op4 must be 16-byte aligned");
    const i64 C = (i64)nx * ny * nz;
    CLB_REQUIRE(C < (1ll << 31), "mg_coarse_solve_level: level too large");
    const float4* opc = reinterpret_cast<const float4*>(op4);
    cudaStream_t s = CLB_STREAM(stream);
    if (C <= COARSE_SMEM_CELLS)
        launch(1, COARSE_THREADS, coarse_smem_bytes((int)C), s)(k_coarse_solve<true, false>, p, b,
                                                                (const uint8_t*)nullptr, opc, mask, delta, iterations,
                                                                nx, ny, nz, (const float*)nullptr);
    else
        launch(1, COARSE_THREADS, 0, s)(k_coarse_solve<false, false>, p, b, (const uint8_t*)nullptr, opc, mask, delta,
                                        iterations, nx, ny, nz, (const float*)nullptr);
    CLB_LAUNCH_CHECK("k_coarse_solve");
    return 0;
}

// ---- multigrid, packed layout ---------------------------------------------------------------------

int clb_mg_rhs_operator(const float* u, const float* v, const float* w, const float* fluid_fraction, float* rhs,
                        uint8_t* op0, float rho_over_dt, float inv_dx, int nx, int ny, int nz, void* stream) {
    CLB_GRID_ARGS_OK(nx, ny, nz);
    CLB_REQUIRE(u && v && w && fluid_fraction && rhs && op0, "mg_rhs_operator: null pointer");
    const i64 C = (i64)nx * ny * nz;
    launch(blocks_for(C, MGT), MGT, 0, CLB_STREAM(stream))(k_rhs_op0, u, v, w, fluid_fraction, rhs, op0, rho_over_dt,
                                                           inv_dx, nx, ny, nz);
    CLB_LAUNCH_CHECK("k_rhs_op0");
    return 0;
}

static int check_hierarchy(const clb_mg_hierarchy* h) {
    CLB_REQUIRE(h != nullptr, "multigrid: null hierarchy");
    CLB_REQUIRE(h->levels >= 1 && h->levels <= CLB_MG_MAX_LEVELS, "multigrid: %d levels (1..%d allowed)", h->levels,
                CLB_MG_MAX_LEVELS);
    CLB_REQUIRE(h->op0 != nullptr, "multigrid: null level-0 operator");
    for (int l = 0; l < h->levels; ++l) {
        CLB_GRID_ARGS_OK(h->shape[l][0], h->shape[l][1], h->shape[l][2]);
        if (l > 0)
            CLB_REQUIRE(h->p[l] && h->b[l] && h->mask[l] && h->op[l], "multigrid: level %d has a null array", l);
    }
    if (h->fp16_level != 0) {
        CLB_REQUIRE(h->fp16_level >= 1 && h->fp16_level <= h->levels - 2,
                    "multigrid: fp16_level %d outside 1..levels-2 (%d)", h->fp16_level, h->levels - 2);
        CLB_REQUIRE(h->fp16_scale && h->fp16_inexact, "multigrid: FP16 levels need fp16_scale and fp16_inexact");
        const int* c = h->shape[h->levels - 1];
        CLB_REQUIRE(c[0] * c[1] * c[2] <= COARSE_SMEM_CELLS, "multigrid: FP16 coarsest level too large (%d cells)",
                    c[0] * c[1] * c[2]);
    }
    return 0;
}

static inline bool is_half(const clb_mg_hierarchy* h, int l) { return h->fp16_level > 0 && l >= h->fp16_level; }
// The factor of every prolonged correction (clb_mg_hierarchy.prolong_scale; 0 reads as 1).
static inline float pscale(const clb_mg_hierarchy* h) { return h->prolong_scale > 0.0f ? h->prolong_scale : 1.0f; }

// The cluster launch that runs the visits of the third-coarsest level `level` with both bottom levels
// (mg_cluster.cuh), whatever the launch options: false when these levels cannot run as one (their
// storage types differ, or they do not fit).
struct ClusterShape {
    int cs;        // slab CTAs (the cluster has cs + 1)
    int ka, ns;    // A slots and C slots of each colour per thread
    size_t bytes;  // dynamic shared memory per CTA
    bool half;
};

static bool cluster_shape(const clb_mg_hierarchy* h, int level, ClusterShape& out) {
    if (level < 1 || level != h->levels - 3) return false;
    const bool half = is_half(h, level);
    if (is_half(h, level + 1) != half || is_half(h, level + 2) != half) return false;
    const int* c = h->shape[level];
    const int* a = h->shape[level + 1];
    const int* b = h->shape[level + 2];
    const int sa = colour_slots(a[0], a[1], a[2]), sb = colour_slots(b[0], b[1], b[2]);
    const int ka = (sa + BOTTOM_THREADS - 1) / BOTTOM_THREADS, kb = (sb + BOTTOM_BTHREADS - 1) / BOTTOM_BTHREADS;
    if (kb > 1 || ka > 4) return false;
    const int pairs = (c[0] - 1) / 2;
    const int cs = pairs < CLUSTER_MAX - 1 ? pairs : CLUSTER_MAX - 1;
    if (cs < 1) return false;
    const ClusterLayout L = cluster_layout(cs, c[0], c[1], c[2], half);
    const size_t bottom = bottom_smem_bytes(a[0] * a[1] * a[2], b[0] * b[1] * b[2]);
    const size_t bytes = L.slab_bytes > bottom ? L.slab_bytes : bottom;
    if (bytes > kBottomSmemLimit) return false;
    const long long slots = (long long)L.own_max * (c[1] - 2) * ((c[2] - 1) / 2);
    const int ns = (int)((slots + BOTTOM_THREADS - 1) / BOTTOM_THREADS);
    if (ns > 8) return false;
    out = ClusterShape{cs, ka, ns, bytes, half};
    return true;
}

static int64_t cluster_list_ints(const clb_mg_hierarchy* h, const ClusterShape& cl) {
    const int level = h->levels - 3;
    const int* c = h->shape[level];
    const int* a = h->shape[level + 1];
    const int* b = h->shape[level + 2];
    return cluster_lists_bottom_ints(a[0] * a[1] * a[2], b[0] * b[1] * b[2]) +
           (int64_t)cl.cs * cluster_lists_slab_ints(cluster_layout(cl.cs, c[0], c[1], c[2], cl.half));
}

int64_t clb_mg_cluster_list_capacity(const clb_mg_hierarchy* h) {
    ClusterShape cl;
    if (!h || h->levels < 4 || h->levels > CLB_MG_MAX_LEVELS || !cluster_shape(h, h->levels - 3, cl)) return 0;
    return cluster_list_ints(h, cl);
}

int clb_mg_build_coarse(const clb_mg_hierarchy* h, void* stream) {
    if (check_hierarchy(h)) return 1;
    cudaStream_t s = CLB_STREAM(stream);
    if (h->fp16_level > 0 && check_call(cudaMemsetAsync(h->fp16_inexact, 0, sizeof(int32_t), s), "fp16 counter"))
        return 1;
    for (int l = 1; l < h->levels; ++l) {
        const int* f = h->shape[l - 1];
        const int* c = h->shape[l];
        const i64 C = (i64)c[0] * c[1] * c[2];
        const dim3 grid = blocks_for(C, MGT);
        const int fs = l == 1 ? 0 : (is_half(h, l - 1) ? 2 : 1);
        const bool ch = is_half(h, l);
        const uint8_t* fop0 = l == 1 ? h->op0 : nullptr;
        const void* fopc = l == 1 ? nullptr : h->op[l - 1];
        const uint8_t* fmask = l == 1 ? nullptr : h->mask[l - 1];
#define CLB_COARSE_OP(FS, CH)                                                                             \
    launch(grid, MGT, 0, s)(k_coarse_operator<FS, CH>, fop0, fopc, fmask, h->op[l], h->mask[l], h->fp16_inexact, \
                            f[0], f[1], f[2], c[0], c[1], c[2])
        if (fs == 0 && !ch) CLB_COARSE_OP(0, false);
        else if (fs == 1 && !ch) CLB_COARSE_OP(1, false);
        else if (fs == 0) CLB_COARSE_OP(0, true);
        else if (fs == 1) CLB_COARSE_OP(1, true);
        else CLB_COARSE_OP(2, true);
#undef CLB_COARSE_OP
        CLB_LAUNCH_CHECK("k_coarse_operator");
        // coarse p and b start at 0: cells without fluid keep it for the whole solve (mg_tiles.cuh)
        const size_t bytes = (size_t)C * (ch ? 2 : 4);
        if (check_call(cudaMemsetAsync(h->p[l], 0, bytes, s), "coarse p") ||
            check_call(cudaMemsetAsync(h->b[l], 0, bytes, s), "coarse b"))
            return 1;
    }
    if (h->tile_counts) {
        if (check_call(cudaMemsetAsync(h->tile_counts, 0, sizeof(int32_t) * CLB_MG_MAX_LEVELS, s), "tile counts"))
            return 1;
        for (int l = 0; l < h->levels; ++l) {
            if (!h->tiles[l]) continue;
            const int* n = h->shape[l];
            const i64 tiles = tile_capacity(n[0], n[1], n[2], l == 0);
            const unsigned grid = blocks_for(tiles * 32, 256);
            if (l == 0)
                launch(grid, 256, 0, s)(k_mg_tiles<true>, (const uint8_t*)h->op0, n[0], n[1], n[2], h->tiles[l],
                                        h->tile_counts + l);
            else
                launch(grid, 256, 0, s)(k_mg_tiles<false>, (const uint8_t*)h->mask[l], n[0], n[1], n[2], h->tiles[l],
                                        h->tile_counts + l);
            CLB_LAUNCH_CHECK("k_mg_tiles");
        }
    }
    if (h->fused_tiles) {
        CLB_REQUIRE(h->fused_tile_count != nullptr, "multigrid: fused_tiles without fused_tile_count");
        const int* n = h->shape[0];
        const i64 tiles = l0_tile_capacity(n[0], n[1], n[2]);
        if (check_call(cudaMemsetAsync(h->fused_tile_count, 0, sizeof(int32_t), s), "fused tile count")) return 1;
        if (tiles > 0) {
            launch((unsigned)tiles, L0T_THREADS, 0, s)(k_l0_fused_tiles, (const uint8_t*)h->op0, n[0], n[1], n[2],
                                                      h->fused_tiles, h->fused_tile_count);
            CLB_LAUNCH_CHECK("k_l0_fused_tiles");
        }
    }
    ClusterShape cl;
    if (h->cluster_lists && cluster_shape(h, h->levels - 3, cl)) {
        const int level = h->levels - 3;
        const int* c = h->shape[level];
        const int* a = h->shape[level + 1];
        const int* b = h->shape[level + 2];
#define CLB_CLUSTER_LISTS(H)                                                                                    \
    launch(cl.cs + 1, BOTTOM_THREADS, 0, s)(k_cluster_lists<H>, h->cluster_lists, (const void*)h->op[level],     \
                                            (const uint8_t*)h->mask[level], c[0], c[1], c[2],                    \
                                            (const void*)h->op[level + 1], (const uint8_t*)h->mask[level + 1],   \
                                            a[0], a[1], a[2], (const void*)h->op[level + 2],                     \
                                            (const uint8_t*)h->mask[level + 2], b[0], b[1], b[2], cl.cs)
        if (cl.half) CLB_CLUSTER_LISTS(true);
        else CLB_CLUSTER_LISTS(false);
#undef CLB_CLUSTER_LISTS
        CLB_LAUNCH_CHECK("k_cluster_lists");
    }
    return 0;
}

int64_t clb_mg_tile_capacity(int nx, int ny, int nz, int finest) {
    if (nx <= 0 || ny <= 0 || nz <= 0) return 0;
    return tile_capacity(nx, ny, nz, finest != 0);
}

int64_t clb_mg_fused_tile_capacity(int nx, int ny, int nz) { return l0_tile_capacity(nx, ny, nz); }

namespace {

struct LevelView {
    float* p;
    float* alt;
    int sweep;
    const float* b;
    const uint8_t* op0;
    const float4* opc;
    const uint8_t* mask;
    int nx, ny, nz;
    bool l0;
    bool half;            // FP16 storage (p, b as __half, opc as Half4)
    const float* scale;   // FP16 scales (mg_half.cuh)
    const int* tiles;     // fluid tiles (mg_tiles.cuh) or null
    const int* tile_count;
};

LevelView level_view(const clb_mg_hierarchy* h, int l, float* x, const float* rhs) {
    LevelView v;
    v.l0 = (l == 0);
    v.half = is_half(h, l);
    v.scale = h->fp16_scale;
    v.alt = h->alt[l];
    v.sweep = h->sweep[l];
    v.p = v.l0 ? x : h->p[l];
    v.b = v.l0 ? rhs : h->b[l];
    v.op0 = h->op0;
    v.opc = v.l0 ? nullptr : (const float4*)h->op[l];
    v.mask = v.l0 ? nullptr : h->mask[l];
    v.nx = h->shape[l][0];
    v.ny = h->shape[l][1];
    v.nz = h->shape[l][2];
    v.tiles = h->tile_counts ? h->tiles[l] : nullptr;
    v.tile_count = h->tile_counts ? h->tile_counts + l : nullptr;
    return v;
}

// Blocks of the tile-list kernels: enough to fill the GPU, never more than there are tiles.
static unsigned tile_grid(const LevelView& v) {
    const i64 cap = tile_capacity(v.nx, v.ny, v.nz, v.l0);
    const i64 most = (i64)(g_sm_count > 0 ? g_sm_count : 148) * 16;
    return (unsigned)(cap < most ? (cap > 0 ? cap : 1) : most);
}

extern "C++" {
// One launch of k_rbgs_iter: T iterations on big (8 x 8 x 32) or small (4 x 4 x 32) tiles.
template <bool L0, bool H, int TI, int TJ, int T>
static void launch_rbgs_iter(const LevelView& v, const float* in, float* out, float delta, cudaStream_t s) {
    const dim3 grid((v.nz + 31) / 32, (v.ny + TJ - 1) / TJ, (v.nx + TI - 1) / TI);
    launch(grid, SW_THREADS, SweepTile<L0, H, TI, TJ, 32, T>::smem(), s)(
        k_rbgs_iter<L0, H, TI, TJ, 32, T>, in, out, v.b, L0 ? v.op0 : nullptr, L0 ? nullptr : v.opc,
        L0 ? nullptr : v.mask, delta, v.scale, v.nx, v.ny, v.nz);
}

template <bool L0, bool H>
static void launch_rbgs_iter(const LevelView& v, bool big, int t, const float* in, float* out, float delta,
                             cudaStream_t s) {
    if (big && t == 2 && (L0 || H)) launch_rbgs_iter<L0, H, 8, 8, (L0 || H) ? 2 : 1>(v, in, out, delta, s);
    else if (t == 2) launch_rbgs_iter<L0, H, 4, 4, 2>(v, in, out, delta, s);  // FP32 coarse: no big pair tile
    else if (big) launch_rbgs_iter<L0, H, 8, 8, 1>(v, in, out, delta, s);
    else launch_rbgs_iter<L0, H, 4, 4, 1>(v, in, out, delta, s);
}
}  // extern "C++"

// clb_mg_hierarchy.sweep kinds: 1 two colour launches with 16-byte row vectors (FP32 levels), 2/3 one
// fused launch per iteration on 8x8x32 / 4x4x32 tiles, 4 two colour launches with one thread per
// cell, 5/6 one fused launch per two iterations on 8x8x32 / 4x4x32 tiles (on FP32 coarse levels kind 5
// runs as 6). Kinds 2, 3, 5 and 6 need the level's second buffer. All give identical values.
// sparse: every cell without fluid holds 0 (inside a W-cycle, mg_tiles.cuh), so an FP32 level with a
// tile list is swept on its fluid tiles only.
// Whether smooth(..., sparse = true) takes the fluid-tile colour sweeps on this level.
bool tile_sweeps(const LevelView& v) {
    const int vec = v.l0 && tile_k(v.nz, true) == 128 ? 4 : 1;
    return v.tiles && !v.half && (vec == 1 || (((uintptr_t)v.p) & 15) == 0);
}

// from_zero (level 0, tile sweeps, iterations >= 1): the first colour treats p as 0 (clb_mg_hierarchy
// zero_outside = 2).
int smooth(const LevelView& v, float delta, int iterations, cudaStream_t s, bool sparse = false,
           bool from_zero = false) {
    const i64 C = (i64)v.nx * v.ny * v.nz;
    const int kind = v.sweep == 0 || v.sweep == 7 ? (v.half ? 4 : 1) : v.sweep;  // 7: see level0_fused
    const int vec = v.l0 && tile_k(v.nz, true) == 128 ? 4 : 1;
    if (sparse && tile_sweeps(v)) {
        const unsigned grid = tile_grid(v);
        const dim3 block(32, 4);
        for (int it = 0; it < iterations; ++it)
            for (int parity = 0; parity < 2; ++parity) {
                if (from_zero && v.l0 && it == 0 && parity == 0) {
                    if (vec == 4)
                        launch(grid, block, 0, s)(k_rbgs_colour_tiles<true, 4, true>, v.tiles, v.tile_count, v.p,
                                                  v.b, v.op0, nullptr, nullptr, delta, parity, v.nx, v.ny, v.nz);
                    else
                        launch(grid, block, 0, s)(k_rbgs_colour_tiles<true, 1, true>, v.tiles, v.tile_count, v.p,
                                                  v.b, v.op0, nullptr, nullptr, delta, parity, v.nx, v.ny, v.nz);
                } else if (v.l0 && vec == 4)
                    launch(grid, block, 0, s)(k_rbgs_colour_tiles<true, 4>, v.tiles, v.tile_count, v.p, v.b, v.op0,
                                              nullptr, nullptr, delta, parity, v.nx, v.ny, v.nz);
                else if (v.l0)
                    launch(grid, block, 0, s)(k_rbgs_colour_tiles<true, 1>, v.tiles, v.tile_count, v.p, v.b, v.op0,
                                              nullptr, nullptr, delta, parity, v.nx, v.ny, v.nz);
                else
                    launch(grid, block, 0, s)(k_rbgs_colour_tiles<false, 1>, v.tiles, v.tile_count, v.p, v.b,
                                              nullptr, v.opc, v.mask, delta, parity, v.nx, v.ny, v.nz);
                CLB_LAUNCH_CHECK("k_rbgs_colour_tiles");
            }
        return 0;
    }
    if ((kind == 2 || kind == 3 || kind == 5 || kind == 6) && v.alt != nullptr && iterations > 0) {
        // fused iterations, alternating between the level's buffer and its second buffer
        const bool big = kind == 2 || kind == 5;
        const int per = kind >= 5 ? 2 : 1;
        float* cur = v.p;
        float* other = v.alt;
        for (int left = iterations; left > 0;) {
            const int t = left >= per ? per : 1;
            if (v.l0) launch_rbgs_iter<true, false>(v, big, t, cur, other, delta, s);
            else if (v.half) launch_rbgs_iter<false, true>(v, big, t, cur, other, delta, s);
            else launch_rbgs_iter<false, false>(v, big, t, cur, other, delta, s);
            CLB_LAUNCH_CHECK("k_rbgs_iter");
            float* tmp = cur;
            cur = other;
            other = tmp;
            left -= t;
        }
        const size_t bytes = (size_t)C * (v.half ? 2 : 4);
        if (cur != v.p && check_call(cudaMemcpyAsync(v.p, cur, bytes, cudaMemcpyDeviceToDevice, s), "smooth copy-back"))
            return 1;
        return 0;
    }
    if (v.half) {  // FP16 levels otherwise: one thread per cell
        for (int it = 0; it < iterations; ++it)
            for (int parity = 0; parity < 2; ++parity) {
                launch(blocks_for(C, MGT), MGT, 0, s)(k_rbgs_h, reinterpret_cast<__half*>(v.p),
                                                      reinterpret_cast<const __half*>(v.b),
                                                      reinterpret_cast<const Half4*>(v.opc), v.mask, v.scale,
                                                      parity, v.nx, v.ny, v.nz);
                CLB_LAUNCH_CHECK("k_rbgs_h");
            }
        return 0;
    }
    if (kind == 1) {
        const bool vec4 = (v.nz % 4) == 0 && (((uintptr_t)v.p) & 15) == 0;
        const int vec = vec4 ? 4 : 1;
        const dim3 block(32, 4);
        const dim3 grid((v.nz + 32 * vec - 1) / (32 * vec), (v.ny + 3) / 4, v.nx);
        for (int it = 0; it < iterations; ++it)
            for (int parity = 0; parity < 2; ++parity) {
                if (v.l0 && vec4)
                    launch(grid, block, 0, s)(k_rbgs_colour<true, 4>, v.p, v.b, v.op0, nullptr, nullptr, delta, parity,
                                              v.nx, v.ny, v.nz);
                else if (v.l0)
                    launch(grid, block, 0, s)(k_rbgs_colour<true, 1>, v.p, v.b, v.op0, nullptr, nullptr, delta, parity,
                                              v.nx, v.ny, v.nz);
                else if (vec4)
                    launch(grid, block, 0, s)(k_rbgs_colour<false, 4>, v.p, v.b, nullptr, v.opc, v.mask, delta, parity,
                                              v.nx, v.ny, v.nz);
                else
                    launch(grid, block, 0, s)(k_rbgs_colour<false, 1>, v.p, v.b, nullptr, v.opc, v.mask, delta, parity,
                                              v.nx, v.ny, v.nz);
                CLB_LAUNCH_CHECK("k_rbgs_colour");
            }
        return 0;
    }
    for (int it = 0; it < iterations; ++it)
        for (int parity = 0; parity < 2; ++parity) {
            if (v.l0)
                launch(blocks_for(C, MGT), MGT, 0, s)(k_rbgs<true>, v.p, v.b, v.op0, nullptr, nullptr, delta, parity, v.nx,
                                                      v.ny, v.nz);
            else
                launch(blocks_for(C, MGT), MGT, 0, s)(k_rbgs<false>, v.p, v.b, nullptr, v.opc, v.mask, delta, parity, v.nx,
                                                      v.ny, v.nz);
            CLB_LAUNCH_CHECK("k_rbgs");
        }
    return 0;
}

int coarse_solve(const LevelView& v, float delta, int iterations, cudaStream_t s) {
    const int C = v.nx * v.ny * v.nz;
    if (v.half) {  // checked to fit shared memory by check_hierarchy
        launch(1, COARSE_THREADS, coarse_smem_bytes(C), s)(k_coarse_solve<true, false, true>,
            v.p, v.b, nullptr, v.opc, v.mask, delta, iterations, v.nx, v.ny, v.nz, v.scale);
        CLB_LAUNCH_CHECK("k_coarse_solve");
        return 0;
    }
    if (C <= COARSE_SMEM_CELLS) {
        const size_t bytes = coarse_smem_bytes(C);
        if (v.l0)
            launch(1, COARSE_THREADS, bytes, s)(k_coarse_solve<true, true>, v.p, v.b, v.op0, nullptr, nullptr, delta,
                                                iterations, v.nx, v.ny, v.nz, nullptr);
        else
            launch(1, COARSE_THREADS, bytes, s)(k_coarse_solve<true, false>, v.p, v.b, nullptr, v.opc, v.mask, delta,
                                                iterations, v.nx, v.ny, v.nz, nullptr);
    } else {
        if (v.l0)
            launch(1, COARSE_THREADS, 0, s)(k_coarse_solve<false, true>, v.p, v.b, v.op0, nullptr, nullptr, delta,
                                            iterations, v.nx, v.ny, v.nz, nullptr);
        else
            launch(1, COARSE_THREADS, 0, s)(k_coarse_solve<false, false>, v.p, v.b, nullptr, v.opc, v.mask, delta,
                                            iterations, v.nx, v.ny, v.nz, nullptr);
    }
    CLB_LAUNCH_CHECK("k_coarse_solve");
    return 0;
}

extern "C++" {
template <int NS, int KA, int KB, bool H>
static int launch_cluster_visit(const clb_mg_hierarchy* h, int level, int csize, size_t bytes, int pre, int post,
                                int coarse_iters, int visits, cudaStream_t s) {
    auto kernel = k_cluster_visit<NS, KA, KB, H>;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(csize);
    cfg.blockDim = dim3(BOTTOM_THREADS);
    cfg.dynamicSmemBytes = bytes;
    cfg.stream = s;
    cudaLaunchAttribute attr[2];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = csize;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    attr[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[1].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    // a cluster of this size and shared memory must be schedulable (checked once per shape)
    static std::mutex mu;
    static int cached_csize = -1, cached_ok = 0;
    static size_t cached_bytes = 0;
    {
        std::lock_guard<std::mutex> lock(mu);
        if (cached_csize != csize || cached_bytes != bytes) {
            int clusters = 0;
            cached_ok = cudaOccupancyMaxActiveClusters(&clusters, kernel, &cfg) == cudaSuccess && clusters >= 1;
            (void)cudaGetLastError();
            cached_csize = csize;
            cached_bytes = bytes;
        }
        if (!cached_ok) return 0;
    }
    cfg.numAttrs = g_use_pdl ? 2 : 1;
    const int* c = h->shape[level];
    const int* a = h->shape[level + 1];
    const int* b = h->shape[level + 2];
    (void)cudaLaunchKernelEx(&cfg, kernel, h->p[level], (const float*)h->b[level], (const void*)h->op[level],
                             (const uint8_t*)h->mask[level], c[0], c[1], c[2], h->p[level + 1],
                             (const float4*)h->op[level + 1], (const uint8_t*)h->mask[level + 1], a[0], a[1], a[2],
                             (const float4*)h->op[level + 2], (const uint8_t*)h->mask[level + 2], b[0], b[1], b[2],
                             h->delta, pre, post, coarse_iters, (const float*)h->fp16_scale, visits,
                             visits_of(level + 1), visits_of(level + 2), (const int*)h->cluster_lists, pscale(h));
    return check_launch("k_cluster_visit") ? -1 : 1;
}
}  // extern "C++"

// One cluster launch for `visits` consecutive visits of the third-coarsest level, each with its two
// bottom visits (mg_cluster.cuh), when the three levels share their storage type and fit; returns 1
// if it launched, 0 if the caller must go on level by level, -1 on error.
int cluster_visit(const clb_mg_hierarchy* h, int level, int pre, int post, int coarse_iters, cudaStream_t s,
                  int visits = 1) {
    ClusterShape cl;
    if (!g_use_cluster || !g_use_bottom || !cluster_shape(h, level, cl)) return 0;
    const int cs = cl.cs, ka = cl.ka, ns = cl.ns;
    const size_t bytes = cl.bytes;
    const bool half = cl.half;
#define CLB_CLUSTER(NS, KA, H) \
    launch_cluster_visit<NS, KA, 1, H>(h, level, cs + 1, bytes, pre, post, coarse_iters, visits, s)
#define CLB_CLUSTER_KINDS(H)                                  \
    if (ka <= 2 && ns <= 4) return CLB_CLUSTER(4, 2, H);      \
    if (ns <= 2) return CLB_CLUSTER(2, 4, H);                 \
    if (ns <= 4) return CLB_CLUSTER(4, 4, H);                 \
    if (ns <= 8) return CLB_CLUSTER(8, 4, H);                 \
    return 0;
    if (half) {
        CLB_CLUSTER_KINDS(true)
    } else {
        CLB_CLUSTER_KINDS(false)
    }
#undef CLB_CLUSTER_KINDS
#undef CLB_CLUSTER
}

// One launch for a whole visit of the second-coarsest level when both bottom levels fit in shared
// memory (mg_bottom.cuh); returns 1 if it launched, 0 if the caller must recurse, -1 on error.
int bottom_visit(const clb_mg_hierarchy* h, int level, int pre, int post, int coarse_iters, cudaStream_t s) {
    if (!g_use_bottom || level < 1 || level != h->levels - 2) return 0;
    const int* a = h->shape[level];
    const int* b = h->shape[level + 1];
    const int ca = a[0] * a[1] * a[2], cb = b[0] * b[1] * b[2];
    const int sa = colour_slots(a[0], a[1], a[2]), sb = colour_slots(b[0], b[1], b[2]);
    const size_t bytes = bottom_smem_bytes(ca, cb);
    if (bytes > kBottomSmemLimit || sb > BOTTOM_MAX_B * BOTTOM_BTHREADS || sa > BOTTOM_MAX_A * BOTTOM_THREADS)
        return 0;
    const int ka = (sa + BOTTOM_THREADS - 1) / BOTTOM_THREADS;
    const int kb = (sb + BOTTOM_BTHREADS - 1) / BOTTOM_BTHREADS;
#define CLB_BOTTOM(KA, KB, H)                                                                                   \
    launch(1, BOTTOM_THREADS, bytes, s)(k_bottom_visit<KA, KB, H>,                                                    \
        h->p[level], h->b[level], (const float4*)h->op[level], h->mask[level], a[0], a[1], a[2], h->p[level + 1],      \
        h->b[level + 1], (const float4*)h->op[level + 1], h->mask[level + 1], b[0], b[1], b[2], h->delta, pre,         \
                                        post, coarse_iters, h->fp16_scale, visits_of(level + 1), pscale(h))
#define CLB_BOTTOM_KINDS(H)                                 \
    if (ka <= 1 && kb <= 1) CLB_BOTTOM(1, 1, H);            \
    else if (ka <= 2 && kb <= 1) CLB_BOTTOM(2, 1, H);       \
    else if (ka <= 4 && kb <= 1) CLB_BOTTOM(4, 1, H);       \
    else if (ka <= 4 && kb <= 2) CLB_BOTTOM(4, 2, H);       \
    else CLB_BOTTOM(8, 4, H);
    if (is_half(h, level)) {  // the suffix of FP16 levels then holds both bottom levels
        CLB_BOTTOM_KINDS(true)
    } else {
        CLB_BOTTOM_KINDS(false)
    }
#undef CLB_BOTTOM_KINDS
#undef CLB_BOTTOM
    if (check_launch("k_bottom_visit")) return -1;
    return 1;
}

// multigrid.py:53-187 w_cycle
// zero_outside = 2 on level 0: x counts as 0 inside the fluid tiles (and is 0 outside them). When the
// first thing done to level 0 is a fluid-tile colour sweep, that sweep ignores x (from_zero);
// otherwise x is zeroed here.
int level0_zero(const clb_mg_hierarchy* h, const LevelView& v, int first_sweeps, bool sweep_first, bool sparse,
                cudaStream_t s, bool& from_zero) {
    from_zero = false;
    if (h->zero_outside != 2) return 0;
    from_zero = sweep_first && sparse && first_sweeps >= 1 && tile_sweeps(v);
    if (from_zero) return 0;
    return check_call(cudaMemsetAsync(v.p, 0, (size_t)v.nx * v.ny * v.nz * sizeof(float), s), "zero level-0 x");
}

int w_cycle(const clb_mg_hierarchy* h, int level, float* x, const float* rhs, int pre, int post, int coarse_iters,
            cudaStream_t s);

// pre / post: the W-cycle's smoothing counts (level 0's). Levels >= 1 use the hierarchy's coarse counts
// when it sets them (clb_mg_hierarchy.coarse_smoothing), so each frame maps the counts of its own level
// and of the level below, and passes the W-cycle's on.
static inline int coarse_pre(const clb_mg_hierarchy* h, int pre) { return h->coarse_smoothing ? h->coarse_pre_smooth : pre; }
static inline int coarse_post(const clb_mg_hierarchy* h, int post) {
    return h->coarse_smoothing ? h->coarse_post_smooth : post;
}

// Whether level 0 of this W-cycle runs as the fused tile launches of mg_level0.cuh: sweep kind 7 on
// level 0, its 3-D fluid tiles and second buffer, a correction from zero (zero_outside = 2), at least
// one pre- and one post-smoothing iteration, and an FP32 level 1 below.
bool level0_fused(const clb_mg_hierarchy* h, int pre, int post) {
    return h->sweep[0] == 7 && h->fused_tiles && h->fused_tile_count && h->alt[0] && h->zero_outside == 2 &&
           pre >= 1 && post >= 1 && h->levels >= 2 && !is_half(h, 1);
}

extern "C++" {
template <int MODE>
void launch_l0_iter(const clb_mg_hierarchy* h, const float* in, float* out, const float* rhs, cudaStream_t s) {
    const int* n = h->shape[0];
    const int* c = h->shape[1];
    const i64 cap = l0_tile_capacity(n[0], n[1], n[2]);
    static const int per_sm = [] {  // once per mode
        int b = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_l0_iter_tiles<MODE>, L0T_THREADS,
                                                          L0Region<(MODE & L0F_RESTRICT) ? 3 : 2>::smem()) !=
            cudaSuccess) {
            (void)cudaGetLastError();
            b = 0;
        }
        return b > 0 ? b : 1;
    }();
    const i64 most = (i64)per_sm * (g_sm_count > 0 ? g_sm_count : 148);
    const unsigned grid = (unsigned)(cap < most ? (cap > 0 ? cap : 1) : most);
    launch(grid, L0T_THREADS, L0Region<(MODE & L0F_RESTRICT) ? 3 : 2>::smem(), s)(
        k_l0_iter_tiles<MODE>, h->fused_tiles, h->fused_tile_count, in, out, rhs, h->op0, h->delta, n[0], n[1], n[2],
        h->p[1], h->b[1], h->p[1], c[0], c[1], c[2], pscale(h));
}
}  // extern "C++"

// Level 0 of a W-cycle from a zero correction in pre + post fused launches: the first pre-smoothing
// iteration reads no x, the last one restricts, the first post-smoothing one prolongs. The launches
// alternate between x and the level's second buffer, the first writing the one that makes the last
// write land in x.
int w_cycle_level0_fused(const clb_mg_hierarchy* h, float* x, const float* rhs, int pre, int post, int coarse_iters,
                         cudaStream_t s) {
    float* buf[2] = {x, h->alt[0]};
    int dst = (pre + post) % 2 == 1 ? 0 : 1;
    const float* src = nullptr;
    for (int it = 0; it < pre; ++it) {
        const bool first = it == 0, last = it == pre - 1;
        if (first && last) launch_l0_iter<L0F_ZERO | L0F_RESTRICT>(h, src, buf[dst], rhs, s);
        else if (first) launch_l0_iter<L0F_ZERO>(h, src, buf[dst], rhs, s);
        else if (last) launch_l0_iter<L0F_RESTRICT>(h, src, buf[dst], rhs, s);
        else launch_l0_iter<0>(h, src, buf[dst], rhs, s);
        CLB_LAUNCH_CHECK("k_l0_iter_tiles");
        src = buf[dst];
        dst ^= 1;
    }
    const int visits = visits_of(1);
    const int both = cluster_visit(h, 1, coarse_pre(h, pre), coarse_post(h, post), coarse_iters, s, visits);
    if (both < 0) return 1;
    if (both == 0)
        for (int v2 = 0; v2 < visits; ++v2)
            if (w_cycle(h, 1, x, rhs, pre, post, coarse_iters, s)) return 1;
    for (int it = 0; it < post; ++it) {
        if (it == 0) launch_l0_iter<L0F_PROLONG>(h, src, buf[dst], rhs, s);
        else launch_l0_iter<0>(h, src, buf[dst], rhs, s);
        CLB_LAUNCH_CHECK("k_l0_iter_tiles");
        src = buf[dst];
        dst ^= 1;
    }
    CLB_REQUIRE(src == x, "mg_w_cycle: fused level-0 iterations ended outside x");
    return 0;
}

int w_cycle(const clb_mg_hierarchy* h, int level, float* x, const float* rhs, int pre0, int post0, int coarse_iters,
            cudaStream_t s) {
    if (level == 0 && level0_fused(h, pre0, post0))
        return w_cycle_level0_fused(h, x, rhs, pre0, post0, coarse_iters, s);
    const int pre = level > 0 ? coarse_pre(h, pre0) : pre0, post = level > 0 ? coarse_post(h, post0) : post0;
    const int cpre = coarse_pre(h, pre0), cpost = coarse_post(h, post0);  // the level below's
    const LevelView v = level_view(h, level, x, rhs);
    // coarse levels hold 0 outside the fluid (zeroed by clb_mg_build_coarse and the restriction);
    // level 0 does when the caller says so
    const bool sparse = level > 0 || h->zero_outside != 0;
    bool from_zero = false;
    if (level == 0 && level0_zero(h, v, pre, level != h->levels - 1, sparse, s, from_zero)) return 1;
    if (level == h->levels - 1) return coarse_solve(v, h->delta, pre + coarse_iters, s);
    const int cluster = cluster_visit(h, level, pre, post, coarse_iters, s);
    if (cluster != 0) return cluster < 0 ? 1 : 0;
    const int bottom = bottom_visit(h, level, pre, post, coarse_iters, s);
    if (bottom != 0) return bottom < 0 ? 1 : 0;
    if (smooth(v, h->delta, pre, s, sparse, from_zero)) return 1;
    const LevelView c = level_view(h, level + 1, x, rhs);
    const i64 Cc = (i64)c.nx * c.ny * c.nz;
    if (!c.half && !v.half && c.tiles) {  // restriction of the coarse fluid tiles (inactive cells hold 0)
        if (v.l0)
            launch(tile_grid(c), dim3(32, 4), 0, s)(k_restrict_tiles<true>, c.tiles, c.tile_count, v.p, v.b, v.op0,
                                                    nullptr, nullptr, c.p, const_cast<float*>(c.b), h->delta, v.nx,
                                                    v.ny, v.nz, c.nx, c.ny, c.nz);
        else
            launch(tile_grid(c), dim3(32, 4), 0, s)(k_restrict_tiles<false>, c.tiles, c.tile_count, v.p, v.b,
                                                    nullptr, v.opc, v.mask, c.p, const_cast<float*>(c.b), h->delta,
                                                    v.nx, v.ny, v.nz, c.nx, c.ny, c.nz);
    } else if (c.half) {
        const dim3 grid = blocks_for(Cc, MGT);
#define CLB_RESTRICT_H(FS)                                                                                        \
    launch(grid, MGT, 0, s)(k_restrict_h<FS>, v.p, v.b, v.op0, v.opc, v.mask, reinterpret_cast<__half*>(c.p),          \
                            reinterpret_cast<__half*>(const_cast<float*>(c.b)), h->delta, h->fp16_scale,               \
                            v.nx, v.ny, v.nz, c.nx, c.ny, c.nz)
        if (v.half) CLB_RESTRICT_H(2);
        else if (v.l0) CLB_RESTRICT_H(0);
        else CLB_RESTRICT_H(1);
#undef CLB_RESTRICT_H
    } else if (v.l0)
        launch(blocks_for(Cc, MGT), MGT, 0, s)(k_restrict<true>, v.p, v.b, v.op0, nullptr, nullptr, c.p,
                                               const_cast<float*>(c.b), h->delta, v.nx, v.ny, v.nz,
                                               c.nx, c.ny, c.nz);
    else
        launch(blocks_for(Cc, MGT), MGT, 0, s)(k_restrict<false>, v.p, v.b, nullptr, v.opc, v.mask, c.p,
                                               const_cast<float*>(c.b), h->delta, v.nx, v.ny, v.nz,
                                               c.nx, c.ny, c.nz);
    CLB_LAUNCH_CHECK("k_restrict");
    // the visits of the level below (two, or one from the single-visit level on): one cluster launch
    // for them when it takes the cluster path
    const int visits = visits_of(level + 1);
    const int both = cluster_visit(h, level + 1, cpre, cpost, coarse_iters, s, visits);
    if (both < 0) return 1;
    if (both == 0)
        for (int v2 = 0; v2 < visits; ++v2)
            if (w_cycle(h, level + 1, x, rhs, pre0, post0, coarse_iters, s)) return 1;
    const i64 Cf = (i64)v.nx * v.ny * v.nz;
    const int fvec = v.l0 && tile_k(v.nz, true) == 128 ? 4 : 1;
    const float w = pscale(h);
    if (!c.half && !v.half && v.tiles) {  // prolongation into the fine fluid tiles
        if (v.l0 && fvec == 4 && ((((uintptr_t)v.p) & 15) | (((uintptr_t)v.op0) & 3)) == 0)
            launch(tile_grid(v), dim3(32, 4), 0, s)(k_prolong_tiles<true, 4, true>, v.tiles, v.tile_count, c.p, v.p,
                                                    v.op0, nullptr, c.nx, c.ny, c.nz, v.nx, v.ny, v.nz, w);
        else if (v.l0 && fvec == 4)
            launch(tile_grid(v), dim3(32, 4), 0, s)(k_prolong_tiles<true, 4>, v.tiles, v.tile_count, c.p, v.p, v.op0,
                                                    nullptr, c.nx, c.ny, c.nz, v.nx, v.ny, v.nz, w);
        else if (v.l0)
            launch(tile_grid(v), dim3(32, 4), 0, s)(k_prolong_tiles<true, 1>, v.tiles, v.tile_count, c.p, v.p, v.op0,
                                                    nullptr, c.nx, c.ny, c.nz, v.nx, v.ny, v.nz, w);
        else
            launch(tile_grid(v), dim3(32, 4), 0, s)(k_prolong_tiles<false, 1>, v.tiles, v.tile_count, c.p, v.p,
                                                    nullptr, v.mask, c.nx, c.ny, c.nz, v.nx, v.ny, v.nz, w);
    } else if (c.half) {
        const dim3 grid = blocks_for(Cf, MGT);
        const __half* ce = reinterpret_cast<const __half*>(c.p);
        if (v.half)
            launch(grid, MGT, 0, s)(k_prolong_h<2>, ce, v.p, nullptr, v.mask, h->fp16_scale, c.nx, c.ny, c.nz, v.nx, v.ny,
                                    v.nz, w);
        else if (v.l0)
            launch(grid, MGT, 0, s)(k_prolong_h<0>, ce, v.p, v.op0, nullptr, h->fp16_scale, c.nx, c.ny, c.nz, v.nx, v.ny,
                                    v.nz, w);
        else
            launch(grid, MGT, 0, s)(k_prolong_h<1>, ce, v.p, nullptr, v.mask, h->fp16_scale, c.nx, c.ny, c.nz, v.nx, v.ny,
                                    v.nz, w);
    } else if (v.l0)
        launch(blocks_for(Cf, MGT), MGT, 0, s)(k_prolong<true>, c.p, v.p, v.op0, nullptr, c.nx, c.ny, c.nz, v.nx, v.ny,
                                               v.nz, w);
    else
        launch(blocks_for(Cf, MGT), MGT, 0, s)(k_prolong<false>, c.p, v.p, nullptr, v.mask, c.nx, c.ny, c.nz, v.nx, v.ny,
                                               v.nz, w);
    CLB_LAUNCH_CHECK("k_prolong");
    return smooth(v, h->delta, post, s, sparse);
}

}  // namespace

int clb_mg_w_cycle(const clb_mg_hierarchy* h, float* x, const float* rhs, int pre_smooth, int post_smooth,
                   int coarse_iterations, void* stream) {
    if (check_hierarchy(h)) return 1;
    CLB_REQUIRE(x && rhs, "mg_w_cycle: null level-0 array");
    CLB_REQUIRE(pre_smooth >= 0 && post_smooth >= 0 && coarse_iterations >= 0, "mg_w_cycle: negative sweep count");
    CLB_REQUIRE(!h->coarse_smoothing || (h->coarse_pre_smooth >= 0 && h->coarse_post_smooth >= 0),
                "mg_w_cycle: negative coarse-level sweep count");
    cudaStream_t s = CLB_STREAM(stream);
    if (h->fp16_level > 0) {
        CLB_REQUIRE(h->rhs_norms != nullptr, "mg_w_cycle: FP16 levels need rhs_norms");
        launch(1, 32, 0, s)(k_fp16_scale, h->rhs_norms, h->delta, h->fp16_scale);
        CLB_LAUNCH_CHECK("k_fp16_scale");
    }
    return w_cycle(h, 0, x, rhs, pre_smooth, post_smooth, coarse_iterations, s);
}

int clb_mg_level0_iteration(const clb_mg_hierarchy* h, const float* x_in, float* x_out, const float* rhs, int mode,
                            void* stream) {
    if (check_hierarchy(h)) return 1;
    CLB_REQUIRE(h->fused_tiles && h->fused_tile_count, "mg_level0_iteration: no fused tiles");
    CLB_REQUIRE(h->levels >= 2 && !is_half(h, 1), "mg_level0_iteration: level 1 must exist and be FP32");
    CLB_REQUIRE(x_out && rhs && ((mode & L0F_ZERO) || x_in), "mg_level0_iteration: null array");
    CLB_REQUIRE((mode & L0F_ZERO) || x_in != x_out, "mg_level0_iteration: x_in and x_out must differ");
    cudaStream_t s = CLB_STREAM(stream);
    switch (mode) {
        case 0: launch_l0_iter<0>(h, x_in, x_out, rhs, s); break;
        case L0F_ZERO: launch_l0_iter<L0F_ZERO>(h, nullptr, x_out, rhs, s); break;
        case L0F_RESTRICT: launch_l0_iter<L0F_RESTRICT>(h, x_in, x_out, rhs, s); break;
        case L0F_ZERO | L0F_RESTRICT: launch_l0_iter<L0F_ZERO | L0F_RESTRICT>(h, nullptr, x_out, rhs, s); break;
        case L0F_PROLONG: launch_l0_iter<L0F_PROLONG>(h, x_in, x_out, rhs, s); break;
        default: return set_error("mg_level0_iteration: mode %d is not 0, 1, 2, 3 or 4", mode);
    }
    CLB_LAUNCH_CHECK("k_l0_iter_tiles");
    return 0;
}

int clb_mg_smooth(const clb_mg_hierarchy* h, int level, float* x, const float* rhs, int iterations, void* stream) {
    if (check_hierarchy(h)) return 1;
    CLB_REQUIRE(level >= 0 && level < h->levels, "mg_smooth: level %d outside 0..%d", level, h->levels - 1);
    CLB_REQUIRE(iterations >= 0, "mg_smooth: negative iterations");
    CLB_REQUIRE(level > 0 || (x && rhs), "mg_smooth: null level-0 array");
    const LevelView v = level_view(h, level, x, rhs);
    const bool sparse = h->zero_outside != 0 && h->tile_counts != nullptr;
    bool from_zero = false;
    if (level == 0 && level0_zero(h, v, iterations, true, sparse, CLB_STREAM(stream), from_zero)) return 1;
    return smooth(v, h->delta, iterations, CLB_STREAM(stream), sparse, from_zero);
}

int clb_mg_set_option(int option, int value) {
    CLB_REQUIRE(option >= 0 && option <= 4, "mg_set_option: unknown option %d", option);
    CLB_REQUIRE(option != 4 || value >= 0, "mg_set_option: negative single-visit level");
    if (option == 0) g_use_bottom = value != 0;
    else if (option == 1) g_use_pdl = value != 0;
    else if (option == 2) g_use_cluster = value != 0;
    else if (option == 3) g_skip_air = value != 0;
    else g_single_from = value;
    return 0;
}

int clb_mg_residual_partials(int64_t cells) {
    const i64 need = (cells + RN_THREADS - 1) / RN_THREADS;
    const i64 cap = 148 * 8;
    return (int)(need < cap ? (need > 0 ? need : 1) : cap);
}

extern "C++" {
namespace {
// Grid of a row kernel (k_residual_rows, k_fcg_dots): at most the blocks that are resident on the
// device at once, so that no partial second wave waits for the first (the rows are spread over the
// blocks' warps in any case). Never more than clb_mg_residual_partials, the callers' partial count.
template <auto KERNEL>
int row_grid(i64 cells) {
    static const int per_sm = [] {  // once per kernel
        int n = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, KERNEL, RN_THREADS, 0) != cudaSuccess) {
            (void)cudaGetLastError();
            n = 0;
        }
        return n;
    }();
    const int want = clb_mg_residual_partials(cells);
    const int resident = per_sm * (g_sm_count > 0 ? g_sm_count : 148);
    return resident >= 1 && resident < want ? resident : want;
}
}  // namespace
}  // extern "C++"

int clb_mg_residual_norms(const void* p, int p_is_double, const float* b, const uint8_t* op0, float delta, int nx,
                          int ny, int nz, float* r_out, void* partials, double* out, void* stream) {
    CLB_GRID_ARGS_OK(nx, ny, nz);
    CLB_REQUIRE(p && b && op0 && partials && out, "mg_residual_norms: null pointer");
    const i64 C = (i64)nx * ny * nz;
    const int blocks = clb_mg_residual_partials(C);
    const double inv_delta2 = 1.0 / ((double)delta * (double)delta);
    cudaStream_t s = CLB_STREAM(stream);
    if (p_is_double)
        launch(blocks, RN_THREADS, 0, s)(k_residual_rows<double, RES_NORM>, (const double*)p, nullptr, nullptr, b, op0,
                                         inv_delta2, nx, ny, nz, r_out,
                                         (double2*)partials, nullptr, nullptr, nullptr);
    else
        launch(blocks, RN_THREADS, 0, s)(k_residual_rows<float, RES_NORM>, (const float*)p, nullptr, nullptr, b, op0,
                                         inv_delta2, nx, ny, nz, r_out, (double2*)partials,
                                         nullptr, nullptr, nullptr);
    CLB_LAUNCH_CHECK("k_residual_rows");
    launch(1, 256, 0, s)(k_reduce_partials, (const double2*)partials, blocks, (double2*)out);
    CLB_LAUNCH_CHECK("k_reduce_partials");
    return 0;
}

int clb_mg_ir_step(const double* p64_in, const float* e, double* p64_out, const float* b, const uint8_t* op0,
                   float delta, int nx, int ny, int nz, float* r_out, void* partials, double* out, void* stream) {
    CLB_GRID_ARGS_OK(nx, ny, nz);
    CLB_REQUIRE(p64_in && e && p64_out && b && op0 && r_out && partials && out, "mg_ir_step: null pointer");
    CLB_REQUIRE(p64_in != p64_out, "mg_ir_step: p64_out must not alias p64_in");
    const i64 C = (i64)nx * ny * nz;
    const double inv_delta2 = 1.0 / ((double)delta * (double)delta);
    cudaStream_t s = CLB_STREAM(stream);
    int blocks;
    if (g_skip_air) {
        blocks = row_grid<k_residual_rows<double, RES_IR, true>>(C);
        launch(blocks, RN_THREADS, 0, s)(k_residual_rows<double, RES_IR, true>, p64_in, e, p64_out, b, op0, inv_delta2,
                                         nx, ny, nz, r_out, (double2*)partials, nullptr, nullptr, nullptr);
    } else {
        blocks = clb_mg_residual_partials(C);
        launch(blocks, RN_THREADS, 0, s)(k_residual_rows<double, RES_IR, false>, p64_in, e, p64_out, b, op0,
                                         inv_delta2, nx, ny, nz, r_out, (double2*)partials, nullptr, nullptr, nullptr);
    }
    CLB_LAUNCH_CHECK("k_residual_rows");
    launch(1, 256, 0, s)(k_reduce_partials, (const double2*)partials, blocks, (double2*)out);
    CLB_LAUNCH_CHECK("k_reduce_partials");
    return 0;
}

int clb_mg_fcg_dots(const float* z, const float* d, const float* r, const uint8_t* op0, float delta, int nx, int ny,
                    int nz, void* partials4, double* state, void* stream) {
    CLB_GRID_ARGS_OK(nx, ny, nz);
    CLB_REQUIRE(z && d && r && op0 && partials4 && state, "mg_fcg_dots: null pointer");
    const i64 C = (i64)nx * ny * nz;
    const int blocks = row_grid<k_fcg_dots>(C);
    const double inv_delta2 = 1.0 / ((double)delta * (double)delta);
    cudaStream_t s = CLB_STREAM(stream);
    launch(blocks, RN_THREADS, 0, s)(k_fcg_dots, z, d, r, op0, inv_delta2, nx, ny, nz, (Sum4*)partials4);
    CLB_LAUNCH_CHECK("k_fcg_dots");
    launch(1, 256, 0, s)(k_fcg_scalars, (const Sum4*)partials4, blocks, state);
    CLB_LAUNCH_CHECK("k_fcg_scalars");
    return 0;
}

int clb_mg_fcg_step(const double* p64_in, const float* z, const float* d_in, double* p64_out, float* d_out,
                    const double* state, const float* b, const uint8_t* op0, float delta, int nx, int ny, int nz,
                    float* r_out, void* partials, double* out, void* stream) {
    CLB_GRID_ARGS_OK(nx, ny, nz);
    CLB_REQUIRE(p64_in && z && d_in && p64_out && d_out && state && b && op0 && r_out && partials && out,
                "mg_fcg_step: null pointer");
    CLB_REQUIRE(p64_in != p64_out && d_in != d_out, "mg_fcg_step: outputs must not alias inputs");
    const i64 C = (i64)nx * ny * nz;
    const double inv_delta2 = 1.0 / ((double)delta * (double)delta);
    cudaStream_t s = CLB_STREAM(stream);
    int blocks;
    if (g_skip_air) {
        blocks = row_grid<k_residual_rows<double, RES_FCG, true>>(C);
        launch(blocks, RN_THREADS, 0, s)(k_residual_rows<double, RES_FCG, true>, p64_in, z, p64_out, b, op0,
                                         inv_delta2, nx, ny, nz, r_out, (double2*)partials, d_in, d_out, state);
    } else {
        blocks = clb_mg_residual_partials(C);
        launch(blocks, RN_THREADS, 0, s)(k_residual_rows<double, RES_FCG, false>, p64_in, z, p64_out, b, op0,
                                         inv_delta2, nx, ny, nz, r_out, (double2*)partials, d_in, d_out, state);
    }
    CLB_LAUNCH_CHECK("k_residual_rows");
    launch(1, 256, 0, s)(k_reduce_partials, (const double2*)partials, blocks, (double2*)out);
    CLB_LAUNCH_CHECK("k_reduce_partials");
    return 0;
}

int clb_mg_ir_init(const float* p32, const uint8_t* op0, double* p64, int nx, int ny, int nz, void* stream) {
    CLB_GRID_ARGS_OK(nx, ny, nz);
    CLB_REQUIRE(p32 && op0 && p64, "mg_ir_init: null pointer");
    const i64 C = (i64)nx * ny * nz;
    if (nz % 4 == 0 && (((uintptr_t)p32 | (uintptr_t)p64) & 15) == 0 && (((uintptr_t)op0) & 3) == 0)
        launch(blocks_for(C / 4, MGT), MGT, 0, CLB_STREAM(stream))(k_ir_init4, p32, op0, p64, nx, ny, nz);
    else
        launch(blocks_for(C, MGT), MGT, 0, CLB_STREAM(stream))(k_ir_init, p32, op0, p64, nx, ny, nz);
    CLB_LAUNCH_CHECK("k_ir_init");
    return 0;
}

int clb_mg_ir_update(double* p64, const float* e, int64_t cells, void* stream) {
    CLB_REQUIRE(p64 && e && cells >= 0, "mg_ir_update: bad arguments");
    if (cells == 0) return 0;
    launch(blocks_for(cells, MGT), MGT, 0, CLB_STREAM(stream))(k_ir_update, p64, e, cells);
    CLB_LAUNCH_CHECK("k_ir_update");
    return 0;
}

int clb_mg_ir_store(const double* p64, float* p32, int64_t cells, void* stream) {
    CLB_REQUIRE(p64 && p32 && cells >= 0, "mg_ir_store: bad arguments");
    if (cells == 0) return 0;
    if (cells % 4 == 0 && (((uintptr_t)p32 | (uintptr_t)p64) & 15) == 0)
        launch(blocks_for(cells / 4, MGT), MGT, 0, CLB_STREAM(stream))(k_ir_store4, p64, p32, cells / 4);
    else
        launch(blocks_for(cells, MGT), MGT, 0, CLB_STREAM(stream))(k_ir_store, p64, p32, cells);
    CLB_LAUNCH_CHECK("k_ir_store");
    return 0;
}

// ---- tensor-core GEMM check ----------------------------------------------------------------------

int clb_tc_test_gemm(const void* a, const void* b, float* c, int M, int N, int K, int mn_major, void* stream) {
    CLB_REQUIRE(a && b && c, "tc_test_gemm: null pointer");
    CLB_REQUIRE(M > 0 && K > 0 && K % 8 == 0 && M % 8 == 0, "tc_test_gemm: M, K must be positive multiples of 8");
    CLB_REQUIRE(N == 16 || N == 32 || N == 64 || N == 128, "tc_test_gemm: N must be 16, 32, 64 or 128");
    const dim3 grid((M + tc::TC_M - 1) / tc::TC_M);
    cudaStream_t s = CLB_STREAM(stream);
    const __nv_bfloat16* A = (const __nv_bfloat16*)a;
    const __nv_bfloat16* B = (const __nv_bfloat16*)b;
#define CLB_TCG(AMN, BMN, NN)                                                                               \
    do {                                                                                                    \
        const size_t bytes = tc::tile_smem_bytes<NN>();                                                     \
        if (check_call(cudaFuncSetAttribute(tc::k_tc_test_gemm<AMN, BMN, NN>,                               \
                                            cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes),       \
                       "tc_test_gemm attribute"))                                                           \
            return 1;                                                                                       \
        tc::k_tc_test_gemm<AMN, BMN, NN><<<grid, tc::TC_THREADS, bytes, s>>>(A, B, c, M, K);                \
    } while (0)
    if (mn_major) {
        if (N == 16) CLB_TCG(true, true, 16);
        else if (N == 32) CLB_TCG(true, true, 32);
        else if (N == 64) CLB_TCG(true, true, 64);
        else CLB_TCG(true, true, 128);
    } else {
        if (N == 16) CLB_TCG(false, false, 16);
        else if (N == 32) CLB_TCG(false, false, 32);
        else if (N == 64) CLB_TCG(false, false, 64);
        else CLB_TCG(false, false, 128);
    }
#undef CLB_TCG
    CLB_LAUNCH_CHECK("k_tc_test_gemm");
    return 0;
}

// ---- 3-D convolutions and the U-Net's elementwise operations ------------------------------------

#define CLB_VOL_OK(B, D, H, W)                                                                   \
    CLB_REQUIRE((B) > 0 && (D) > 0 && (H) > 0 && (W) > 0 && (i64)(B) * (D) * (H) * (W) < (1ll << 31), \
                "volume %dx%dx%dx%d out of range", (B), (D), (H), (W))

static unsigned ew_blocks(i64 n) {
    const i64 b = (n + conv::EW - 1) / conv::EW;
    return (unsigned)(b < 148 * 32 ? (b > 0 ? b : 1) : 148 * 32);
}

int clb_conv3d_forward(const void* x, const void* wf, const float* bias, void* y, int B, int D, int H, int W, int cin,
                       int cout, int kpad, int relu, void* stream) {
    CLB_VOL_OK(B, D, H, W);
    CLB_REQUIRE(x && wf && y, "conv3d_forward: null pointer");
    CLB_REQUIRE(cin > 0 && cin % 8 == 0, "conv3d_forward: cin=%d must be a positive multiple of 8", cin);
    CLB_REQUIRE(kpad % 64 == 0 && kpad >= 27 * cin, "conv3d_forward: kpad=%d must be a multiple of 64 >= 27*cin", kpad);
    CLB_REQUIRE(cout == 16 || cout == 32 || cout == 64, "conv3d_forward: cout=%d not supported (16, 32, 64)", cout);
    CLB_REQUIRE(bias == nullptr || ((uintptr_t)bias & 15) == 0, "conv3d_forward: bias must be 16-byte aligned");
    conv::WinPlan pl;
    CLB_REQUIRE(conv::win_plan(D, H, W, cin, cout, B, pl), "conv3d_forward: no block shape fits %dx%dx%d", D, H, W);
    const conv::Vol g{B, D, H, W};
    const unsigned blocks = (unsigned)((i64)B * D * pl.ytiles * pl.xtiles);
    cudaStream_t s = CLB_STREAM(stream);
    const auto* X = (const __nv_bfloat16*)x;
    const auto* Wf = (const __nv_bfloat16*)wf;
    auto* Y = (__nv_bfloat16*)y;
#define CLB_FW(NN) \
    conv::k_conv_win<NN, false><<<blocks, conv::CW_THREADS, pl.smem, s>>>(X, Wf, bias, nullptr, Y, g, cin, kpad, relu, pl)
    if (cout == 16) CLB_FW(16);
    else if (cout == 32) CLB_FW(32);
    else CLB_FW(64);
#undef CLB_FW
    CLB_LAUNCH_CHECK("k_conv_win<forward>");
    return 0;
}

int clb_conv3d_dgrad(const void* dy, const void* wd, const void* mask_x, void* dx, int B, int D, int H, int W, int cout,
                     int cin, int kpad, void* stream) {
    CLB_VOL_OK(B, D, H, W);
    CLB_REQUIRE(dy && wd && dx, "conv3d_dgrad: null pointer");
    CLB_REQUIRE(cout > 0 && cout % 8 == 0, "conv3d_dgrad: cout=%d must be a positive multiple of 8", cout);
    CLB_REQUIRE(kpad % 64 == 0 && kpad >= 27 * cout, "conv3d_dgrad: kpad=%d must be a multiple of 64 >= 27*cout", kpad);
    CLB_REQUIRE(cin == 16 || cin == 32 || cin == 48 || cin == 64 || cin == 96,
                "conv3d_dgrad: cin=%d not supported (16, 32, 48, 64, 96)", cin);
    conv::WinPlan pl;
    CLB_REQUIRE(conv::win_plan(D, H, W, cout, cin, B, pl), "conv3d_dgrad: no block shape fits %dx%dx%d", D, H, W);
    const conv::Vol g{B, D, H, W};
    const unsigned blocks = (unsigned)((i64)B * D * pl.ytiles * pl.xtiles);
    cudaStream_t s = CLB_STREAM(stream);
    const auto* DY = (const __nv_bfloat16*)dy;
    const auto* Wd = (const __nv_bfloat16*)wd;
    const auto* MX = (const __nv_bfloat16*)mask_x;
    auto* DX = (__nv_bfloat16*)dx;
#define CLB_DG(NN) \
    conv::k_conv_win<NN, true><<<blocks, conv::CW_THREADS, pl.smem, s>>>(DY, Wd, nullptr, MX, DX, g, cout, kpad, 0, pl)
    if (cin == 16) CLB_DG(16);
    else if (cin == 32) CLB_DG(32);
    else if (cin == 48) CLB_DG(48);
    else if (cin == 64) CLB_DG(64);
    else CLB_DG(96);
#undef CLB_DG
    CLB_LAUNCH_CHECK("k_conv_win<dgrad>");
    return 0;
}

int clb_conv3d_wgrad(const void* x, const void* dy, float* dw, int B, int D, int H, int W, int cin, int cout,
                     int chunks_per_block, void* stream) {
    CLB_VOL_OK(B, D, H, W);
    CLB_REQUIRE(x && dy && dw, "conv3d_wgrad: null pointer");
    CLB_REQUIRE(cin > 0 && cin % 8 == 0, "conv3d_wgrad: cin=%d must be a positive multiple of 8", cin);
    CLB_REQUIRE(chunks_per_block > 0, "conv3d_wgrad: chunks_per_block must be positive");
    const conv::Vol g{B, D, H, W};
    const i64 chunks = ((i64)B * D * H * W + tc::TC_KC - 1) / tc::TC_KC;
    const dim3 grid((unsigned)((27 * cin + tc::TC_M - 1) / tc::TC_M),
                    (unsigned)((chunks + chunks_per_block - 1) / chunks_per_block));
    cudaStream_t s = CLB_STREAM(stream);
    const auto* X = (const __nv_bfloat16*)x;
    const auto* DY = (const __nv_bfloat16*)dy;
    if (cout == 16)
        conv::k_conv_wgrad<16><<<grid, tc::TC_THREADS, tc::tile_smem_bytes<16>(), s>>>(X, DY, dw, g, cin, chunks_per_block);
    else if (cout == 32)
        conv::k_conv_wgrad<32><<<grid, tc::TC_THREADS, tc::tile_smem_bytes<32>(), s>>>(X, DY, dw, g, cin, chunks_per_block);
    else if (cout == 64)
        conv::k_conv_wgrad<64><<<grid, tc::TC_THREADS, tc::tile_smem_bytes<64>(), s>>>(X, DY, dw, g, cin, chunks_per_block);
    else
        return set_error("conv3d_wgrad: cout=%d not supported (16, 32, 64)", cout);
    CLB_LAUNCH_CHECK("k_conv_wgrad");
    return 0;
}

int clb_conv3d_arrange_weights(const float* w, void* wf, void* wd, int cin, int cout, int kpad, int kpad2,
                               void* stream) {
    CLB_REQUIRE(w && wf, "conv3d_arrange_weights: null pointer");
    CLB_REQUIRE(kpad >= 27 * cin && (!wd || kpad2 >= 27 * cout), "conv3d_arrange_weights: K padding too small");
    const i64 total = (i64)cout * kpad + (wd ? (i64)cin * kpad2 : 0);
    conv::k_arrange_weights<<<ew_blocks(total), conv::EW, 0, CLB_STREAM(stream)>>>(
        w, (__nv_bfloat16*)wf, (__nv_bfloat16*)wd, cin, cout, kpad, kpad2);
    CLB_LAUNCH_CHECK("k_arrange_weights");
    return 0;
}

int clb_unet_avgpool2(const void* x, void* y, int B, int D, int H, int W, int C, void* stream) {
    CLB_VOL_OK(B, D, H, W);
    CLB_REQUIRE(D % 2 == 0 && H % 2 == 0 && W % 2 == 0, "unet_avgpool2: extents must be even");
    CLB_REQUIRE(C > 0 && C % 8 == 0, "unet_avgpool2: C=%d must be a multiple of 8", C);
    const conv::Vol g{B, D, H, W};
    conv::k_avgpool2<<<ew_blocks((i64)B * D * H * W * C / 64), conv::EW, 0, CLB_STREAM(stream)>>>(
        (const __nv_bfloat16*)x, (__nv_bfloat16*)y, g, C);
    CLB_LAUNCH_CHECK("k_avgpool2");
    return 0;
}

int clb_unet_avgpool2_backward(const void* dy, const void* x, void* dx, int B, int D, int H, int W, int C,
                               void* stream) {
    CLB_VOL_OK(B, D, H, W);
    CLB_REQUIRE(C > 0 && C % 8 == 0 && D % 2 == 0 && H % 2 == 0 && W % 2 == 0,
                "unet_avgpool2_backward: C=%d must be a multiple of 8 and extents even", C);
    const conv::Vol g{B, D, H, W};
    conv::k_avgpool2_backward<<<ew_blocks((i64)B * D * H * W * C / 8), conv::EW, 0, CLB_STREAM(stream)>>>(
        (const __nv_bfloat16*)dy, (const __nv_bfloat16*)x, (__nv_bfloat16*)dx, g, C);
    CLB_LAUNCH_CHECK("k_avgpool2_backward");
    return 0;
}

int clb_unet_upsample_concat(const void* coarse, const void* skip, void* out, int B, int D, int H, int W, int c1,
                             int c2, void* stream) {
    CLB_VOL_OK(B, D, H, W);
    CLB_REQUIRE(c1 > 0 && c2 > 0 && c1 % 8 == 0 && c2 % 8 == 0, "unet_upsample_concat: channels must be multiples of 8");
    const conv::Vol g{B, D, H, W};
    conv::k_upsample_concat<<<ew_blocks((i64)B * D * H * W * (c1 + c2) / 8), conv::EW, 0, CLB_STREAM(stream)>>>(
        (const __nv_bfloat16*)coarse, (const __nv_bfloat16*)skip, (__nv_bfloat16*)out, g, c1, c2);
    CLB_LAUNCH_CHECK("k_upsample_concat");
    return 0;
}

int clb_unet_upsample_concat_backward(const void* dout, void* dcoarse, void* dskip, int B, int D, int H, int W,
                                      int c1, int c2, void* stream) {
    CLB_VOL_OK(B, D, H, W);
    CLB_REQUIRE(c1 > 0 && c2 > 0 && c1 % 8 == 0 && c2 % 8 == 0 && D % 2 == 0 && H % 2 == 0 && W % 2 == 0,
                "unet_upsample_concat_backward: channels must be multiples of 8 and extents even");
    const conv::Vol g{B, D, H, W};
    conv::k_upsample_concat_backward<<<ew_blocks((i64)B * D * H * W * (c1 + c2) / 8), conv::EW, 0, CLB_STREAM(stream)>>>(
        (const __nv_bfloat16*)dout, (__nv_bfloat16*)dcoarse, (__nv_bfloat16*)dskip, g, c1, c2);
    CLB_LAUNCH_CHECK("k_upsample_concat_backward");
    return 0;
}

int clb_unet_head_forward(const void* h, const float* w, const float* b, float* out, int voxels, int C,
                          void* stream) {
    CLB_REQUIRE(C == 16, "unet_head_forward: C=%d must be 16", C);
    conv::k_head_forward<<<ew_blocks(voxels), conv::EW, 0, CLB_STREAM(stream)>>>((const __nv_bfloat16*)h, w, b, out,
                                                                                 voxels, C);
    CLB_LAUNCH_CHECK("k_head_forward");
    return 0;
}

int clb_unet_head_backward(const void* h, const float* w, const float* dout, void* dh, float* dw, float* db,
                           int voxels, int C, void* stream) {
    CLB_REQUIRE(C == 16, "unet_head_backward: C=%d must be 16", C);
    conv::k_head_backward<<<ew_blocks(voxels), conv::EW, 0, CLB_STREAM(stream)>>>(
        (const __nv_bfloat16*)h, w, dout, (__nv_bfloat16*)dh, dw, db, voxels, C);
    CLB_LAUNCH_CHECK("k_head_backward");
    return 0;
}

int clb_unet_bias_grad(const void* dy, float* db, int voxels, int C, void* stream) {
    CLB_REQUIRE(C > 0 && C <= 256 && C % 8 == 0, "unet_bias_grad: C=%d must be a multiple of 8 in 8..256", C);
    conv::k_bias_grad<<<ew_blocks((i64)voxels * C / 16), conv::EW, 0, CLB_STREAM(stream)>>>((const __nv_bfloat16*)dy, db,
                                                                                            voxels, C);
    CLB_LAUNCH_CHECK("k_bias_grad");
    return 0;
}

int clb_adam_step(float* p, const float* g, float* m, float* v, int64_t n, float lr, float beta1, float beta2, float eps,
                  int step, void* stream) {
    CLB_REQUIRE(p && g && m && v && n >= 0 && step >= 1, "adam_step: bad arguments");
    const float bc1 = 1.0f - powf(beta1, (float)step), bc2 = 1.0f - powf(beta2, (float)step);
    conv::k_adam<<<ew_blocks(n), conv::EW, 0, CLB_STREAM(stream)>>>(p, g, m, v, n, lr, beta1, beta2, eps, bc1, bc2);
    CLB_LAUNCH_CHECK("k_adam");
    return 0;
}

int clb_unet_pack_input(const float* b, const uint8_t* op0, const uint8_t* solid, const float* p, float scale_b,
                        float inv_s, int nx, int ny, int nz, int oi, int oj, int ok, void* x0, int slot, int D, int H,
                        int W, void* stream) {
    CLB_GRID_ARGS_OK(nx, ny, nz);
    CLB_REQUIRE(b && op0 && p && x0 && slot >= 0, "unet_pack_input: bad arguments");
    conv::k_pack_input<<<ew_blocks((i64)D * H * W), conv::EW, 0, CLB_STREAM(stream)>>>(
        b, op0, solid, p, scale_b, inv_s, nx, ny, nz, oi, oj, ok, (__nv_bfloat16*)x0, slot, D, H, W);
    CLB_LAUNCH_CHECK("k_pack_input");
    return 0;
}

int clb_unet_pack_target(const float* p, const float* p_prev, const uint8_t* op0, float inv_s, int nx, int ny,
                         int nz, int oi, int oj, int ok, float* t, float* m, int slot, int D, int H, int W,
                         void* stream) {
    CLB_GRID_ARGS_OK(nx, ny, nz);
    CLB_REQUIRE(p && p_prev && op0 && t && m && slot >= 0, "unet_pack_target: bad arguments");
    conv::k_pack_target<<<ew_blocks((i64)D * H * W), conv::EW, 0, CLB_STREAM(stream)>>>(
        p, p_prev, op0, inv_s, nx, ny, nz, oi, oj, ok, t, m, slot, D, H, W);
    CLB_LAUNCH_CHECK("k_pack_target");
    return 0;
}

int clb_unet_unpack_output(const float* out, const float* p_prev, const uint8_t* op0, float s, float* p, int nx,
                           int ny, int nz, int D, int H, int W, void* stream) {
    CLB_GRID_ARGS_OK(nx, ny, nz);
    CLB_REQUIRE(out && p_prev && op0 && p && D >= nx && H >= ny && W >= nz, "unet_unpack_output: bad arguments");
    conv::k_unpack_output<<<ew_blocks((i64)nx * ny * nz), conv::EW, 0, CLB_STREAM(stream)>>>(out, p_prev, op0, s, p, nx,
                                                                                           ny, nz, D, H, W);
    CLB_LAUNCH_CHECK("k_unpack_output");
    return 0;
}

int clb_unet_mse(const float* out, const float* t, const float* m, float* dout, float* loss, int64_t n, float inv_count,
                 void* stream) {
    CLB_REQUIRE(out && t && m && dout && loss && n >= 0, "unet_mse: bad arguments");
    conv::k_mse<<<ew_blocks(n), conv::EW, 0, CLB_STREAM(stream)>>>(out, t, m, dout, loss, n, inv_count);
    CLB_LAUNCH_CHECK("k_mse");
    return 0;
}

// ---- voxelisation ---------------------------------------------------------------------------------

int clb_voxelise_direction(float* out3) {
    CLB_REQUIRE(out3 != nullptr, "voxelise_direction: null output");
    voxelise_direction(out3);
    return 0;
}

int clb_voxelise_mesh(const float* triangles, uint8_t* mask, int triangle_count, int nx, int ny, int nz, float delta,
                      float ox, float oy, float oz, int cull, void* stream) {
    CLB_GRID_ARGS_OK(nx, ny, nz);
    CLB_REQUIRE(triangle_count >= 0, "voxelise_mesh: negative triangle count");
    CLB_REQUIRE(mask != nullptr, "voxelise_mesh: null mask");
    if (triangle_count == 0) return 0;
    CLB_REQUIRE(triangles != nullptr, "voxelise_mesh: null triangles");
    float d[3];
    voxelise_direction(d);
    const dim3 grid((nz + VOX_BK - 1) / VOX_BK, (ny + VOX_BJ - 1) / VOX_BJ, (nx + VOX_BI - 1) / VOX_BI);
    if (cull)
        k_voxelise<true><<<grid, VOX_THREADS, 0, CLB_STREAM(stream)>>>(triangles, mask, triangle_count, nx, ny, nz,
                                                                       delta, ox, oy, oz, d[0], d[1], d[2]);
    else
        k_voxelise<false><<<grid, VOX_THREADS, 0, CLB_STREAM(stream)>>>(triangles, mask, triangle_count, nx, ny, nz,
                                                                        delta, ox, oy, oz, d[0], d[1], d[2]);
    CLB_LAUNCH_CHECK("k_voxelise");
    return 0;
}

// ---- particle sources ------------------------------------------------------------------------------

int clb_source_cell_counts(const float* particles, int64_t n, float delta, int nx, int ny, int nz, int32_t* counts,
                           void* stream) {
    CLB_GRID_ARGS_OK(nx, ny, nz);
    CLB_REQUIRE(n >= 0 && delta > 0.0f && counts && (n == 0 || particles), "source_cell_counts: bad arguments");
    if (n == 0) return 0;
    k_source_cell_counts<<<blocks_for(n, PT), PT, 0, CLB_STREAM(stream)>>>(particles, n, delta, nx, ny, nz, counts);
    CLB_LAUNCH_CHECK("k_source_cell_counts");
    return 0;
}

int clb_source_keep(const float* particles, int64_t n, float delta, int nx, int ny, int nz, const uint8_t* outflow,
                    int32_t* keep, void* stream) {
    CLB_GRID_ARGS_OK(nx, ny, nz);
    CLB_REQUIRE(n >= 0 && delta > 0.0f && outflow && keep && (n == 0 || particles), "source_keep: bad arguments");
    if (n == 0) return 0;
    k_source_keep<<<blocks_for(n, PT), PT, 0, CLB_STREAM(stream)>>>(particles, n, delta, nx, ny, nz, outflow, keep);
    CLB_LAUNCH_CHECK("k_source_keep");
    return 0;
}

int clb_source_compact(const float* particles, const float* velocity, const int32_t* keep, const int32_t* slots,
                       int64_t n, float* particles_out, float* velocity_out, void* stream) {
    CLB_REQUIRE(n >= 0, "source_compact: negative n");
    if (n == 0) return 0;
    CLB_REQUIRE(particles && velocity && keep && slots && particles_out && velocity_out,
                "source_compact: null pointer");
    CLB_REQUIRE(particles_out != particles && velocity_out != velocity, "source_compact: outputs must not alias");
    k_source_compact<<<blocks_for(n, PT), PT, 0, CLB_STREAM(stream)>>>(particles, velocity, keep, slots, n,
                                                                        particles_out, velocity_out);
    CLB_LAUNCH_CHECK("k_source_compact");
    return 0;
}

int clb_source_missing(const int32_t* counts, const uint8_t* source, const uint8_t* solid, int target, int64_t cells,
                       int32_t* missing, void* stream) {
    CLB_REQUIRE(counts && source && missing && cells >= 0 && target >= 1, "source_missing: bad arguments");
    if (cells == 0) return 0;
    k_source_missing<<<blocks_for(cells, PT), PT, 0, CLB_STREAM(stream)>>>(counts, source, solid, target, cells,
                                                                            missing);
    CLB_LAUNCH_CHECK("k_source_missing");
    return 0;
}

int clb_source_spawn(const int32_t* missing, const int32_t* offsets, int nx, int ny, int nz, double delta, float vx,
                     float vy, float vz, uint64_t state_hi, uint64_t state_lo, uint64_t inc_hi, uint64_t inc_lo,
                     float* particles_out, float* velocity_out, void* stream) {
    CLB_GRID_ARGS_OK(nx, ny, nz);
    CLB_REQUIRE(missing && offsets && particles_out && velocity_out && delta > 0.0, "source_spawn: bad arguments");
    const i64 C = (i64)nx * ny * nz;
    k_source_spawn<<<blocks_for(C, PT), PT, 0, CLB_STREAM(stream)>>>(missing, offsets, C, ny, nz, delta, vx, vy, vz,
                                                                      state_hi, state_lo, inc_hi, inc_lo,
                                                                      particles_out, velocity_out);
    CLB_LAUNCH_CHECK("k_source_spawn");
    return 0;
}

// ---- the tolerance-mode iteration looping on the device --------------------------------------------
#include "solve_loop.cuh"

// ---- batched scenes --------------------------------------------------------------------------------
#include "batch_abi.cuh"

}  // extern "C"
