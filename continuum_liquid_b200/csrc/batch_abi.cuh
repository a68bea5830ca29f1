// C ABI of the batched stages (include/clb200.h, "batched scenes"). Included by clb200.cu inside its
// extern "C" block: the helpers below are C++ (static), the clb_batch_* functions are the exports.

extern "C++" {
namespace {

using namespace clb;

inline BList blist(const clb_batch_list& l) { return BList{l.scene, l.start, l.count}; }

// Grid of a grid-stride batched launch: enough blocks for the items, at most 32 per SM.
inline unsigned batch_grid(i64 total, int threads) {
    const i64 need = (total + threads - 1) / threads;
    const i64 cap = 148 * 32;
    return (unsigned)(need < 1 ? 1 : (need < cap ? need : cap));
}

int check_batch(const clb_batch* b) {
    CLB_REQUIRE(b != nullptr && b->geom != nullptr && b->geom_host != nullptr, "batch: null batch or geometry");
    CLB_REQUIRE(b->scenes >= 1 && b->scenes <= CLB_BATCH_MAX_SCENES, "batch: %d scenes (1..%d allowed)", b->scenes,
                CLB_BATCH_MAX_SCENES);
    CLB_REQUIRE(b->levels >= 1 && b->levels <= CLB_MG_MAX_LEVELS, "batch: %d levels", b->levels);
    CLB_REQUIRE(b->cells[0].count == b->scenes && b->particles.count == b->scenes,
                "batch: the level-0 and particle lists must hold every scene");
    CLB_REQUIRE(b->reduce_blocks >= 1, "batch: reduce_blocks must be >= 1");
    return 0;
}

bool list_ok(const clb_batch_list& l) { return l.count > 0 && l.total > 0 && l.scene && l.start; }

int batch_smooth(const clb_batch* B, int level, const clb_batch_list& L, float* x, const float* rhs, int iterations,
                 cudaStream_t s) {
    if (!list_ok(L) || iterations <= 0) return 0;
    for (int it = 0; it < iterations; ++it)
        for (int parity = 0; parity < 2; ++parity) {
            if (level == 0 && B->sweep0 == 1) {
                const unsigned blocks = (unsigned)B->colour0.total;
                if (B->vec0 == 4)
                    kb_rbgs_colour<4><<<blocks, dim3(32, 4), 0, s>>>(blist(B->colour0), B->geom, x, rhs, B->op0,
                                                                       parity);
                else
                    kb_rbgs_colour<1><<<blocks, dim3(32, 4), 0, s>>>(blist(B->colour0), B->geom, x, rhs, B->op0,
                                                                       parity);
                CLB_LAUNCH_CHECK("kb_rbgs_colour");
            } else if (level == 0) {
                kb_rbgs<true><<<batch_grid(L.total, BT), BT, 0, s>>>(blist(L), L.total, B->geom, 0, x, rhs, B->op0,
                                                                      nullptr, nullptr, parity);
                CLB_LAUNCH_CHECK("kb_rbgs");
            } else {
                kb_rbgs<false><<<batch_grid(L.total, BT), BT, 0, s>>>(blist(L), L.total, B->geom, level, B->p[level],
                                                                       B->b[level], nullptr,
                                                                       (const float4*)B->op[level], B->mask[level],
                                                                       parity);
                CLB_LAUNCH_CHECK("kb_rbgs");
            }
        }
    return 0;
}

// The factor of every prolonged correction (clb_batch.prolong_scale; 0 reads as 1).
static inline float batch_pscale(const clb_batch* B) { return B->prolong_scale > 0.0f ? B->prolong_scale : 1.0f; }

int batch_bottom(const clb_batch* B, int level, int pre, int post, int coarse_iters, cudaStream_t s) {
    const clb_batch_list& L = B->bottom[level];
    if (L.count <= 0) return 0;
    const size_t bytes = (size_t)B->bottom_smem;
    CLB_REQUIRE(bytes <= kBottomSmemLimit, "batch: bottom visit needs %zu bytes of shared memory", bytes);
#define CLB_BB(KA, KB)                                                                                           \
    kb_bottom_visit<KA, KB><<<L.count, BOTTOM_THREADS, bytes, s>>>(                                               \
        blist(L), B->geom, level, B->p[level], B->b[level], (const float4*)B->op[level], B->mask[level],          \
        B->p[level + 1], B->b[level + 1], (const float4*)B->op[level + 1], B->mask[level + 1], pre, post,         \
        coarse_iters, batch_pscale(B))
    const int ka = B->bottom_ka, kb = B->bottom_kb;
    if (ka <= 1 && kb <= 1) CLB_BB(1, 1);
    else if (ka <= 2 && kb <= 1) CLB_BB(2, 1);
    else if (ka <= 4 && kb <= 1) CLB_BB(4, 1);
    else if (ka <= 4 && kb <= 2) CLB_BB(4, 2);
    else if (ka <= 8 && kb <= 4) CLB_BB(8, 4);
    else CLB_REQUIRE(false, "batch: bottom visit tiles (%d, %d) too large", ka, kb);
#undef CLB_BB
    CLB_LAUNCH_CHECK("kb_bottom_visit");
    return 0;
}

int batch_coarse(const clb_batch* B, int level, int iterations, cudaStream_t s) {
    const clb_batch_list& L = B->coarse[level];
    if (L.count <= 0) return 0;
    int cmax = 0;
    for (int q = 0; q < B->scenes; ++q) {
        const clb_batch_scene& g = B->geom_host[q];
        if (g.levels - 1 == level) {
            const int C = g.shape[level][0] * g.shape[level][1] * g.shape[level][2];
            cmax = C > cmax ? C : cmax;
        }
    }
    CLB_REQUIRE(cmax <= COARSE_SMEM_CELLS, "batch: coarsest level of %d cells does not fit shared memory", cmax);
    kb_coarse_solve<<<L.count, COARSE_THREADS, coarse_smem_bytes(cmax), s>>>(
        blist(L), B->geom, level, B->p[level], B->b[level], (const float4*)B->op[level], B->mask[level], iterations);
    CLB_LAUNCH_CHECK("kb_coarse_solve");
    return 0;
}

// multigrid.py:53-187 w_cycle for every scene at once: at each level the scenes split into those whose
// coarsest level this is, those whose bottom visit runs here and those that smooth and recurse.
// pre0 / post0: the W-cycle's smoothing counts; levels >= 1 use the batch's coarse counts when it sets
// them (clb_batch.coarse_smoothing)
int batch_w_cycle(const clb_batch* B, int level, float* x, const float* rhs, int pre0, int post0, int coarse_iters,
                  cudaStream_t s) {
    const bool coarse = level > 0 && B->coarse_smoothing;
    const int pre = coarse ? B->coarse_pre_smooth : pre0, post = coarse ? B->coarse_post_smooth : post0;
    if (batch_coarse(B, level, pre + coarse_iters, s)) return 1;
    if (batch_bottom(B, level, pre, post, coarse_iters, s)) return 1;
    const clb_batch_list& R = B->recurse[level];
    if (!list_ok(R)) return 0;
    CLB_REQUIRE(level + 1 < B->levels, "batch: recursion below the deepest level");
    float* fp = level == 0 ? x : B->p[level];
    const float* fb = level == 0 ? rhs : B->b[level];
    if (batch_smooth(B, level, R, fp, fb, pre, s)) return 1;
    const clb_batch_list& RC = B->recurse_coarse[level];
    if (level == 0)
        kb_restrict<true><<<batch_grid(RC.total, BT), BT, 0, s>>>(blist(RC), RC.total, B->geom, 0, fp, fb, B->op0,
                                                                   nullptr, nullptr, B->p[1], B->b[1]);
    else
        kb_restrict<false><<<batch_grid(RC.total, BT), BT, 0, s>>>(
            blist(RC), RC.total, B->geom, level, fp, fb, nullptr, (const float4*)B->op[level], B->mask[level],
            B->p[level + 1], B->b[level + 1]);
    CLB_LAUNCH_CHECK("kb_restrict");
    if (batch_w_cycle(B, level + 1, x, rhs, pre0, post0, coarse_iters, s)) return 1;
    if (batch_w_cycle(B, level + 1, x, rhs, pre0, post0, coarse_iters, s)) return 1;
    if (level == 0)
        kb_prolong<true><<<batch_grid(R.total, BT), BT, 0, s>>>(blist(R), R.total, B->geom, 0, B->p[1], fp, B->op0,
                                                                 nullptr, batch_pscale(B));
    else
        kb_prolong<false><<<batch_grid(R.total, BT), BT, 0, s>>>(blist(R), R.total, B->geom, level, B->p[level + 1],
                                                                  fp, nullptr, B->mask[level], batch_pscale(B));
    CLB_LAUNCH_CHECK("kb_prolong");
    return batch_smooth(B, level, R, fp, fb, post, s);
}

}  // namespace
}  // extern "C++"

int clb_batch_particle_to_grid(const clb_batch* b, const float* particles, const float* velocity,
                               float* particles_work, float* velocity_work, float* u, float* v, float* w,
                               float* fluid_fraction, int32_t* bin_counts, int32_t* bin_offsets, int32_t* keys,
                               int32_t* ranks, int32_t* perm, int32_t* slot_keys, void* scan_scratch,
                               int64_t scan_scratch_bytes_, float inv_ppc, void* stream) {
    if (check_batch(b)) return 1;
    CLB_REQUIRE(particles && velocity && particles_work && velocity_work && u && v && w && fluid_fraction &&
                    bin_counts && bin_offsets && keys && ranks && perm && slot_keys,
                "batch_particle_to_grid: null pointer");
    cudaStream_t s = CLB_STREAM(stream);
    const i64 C = b->cells[0].total, n = b->particles.total;
    CLB_REQUIRE(C < (1ll << 31) && n < (1ll << 31), "batch_particle_to_grid: batch too large for int32 keys");
    if (check_call(cudaMemsetAsync(bin_counts, 0, sizeof(int32_t) * C, s), "zero bin_counts")) return 1;
    if (n > 0) {
        kb_bin_count<<<blocks_for(n, PT), PT, 0, s>>>(blist(b->particles), n, b->geom, particles, bin_counts, keys,
                                                       ranks);
        CLB_LAUNCH_CHECK("kb_bin_count");
    }
    if (clb_exclusive_prefix_sum(bin_counts, bin_offsets, nullptr, C, scan_scratch, scan_scratch_bytes_, stream))
        return 1;
    if (clb_sort_particles(particles, velocity, particles_work, velocity_work, bin_offsets, bin_counts, keys, ranks,
                           perm, slot_keys, n, stream))
        return 1;
    if (b->p2g_tiled) {  // each particle visited once per tile (the tolerance mode's P2G)
        i64 tiles = 0;
        for (int q = 0; q < b->scenes; ++q) {
            const clb_batch_scene& g = b->geom_host[q];
            int tj, tk;
            tiles += p2g_tiled_tiles(g.shape[0][0], g.shape[0][1], g.shape[0][2], &tj, &tk);
        }
        kb_p2g_tiled<<<(unsigned)tiles, P2GT_THREADS, P2GT_SMEM, s>>>(blist(b->cells[0]), b->geom, particles_work,
                                                                      velocity_work, bin_offsets, bin_counts, u, v, w,
                                                                      fluid_fraction, inv_ppc);
        CLB_LAUNCH_CHECK("kb_p2g_tiled");
        return 0;
    }
    kb_p2g<<<blocks_for(C * P2G_LANES, P2G_THREADS), P2G_THREADS, 0, s>>>(
        blist(b->cells[0]), C, b->geom, particles_work, velocity_work, bin_offsets, bin_counts, u, v, w,
        fluid_fraction, inv_ppc);
    CLB_LAUNCH_CHECK("kb_p2g");
    return 0;
}

int clb_batch_update_velocity(const clb_batch* b, const float* u, const float* v, const float* w, float* result_u,
                              float* result_v, float* result_w, const float* fluid_fraction, float gravity_x,
                              float gravity_y, float gravity_z, float force_x, float force_y, float force_z, float rho,
                              float nu, float dt, void* stream) {
    if (check_batch(b)) return 1;
    CLB_REQUIRE(u && v && w && result_u && result_v && result_w && fluid_fraction, "batch_update_velocity: null");
    const clb_batch_list& L = b->cells[0];
    kb_update_velocity<<<batch_grid(L.total, BT), BT, 0, CLB_STREAM(stream)>>>(
        blist(L), L.total, b->geom, u, v, w, result_u, result_v, result_w, fluid_fraction, gravity_x, gravity_y,
        gravity_z, force_x, force_y, force_z, rho, nu, dt);
    CLB_LAUNCH_CHECK("kb_update_velocity");
    return 0;
}

int clb_batch_grid_domain_bc(const clb_batch* b, float* u, float* v, float* w, void* stream) {
    if (check_batch(b)) return 1;
    CLB_REQUIRE(u && v && w, "batch_grid_domain_bc: null pointer");
    const clb_batch_list& L = b->cells[0];
    kb_grid_domain_bc<<<batch_grid(L.total, BT), BT, 0, CLB_STREAM(stream)>>>(blist(L), L.total, b->geom, u, v, w);
    CLB_LAUNCH_CHECK("kb_grid_domain_bc");
    return 0;
}

int clb_batch_grid_obstacle_bc(const clb_batch* b, float* u, float* v, float* w, float* fluid_fraction,
                               const uint8_t* obstacle, void* stream) {
    if (check_batch(b)) return 1;
    CLB_REQUIRE(u && v && w && fluid_fraction && obstacle, "batch_grid_obstacle_bc: null pointer");
    const clb_batch_list& L = b->cells[0];
    cudaStream_t s = CLB_STREAM(stream);
    kb_grid_obstacle_bc<<<batch_grid(L.total, BT), BT, 0, s>>>(blist(L), L.total, b->geom, u, v, w, fluid_fraction,
                                                                 obstacle);
    CLB_LAUNCH_CHECK("kb_grid_obstacle_bc");
    kb_extrapolate<<<batch_grid(L.total, BT), BT, 0, s>>>(blist(L), L.total, b->geom, u, v, w, obstacle);
    CLB_LAUNCH_CHECK("kb_extrapolate");
    return 0;
}

int clb_batch_rhs_operator(const clb_batch* b, const float* u, const float* v, const float* w,
                           const float* fluid_fraction, float* rhs, void* stream) {
    if (check_batch(b)) return 1;
    CLB_REQUIRE(u && v && w && fluid_fraction && rhs && b->op0, "batch_rhs_operator: null pointer");
    cudaStream_t s = CLB_STREAM(stream);
    const clb_batch_list& L = b->cells[0];
    kb_rhs_op0<<<batch_grid(L.total, BT), BT, 0, s>>>(blist(L), L.total, b->geom, u, v, w, fluid_fraction, rhs,
                                                       b->op0);
    CLB_LAUNCH_CHECK("kb_rhs_op0");
    for (int l = 1; l < b->levels; ++l) {
        const clb_batch_list& Lc = b->cells[l];
        if (!list_ok(Lc)) continue;
        CLB_REQUIRE(b->p[l] && b->b[l] && b->mask[l] && b->op[l], "batch: level %d has a null array", l);
        if (l == 1)
            kb_coarse_operator<0><<<batch_grid(Lc.total, BT), BT, 0, s>>>(blist(Lc), Lc.total, b->geom, l, b->op0,
                                                                           nullptr, nullptr, (float4*)b->op[l],
                                                                           b->mask[l]);
        else
            kb_coarse_operator<1><<<batch_grid(Lc.total, BT), BT, 0, s>>>(
                blist(Lc), Lc.total, b->geom, l, nullptr, (const float4*)b->op[l - 1], b->mask[l - 1],
                (float4*)b->op[l], b->mask[l]);
        CLB_LAUNCH_CHECK("kb_coarse_operator");
    }
    return 0;
}

int clb_batch_w_cycle(const clb_batch* b, float* x, const float* rhs, int pre_smooth, int post_smooth,
                      int coarse_iterations, void* stream) {
    if (check_batch(b)) return 1;
    CLB_REQUIRE(x && rhs && b->op0, "batch_w_cycle: null level-0 array");
    CLB_REQUIRE(pre_smooth >= 0 && post_smooth >= 0 && coarse_iterations >= 0, "batch_w_cycle: negative count");
    CLB_REQUIRE(!b->coarse_smoothing || (b->coarse_pre_smooth >= 0 && b->coarse_post_smooth >= 0),
                "batch_w_cycle: negative coarse-level count");
    CLB_REQUIRE(b->sweep0 == 4 || (b->sweep0 == 1 && list_ok(b->colour0)), "batch_w_cycle: bad level-0 sweep");
    return batch_w_cycle(b, 0, x, rhs, pre_smooth, post_smooth, coarse_iterations, CLB_STREAM(stream));
}

int clb_batch_residual_norms(const clb_batch* b, const void* p, int p_is_double, const float* rhs, float* r_out,
                             void* partials, double* out, void* stream) {
    if (check_batch(b)) return 1;
    CLB_REQUIRE(p && rhs && partials && out && b->op0, "batch_residual_norms: null pointer");
    cudaStream_t s = CLB_STREAM(stream);
    const int R = b->reduce_blocks;
    if (p_is_double)
        kb_residual_rows<double, RES_NORM><<<b->scenes * R, RN_THREADS, 0, s>>>(
            b->geom, R, (const double*)p, nullptr, nullptr, rhs, b->op0, r_out, (double2*)partials, nullptr, nullptr,
            nullptr);
    else
        kb_residual_rows<float, RES_NORM><<<b->scenes * R, RN_THREADS, 0, s>>>(
            b->geom, R, (const float*)p, nullptr, nullptr, rhs, b->op0, r_out, (double2*)partials, nullptr, nullptr,
            nullptr);
    CLB_LAUNCH_CHECK("kb_residual_rows");
    kb_reduce_partials<<<b->scenes, 256, 0, s>>>(R, (const double2*)partials, (double2*)out);
    CLB_LAUNCH_CHECK("kb_reduce_partials");
    return 0;
}

int clb_batch_ir_init(const clb_batch* b, const float* p32, double* p64, void* stream) {
    if (check_batch(b)) return 1;
    CLB_REQUIRE(p32 && p64 && b->op0, "batch_ir_init: null pointer");
    const clb_batch_list& L = b->cells[0];
    kb_ir_init<<<batch_grid(L.total, BT), BT, 0, CLB_STREAM(stream)>>>(blist(L), L.total, b->geom, p32, b->op0, p64);
    CLB_LAUNCH_CHECK("kb_ir_init");
    return 0;
}

int clb_batch_ir_store(const clb_batch* b, double* p64, float* p32, void* stream) {
    if (check_batch(b)) return 1;
    CLB_REQUIRE(p32 && p64, "batch_ir_store: null pointer");
    const clb_batch_list& L = b->cells[0];
    kb_store_neumann<<<batch_grid(L.total, BT), BT, 0, CLB_STREAM(stream)>>>(blist(L), L.total, b->geom, p64, p32);
    CLB_LAUNCH_CHECK("kb_store_neumann");
    return 0;
}

int clb_batch_fcg_dots(const clb_batch* b, const float* z, const float* d, const float* r, void* partials4,
                       double* state, void* stream) {
    if (check_batch(b)) return 1;
    CLB_REQUIRE(z && d && r && partials4 && state && b->op0, "batch_fcg_dots: null pointer");
    cudaStream_t s = CLB_STREAM(stream);
    const int R = b->reduce_blocks;
    kb_fcg_dots<<<b->scenes * R, RN_THREADS, 0, s>>>(b->geom, R, z, d, r, b->op0, (Sum4*)partials4);
    CLB_LAUNCH_CHECK("kb_fcg_dots");
    kb_fcg_scalars<<<b->scenes, 256, 0, s>>>(R, (const Sum4*)partials4, state);
    CLB_LAUNCH_CHECK("kb_fcg_scalars");
    return 0;
}

int clb_batch_fcg_step(const clb_batch* b, const double* p64_in, const float* z, const float* d_in, double* p64_out,
                       float* d_out, const double* state, const float* rhs, float* r_out, void* partials, double* out,
                       void* stream) {
    if (check_batch(b)) return 1;
    CLB_REQUIRE(p64_in && z && d_in && p64_out && d_out && state && rhs && r_out && partials && out && b->op0,
                "batch_fcg_step: null pointer");
    CLB_REQUIRE(p64_in != p64_out && d_in != d_out, "batch_fcg_step: outputs must not alias inputs");
    cudaStream_t s = CLB_STREAM(stream);
    const int R = b->reduce_blocks;
    kb_residual_rows<double, RES_FCG><<<b->scenes * R, RN_THREADS, 0, s>>>(
        b->geom, R, p64_in, z, p64_out, rhs, b->op0, r_out, (double2*)partials, d_in, d_out, state);
    CLB_LAUNCH_CHECK("kb_residual_rows");
    kb_reduce_partials<<<b->scenes, 256, 0, s>>>(R, (const double2*)partials, (double2*)out);
    CLB_LAUNCH_CHECK("kb_reduce_partials");
    return 0;
}

int clb_batch_pressure_correction(const clb_batch* b, float* u, float* v, float* w, const void* pressure,
                                  int p_is_double, void* stream) {
    if (check_batch(b)) return 1;
    CLB_REQUIRE(u && v && w && pressure, "batch_pressure_correction: null pointer");
    const clb_batch_list& L = b->cells[0];
    if (p_is_double)
        kb_pressure_correction<double><<<batch_grid(L.total, BT), BT, 0, CLB_STREAM(stream)>>>(
            blist(L), L.total, b->geom, u, v, w, (const double*)pressure);
    else
        kb_pressure_correction<float><<<batch_grid(L.total, BT), BT, 0, CLB_STREAM(stream)>>>(
            blist(L), L.total, b->geom, u, v, w, (const float*)pressure);
    CLB_LAUNCH_CHECK("kb_pressure_correction");
    return 0;
}

int clb_batch_neumann_domain_bc(const clb_batch* b, float* pressure, void* stream) {
    if (check_batch(b)) return 1;
    CLB_REQUIRE(pressure, "batch_neumann_domain_bc: null pointer");
    const clb_batch_list& L = b->cells[0];
    kb_neumann<<<batch_grid(L.total, BT), BT, 0, CLB_STREAM(stream)>>>(blist(L), L.total, b->geom, pressure);
    CLB_LAUNCH_CHECK("kb_neumann");
    return 0;
}

int clb_batch_particle_update(const clb_batch* b, float* particles, float* velocity, const float* u, const float* v,
                              const float* w, const float* u_old, const float* v_old, const float* w_old,
                              const uint8_t* obstacle, float flip_ratio, float dt, void* stream) {
    if (check_batch(b)) return 1;
    CLB_REQUIRE(particles && velocity && u && v && w && u_old && v_old && w_old && obstacle,
                "batch_particle_update: null pointer");
    const i64 n = b->particles.total;
    if (n == 0) return 0;
    kb_particle_update<<<blocks_for(n, PT), PT, 0, CLB_STREAM(stream)>>>(
        blist(b->particles), n, b->geom, particles, velocity, u, v, w, u_old, v_old, w_old, obstacle, flip_ratio, dt);
    CLB_LAUNCH_CHECK("kb_particle_update");
    return 0;
}
