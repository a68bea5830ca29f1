/*
 * clb200.h -- C ABI of the Continuum Liquid B200 backend (libclb200.so).
 *
 * Each entry point replaces one OpenCL kernel dispatch (or one host stage function) of the
 * reference add-on's solver, Solver/Kernel/ of Continuum Liquid; the comment above each
 * declaration names the reference interface it replaces (file:line).
 *
 * Conventions
 *  - Every pointer is a device pointer to contiguous memory allocated by the caller; the library
 *    never allocates. Grids are float32 [nx][ny][nz] with k fastest (helper.cl:4-6), particles
 *    are float32 (N,3) records (particles.cl:56), counts and offsets int32, masks uint8.
 *  - `stream` is a cudaStream_t (NULL = legacy default stream). Every call only enqueues work.
 *  - Every function returns 0 on success and non-zero on failure; clb_last_error() then returns
 *    the message (thread-local). Launch-configuration and argument errors are reported this way;
 *    errors of asynchronous work surface at the caller's next synchronisation.
 *  - Device-side bounded waits that run out do not hang: they record a code that
 *    clb_device_error() returns (and clears).
 */
#ifndef CLB200_H
#define CLB200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- library ------------------------------------------------------------------------------ */

/* Selects the device and prepares kernel attributes. Replaces helper.py:51-69
 * select_opencl_device + cl.Context/CommandQueue creation (solver.py:29-37). */
int clb_init(int device);
/* Message of the last failed call on this thread ("" if none). */
const char* clb_last_error(void);
/* Reads and clears the device error word (0 = none, 1 = scan look-back wait gave up). Synchronous. */
int clb_device_error(uint32_t* code);
/* ABI version of this header (bumped on any signature change). */
int clb_abi_version(void);
/* Number of kernels this library has launched directly since it was loaded (replays of captured
 * CUDA graphs are not included). Host-side counter for launch accounting. */
int64_t clb_launch_count(void);

/* ---- particles: binning, scan, sort, P2G (Solver/Kernel/particles.py, OpenCL/particles.cl) -- */

/* particles.cl:44-59 count_particles_per_cell. Accumulates into bin_counts (the caller zero-fills
 * it, as particles.py:146 does). keys/ranks (nullable, int32[n]) receive each particle's bin and a
 * unique slot within it for clb_sort_particles. */
int clb_count_particles_per_cell(const float* particles, int32_t* bin_counts, int32_t* keys, int32_t* ranks,
                                 int64_t n, float inv_dx, int nx, int ny, int nz, void* stream);

/* Scratch bytes clb_exclusive_prefix_sum needs for `count` elements. */
int64_t clb_scan_scratch_bytes(int64_t count);

/* particles.py:39-70 exclusive_prefix_sum (particles.cl:61-108 scan_blocks_exclusive +
 * add_scanned_block_offsets), as one single-pass decoupled look-back scan. total (nullable)
 * receives the sum of all values. scratch: clb_scan_scratch_bytes(count) bytes, 16-byte aligned. */
int clb_exclusive_prefix_sum(const int32_t* values, int32_t* output, int32_t* total, int64_t count, void* scratch,
                             int64_t scratch_bytes, void* stream);

/* No counterpart in the reference. The same scan as clb_exclusive_prefix_sum for callers that
 * cannot allocate device memory -- a host application that has given its whole device memory budget
 * to its own pool, or code that must not add the device-wide synchronisation of cudaMalloc/cudaFree
 * to work already in flight. The look-back scratch is a fixed array inside this library
 * (16 + 8 * 16384 bytes, held on every GPU that loads the library until the process exits), so at
 * most CLB_SCAN_STATIC_MAX_COUNT elements are accepted; larger counts fail with an error. The first
 * call on a device looks up the array's device address (cudaGetSymbolAddress) with that device
 * current; make that first call before any stream capture. The address is kept for the life of the
 * process, so a caller that resets a device (cudaDeviceReset) must not call this function on that
 * device afterwards: the array may then live elsewhere. Every call clears the part of the array
 * it uses and all calls share it: calls whose work overlaps on the GPU (different streams, or
 * different host threads on one device) race and must be serialised by the caller. */
#define CLB_SCAN_STATIC_MAX_COUNT 67108864LL
int clb_exclusive_prefix_sum_static(const int32_t* values, int32_t* output, int32_t* total, int64_t count,
                                    void* stream);

/* particles.cl:110-133 sort_particles (+ the buffer swap of particles.py:119-140 is the caller's).
 * Stable counting-sort scatter: within a bin, particles keep their input order. perm and slot_keys
 * are int32[n] scratch. */
int clb_sort_particles(const float* particles, const float* velocity, float* particles_sorted, float* velocity_sorted,
                       const int32_t* bin_offsets, const int32_t* bin_counts, const int32_t* keys,
                       const int32_t* ranks, int32_t* perm, int32_t* slot_keys, int64_t n, void* stream);

/* particles.cl:135-227 particle_to_grid_gather. */
int clb_particle_to_grid_gather(const float* particles, const float* velocity, const int32_t* bin_offsets,
                                const int32_t* bin_counts, float* u, float* v, float* w, float* fluid_fraction,
                                float inv_dx, float inv_particles_per_cell, int nx, int ny, int nz, void* stream);

/* particles.py:73-171 particle_to_grid: zero-fill, count, scan, stable sort into
 * particles_work/velocity_work, gather. inv_dx and inv_particles_per_cell are the float32 values
 * the reference passes (FIELD_DTYPE(1.0 / dx), FIELD_DTYPE(1.0 / particles_per_cell)). Workspace: keys, ranks, perm, slot_keys int32[n];
 * scan_scratch of clb_scan_scratch_bytes(nx*ny*nz) bytes. The caller swaps the particle buffers
 * afterwards, as the reference does. */
int clb_particle_to_grid(const float* particles, const float* velocity, float* particles_work, float* velocity_work,
                         float* u, float* v, float* w, float* fluid_fraction, int32_t* bin_counts,
                         int32_t* bin_offsets, int32_t* keys, int32_t* ranks, int32_t* perm, int32_t* slot_keys,
                         void* scan_scratch, int64_t scan_scratch_bytes, int64_t n, float inv_dx,
                         float inv_particles_per_cell, int nx, int ny, int nz, void* stream);

/* particles.cl:135-227 particle_to_grid_gather, the same inputs and outputs, computed as a tiled
 * scatter that visits each particle once (the tolerance-mode path). Every weight is the reference's;
 * the sums of a cell are added in a different (fixed) order, so velocities agree with
 * clb_particle_to_grid_gather to float rounding (not bit for bit); the fluid fraction is identical
 * and a face that no particle weighs is 0 in both. Deterministic: the same inputs give the same bits on every run. */
int clb_particle_to_grid_gather_tiled(const float* particles, const float* velocity, const int32_t* bin_offsets,
                                      const int32_t* bin_counts, float* u, float* v, float* w, float* fluid_fraction,
                                      float inv_dx, float inv_particles_per_cell, int nx, int ny, int nz,
                                      void* stream);

/* clb_particle_to_grid with the tiled gather (particles.py:73-171 with
 * clb_particle_to_grid_gather_tiled as its last stage); same arguments. */
int clb_particle_to_grid_tiled(const float* particles, const float* velocity, float* particles_work,
                               float* velocity_work, float* u, float* v, float* w, float* fluid_fraction,
                               int32_t* bin_counts, int32_t* bin_offsets, int32_t* keys, int32_t* ranks,
                               int32_t* perm, int32_t* slot_keys, void* scan_scratch, int64_t scan_scratch_bytes,
                               int64_t n, float inv_dx, float inv_particles_per_cell, int nx, int ny, int nz,
                               void* stream);

/* particles.cl:229-262 grid_to_particle (particles.py:174-206), plus a FLIP/PIC blend:
 * flip_ratio = 1 is the reference's pure FLIP update. */
int clb_grid_to_particle(float* velocity, const float* particles, const float* u, const float* v, const float* w,
                         const float* u_old, const float* v_old, const float* w_old, int64_t n, float inv_dx, int nx,
                         int ny, int nz, float flip_ratio, void* stream);

/* particles.cl:264-276 advect_particles (particles.py:209-225). */
int clb_advect_particles(float* particles, const float* velocity, int64_t n, float dt, void* stream);

/* boundary_conditions.cl:69-97 particle_domain_bc (boundary_conditions.py:82-103). */
int clb_particle_domain_bc(float* particles, float* velocity, int64_t n, float lower, float upper_x, float upper_y,
                           float upper_z, void* stream);

/* boundary_conditions.cl:175-264 particle_obstacle_bc (boundary_conditions.py:106-132). */
int clb_particle_obstacle_bc(float* particles, const float* previous, float* velocity, const uint8_t* obstacle,
                             int64_t n, float inv_dx, int nx, int ny, int nz, void* stream);

/* solver.py:453-510 in one launch: grid_to_particle, the previous-position copy, advection,
 * particle_domain_bc and (obstacle != NULL) particle_obstacle_bc. previous_out is nullable. */
int clb_particle_update(float* particles, float* velocity, float* previous_out, const float* u, const float* v,
                        const float* w, const float* u_old, const float* v_old, const float* w_old,
                        const uint8_t* obstacle, int64_t n, float inv_dx, int nx, int ny, int nz, float flip_ratio,
                        float dt, float lower, float upper_x, float upper_y, float upper_z, void* stream);

/* ---- grid forces and boundary conditions --------------------------------------------------- */

/* velocity_update.cl:3-43 update_velocity (velocity_update.py:8-52). */
int clb_update_velocity(const float* u, const float* v, const float* w, float* result_u, float* result_v,
                        float* result_w, const float* fluid_fraction, float gravity_x, float gravity_y,
                        float gravity_z, float force_x, float force_y, float force_z, float rho, float nu,
                        float inv_dx2, float dt, int nx, int ny, int nz, void* stream);

/* boundary_conditions.cl:33-67 grid_domain_bc (boundary_conditions.py:36-50). */
int clb_grid_domain_bc(float* u, float* v, float* w, int nx, int ny, int nz, void* stream);

/* boundary_conditions.py:53-79 grid_obstacle_bc: boundary_conditions.cl:99-119 grid_obstacle_bc then
 * boundary_conditions.cl:121-173 extrapolate_obstacle_velocity, as two launches. */
int clb_grid_obstacle_bc(float* u, float* v, float* w, float* fluid_fraction, const uint8_t* obstacle, int nx, int ny,
                         int nz, void* stream);

/* pressure_solve.cl:3-24 pressure_rhs (pressure_solve.py:35-49). */
int clb_pressure_rhs(const float* u, const float* v, const float* w, const float* fluid_fraction, float* rhs,
                     float rho_over_dt, float inv_dx, int nx, int ny, int nz, void* stream);

/* pressure_solve.cl:26-47 pressure_correction (pressure_solve.py:88-114). */
int clb_pressure_correction(float* u, float* v, float* w, const float* pressure, float dt_over_rho, float inv_dx,
                            int nx, int ny, int nz, void* stream);

/* boundary_conditions.cl:18-31 neumann_domain_bc (boundary_conditions.py:22-33). */
int clb_neumann_domain_bc(float* pressure, int nx, int ny, int nz, void* stream);
/* The same two steps on an FP64 pressure (no counterpart in the reference): the gradient is taken
 * in FP64 and the updated velocity rounded once to float. Used to project with the FP64 pressure
 * of a refined solve, which is the one that meets the residual tolerance (its float32 rounding
 * alone leaves a relative residual of order 1e-6 at 48^3 and more on finer grids). */
int clb_pressure_correction_f64(float* u, float* v, float* w, const double* pressure, float dt_over_rho,
                                float inv_dx, int nx, int ny, int nz, void* stream);
int clb_neumann_domain_bc_f64(double* pressure, int nx, int ny, int nz, void* stream);

/* ---- moving colliders ------------------------------------------------------------------------- */
/* No counterpart in the reference: its colliders are voxelised once and stay at rest
 * (solver.py:132-139), so its obstacle conditions set solid faces and solid velocities to 0
 * (boundary_conditions.cl:99-264). Here a collider may move as a rigid body. `motion` points to 9
 * host floats (vx, vy, vz, wx, wy, wz, cx, cy, cz): velocity, angular velocity (rad/s) and the pivot
 * at the step's time in grid-local coordinates; the solid's velocity at x is V + W x (x - C). The
 * obstacle mask is the collider voxelised at its pose (clb_voxelise_mesh). With V = W = 0 each call
 * gives exactly what its static counterpart gives. */

/* clb_grid_obstacle_bc with solid faces set to the solid's velocity component at the face centre
 * (the u face of cell (i, j, k) at ((i+1) dx, (j+0.5) dx, (k+0.5) dx)), and solid cells next to
 * fluid given the solid's normal component (the fluid's averaged tangential velocity as before). */
int clb_grid_obstacle_bc_moving(float* u, float* v, float* w, float* fluid_fraction, const uint8_t* obstacle, int nx,
                                int ny, int nz, const float* motion, float dx, void* stream);
/* clb_particle_obstacle_bc where only the velocity relative to the solid (at the particle's
 * position) loses its inward normal component. */
int clb_particle_obstacle_bc_moving(float* particles, const float* previous, float* velocity,
                                    const uint8_t* obstacle, int64_t n, float inv_dx, int nx, int ny, int nz,
                                    const float* motion, void* stream);
/* No counterpart in the reference: clb_particle_update (or, with motion non-NULL, the moving-obstacle
 * form below; motion as there) walking the bins of 8 x 8 x 30-bin tiles: particles must be sorted by
 * bin, bin_offsets / bin_counts describing them (the counting sort of clb_particle_to_grid, before any
 * particle moves). Each block stages the six grid arrays its bins' particles sample in shared memory.
 * The same values as clb_particle_update, bit for bit. */
int clb_particle_update_tiled(float* particles, float* velocity, float* previous_out, const float* u, const float* v,
                              const float* w, const float* u_old, const float* v_old, const float* w_old,
                              const uint8_t* obstacle, const int32_t* bin_offsets, const int32_t* bin_counts,
                              int64_t n, float inv_dx, int nx, int ny, int nz, float flip_ratio, float dt, float lower,
                              float upper_x, float upper_y, float upper_z, const float* motion, void* stream);

/* clb_particle_update with the moving obstacle condition above (obstacle must not be null). */
int clb_particle_update_moving(float* particles, float* velocity, float* previous_out, const float* u, const float* v,
                               const float* w, const float* u_old, const float* v_old, const float* w_old,
                               const uint8_t* obstacle, int64_t n, float inv_dx, int nx, int ny, int nz,
                               float flip_ratio, float dt, float lower, float upper_x, float upper_y, float upper_z,
                               const float* motion, void* stream);

/* ---- multigrid: the reference's level arrays through the product kernels -------------------- */
/* The reference keeps five float32 arrays per level (mask, diagonal, weight_x, weight_y, weight_z;
 * multigrid.py:18-50, built by multigrid.cl:63-88 build_finest_operator and :90-180
 * restrict_residual). The stage functions that take those arrays (multigrid.py:53-249 w_cycle,
 * smooth, coarse_smooth; pressure_solve.py:10-85) convert them with these calls and run the
 * product kernels: the finest level as one byte per cell (see clb_mg_hierarchy), a coarse level as a
 * float4 (diagonal, wx, wy, wz) per cell (op4, 16-byte aligned) and a mask byte. A cell is fluid
 * where its mask is > 0, the reference's test. */

/* Finest level -> packed bytes. Counts into *invalid (device int, zeroed by the caller) the cells
 * whose diagonal is not an integer 0..7 or whose weights are not 0 or 1: such an operator is not a
 * finest operator and has no byte form. */
int clb_mg_pack_finest(const float* mask, const float* diagonal, const float* weight_x, const float* weight_y,
                       const float* weight_z, uint8_t* op0, int32_t* invalid, int nx, int ny, int nz, void* stream);
/* Packed bytes -> the finest operator arrays (what build_finest_operator writes). */
int clb_mg_unpack_finest(const uint8_t* op0, float* diagonal, float* weight_x, float* weight_y, float* weight_z,
                         int nx, int ny, int nz, void* stream);
/* Coarse level arrays -> float4 operator + mask byte, and back (mask written as 1.0 / 0.0). */
int clb_mg_pack_level(const float* mask, const float* diagonal, const float* weight_x, const float* weight_y,
                      const float* weight_z, float* op4, uint8_t* mask_out, int nx, int ny, int nz, void* stream);
int clb_mg_unpack_level(const float* op4, const uint8_t* mask_in, float* mask, float* diagonal, float* weight_x,
                        float* weight_y, float* weight_z, int nx, int ny, int nz, void* stream);
/* multigrid.py:190-220 smooth on a packed coarse-format level: `iterations` red-black iterations
 * (multigrid.cl:203-230 per colour; cells whose mask is 0 are set to 0). */
int clb_mg_smooth_level(float* p, const float* b, const float* op4, const uint8_t* mask, float delta, int iterations,
                        int nx, int ny, int nz, void* stream);
/* multigrid.py:223-249 coarse_smooth on a packed coarse-format level: `iterations` red-black
 * iterations in one block (multigrid.cl:232-264). */
int clb_mg_coarse_solve_level(float* p, const float* b, const float* op4, const uint8_t* mask, float delta,
                              int iterations, int nx, int ny, int nz, void* stream);

/* ---- multigrid, packed layout (product path) ------------------------------------------------ */

#define CLB_MG_MAX_LEVELS 16

/* A level pyramid as created by multigrid.py:18-50 create_multigrid_levels. Level 0 is the
 * simulation grid; its operator is one byte per cell (bits 0-2 diagonal, 3-5 wx/wy/wz, 6 fluid).
 * Coarse levels l >= 1 hold p, b (float32), a mask byte and a float4 (diagonal, wx, wy, wz).
 * Levels l >= fp16_level (when fp16_level > 0; no counterpart in the reference) store p and b as
 * IEEE half and the operator as four halves (8 bytes), with p and b scaled by powers of two taken
 * from rhs_norms (see clb_mg_w_cycle); such levels use sweep kinds 2-6 (0 and 1 mean 4), an alt
 * buffer of halves, and need fp16_scale. */
typedef struct clb_mg_hierarchy {
    int32_t levels;                      /* including level 0 */
    int32_t shape[CLB_MG_MAX_LEVELS][3]; /* nx, ny, nz per level (ghost layer included) */
    float delta;                         /* grid spacing used by every level (multigrid.py:65) */
    int32_t fp16_level;                  /* first FP16 level (>= 1 and <= levels - 2), 0: none */
    uint8_t* op0;                        /* level 0 packed operator */
    float* p[CLB_MG_MAX_LEVELS];         /* [0] unused: level-0 x is passed per call */
    float* b[CLB_MG_MAX_LEVELS];         /* [0] unused: level-0 rhs is passed per call */
    uint8_t* mask[CLB_MG_MAX_LEVELS];    /* [0] unused */
    void* op[CLB_MG_MAX_LEVELS];         /* [0] unused; float4 per cell */
    float* alt[CLB_MG_MAX_LEVELS];       /* optional second buffer per level (level 0 included, the
                                            level's element type), used by the fused sweep kinds */
    int32_t sweep[CLB_MG_MAX_LEVELS];    /* red-black sweep implementation per level:
                                            0 = default (two colour launches),
                                            1 = two colour launches, 16-byte row vectors when nz % 4 == 0,
                                            2 = one fused launch per iteration, 8x8x32 tiles (needs alt),
                                            3 = one fused launch per iteration, 4x4x32 tiles (needs alt),
                                            4 = two colour launches, one thread per cell,
                                            5 = one fused launch per two iterations, 8x8x32 tiles
                                                (needs alt; on FP32 coarse levels it runs as 6),
                                            6 = one fused launch per two iterations, 4x4x32 tiles
                                                (needs alt),
                                            7 = level 0 only: inside clb_mg_w_cycle, the whole level-0
                                                visit in pre + post launches on 3-D fluid tiles (the
                                                last pre-smoothing iteration fused with the residual and
                                                the restriction, the first post-smoothing one with the
                                                prolongation), when fused_tiles, alt[0] and an FP32
                                                level 1 are given, zero_outside is 2 and pre, post >= 1;
                                                otherwise as 1.
                                            All kinds give identical values. */
    float* fp16_scale;                   /* device float[4] written by clb_mg_w_cycle: sigma_b,
                                            1/sigma_p, kappa, 1/kappa (FP16 levels only) */
    const double* rhs_norms;             /* device: rhs_norms[0] = sum of squares of the level-0
                                            right-hand side over fluid cells (FP16 levels only; the
                                            out[0] of clb_mg_residual_norms / ir_step / fcg_step) */
    int32_t* fp16_inexact;               /* device counter: FP16 operator entries that did not convert
                                            exactly (clb_mg_build_coarse zeroes and fills it) */
    /* No counterpart in the reference: fluid tiles (NULL tiles / tile_counts: every sweep covers the
     * whole level). A tile is one plane i, four rows j and 32 cells k (128 on the finest level when
     * nz % 4 == 0), numbered (i * ceil(ny / 4) + j / 4) * ceil(nz / tile_k) + k / tile_k.
     * clb_mg_build_coarse lists the tiles that hold a fluid cell and zeroes every coarse p and b;
     * inside clb_mg_w_cycle the sweeps, restrictions and prolongations of FP32 levels then visit the
     * listed tiles only (cells that are not fluid keep the 0 the reference's sweeps would write). */
    int32_t* tiles[CLB_MG_MAX_LEVELS];   /* per level: clb_mg_tile_capacity(shape, level == 0) entries */
    int32_t* tile_counts;                /* device int32[CLB_MG_MAX_LEVELS]: listed tiles per level */
    int32_t zero_outside;                /* 1: level-0 x is 0 at every cell that is not fluid when
                                            clb_mg_w_cycle is called (the correction of the tolerance
                                            mode), so level-0 sweeps may skip tiles without fluid;
                                            2: as 1, and x counts as 0 inside the level-0 fluid tiles
                                            too (a correction from zero whose buffer still holds the
                                            previous one there): the first colour sweep ignores x, or
                                            x is zeroed first;
                                            0: level-0 sweeps cover the whole grid */
    /* No counterpart in the reference: the 3-D fluid tiles of level 0 (8 x 8 x 32 cells starting at
     * cell (1, 1, 1)) that sweep kind 7 walks; clb_mg_build_coarse lists them. NULL: kind 7 runs as 1. */
    int32_t* fused_tiles;                /* clb_mg_fused_tile_capacity(level-0 shape) entries */
    int32_t* fused_tile_count;           /* device int32: listed tiles */
    /* No counterpart in the reference: the fluid cells of each colour of the three coarsest levels, as
     * the one-launch visits of the third-coarsest level (a thread-block cluster) own them;
     * clb_mg_build_coarse lists them once per solve, so a launch does not. NULL: every launch lists
     * them itself (the same cells). */
    int32_t* cluster_lists;              /* clb_mg_cluster_list_capacity(h) entries */
    /* No counterpart in the reference: every correction a W-cycle prolongs (multigrid.cl:182-201, all
     * levels) is multiplied by it. 0 and 1 give the reference's W-cycle bit for bit. The reference's
     * piecewise-constant prolongation under-corrects; about 1.7 makes the W-cycle a much stronger
     * preconditioner of the tolerance mode's iteration. */
    float prolong_scale;
    /* No counterpart in the reference: 1 gives levels >= 1 their own smoothing counts (coarse_pre_smooth
     * sweeps before and coarse_post_smooth after the coarse-grid correction, the coarsest level's solve
     * coarse_pre_smooth + coarse_iterations); 0: every level uses clb_mg_w_cycle's counts (the reference). */
    int32_t coarse_smoothing;
    int32_t coarse_pre_smooth;
    int32_t coarse_post_smooth;
} clb_mg_hierarchy;

/* Number of tiles of a level of nx x ny x nz cells (finest != 0: the finest level's tile shape). */
int64_t clb_mg_tile_capacity(int nx, int ny, int nz, int finest);

/* Number of 3-D fluid tiles of level 0 (clb_mg_hierarchy.fused_tiles) for nx x ny x nz cells. */
int64_t clb_mg_fused_tile_capacity(int nx, int ny, int nz);

/* Entries of clb_mg_hierarchy.cluster_lists for the hierarchy's levels and shapes (0 when the visits of
 * its third-coarsest level do not run as one cluster launch). */
int64_t clb_mg_cluster_list_capacity(const clb_mg_hierarchy* h);

/* pressure_solve.cl:3-24 pressure_rhs fused with multigrid.cl:63-88 build_finest_operator, writing
 * the packed level-0 operator. */
int clb_mg_rhs_operator(const float* u, const float* v, const float* w, const float* fluid_fraction, float* rhs,
                        uint8_t* op0, float rho_over_dt, float inv_dx, int nx, int ny, int nz, void* stream);

/* Operator part of multigrid.cl:90-180 restrict_residual for every coarse level, once per solve. */
int clb_mg_build_coarse(const clb_mg_hierarchy* h, void* stream);

/* multigrid.py:53-187 w_cycle on level-0 unknown x and right-hand side rhs (pre/post/coarse sweeps
 * as pressure_solve.py:61-83: 2, 4, 64). */
int clb_mg_w_cycle(const clb_mg_hierarchy* h, float* x, const float* rhs, int pre_smooth, int post_smooth,
                   int coarse_iterations, void* stream);

/* No counterpart in the reference: one launch of sweep kind 7's level-0 kernel on the fused tiles
 * (clb_mg_build_coarse lists them): x_out = one red-black iteration of x_in on level 0, with
 *   mode 1: x_in counts as 0 (not read),
 *   mode 2: also the residual of the result restricted into level 1 (p = 0, b = the children's sum),
 *   mode 3: both, mode 4: x_in plus level 1's p prolonged first (multigrid.cl:182-201), mode 0: neither.
 * Cells of tiles that are not listed are not written. x_in and x_out must differ. */
int clb_mg_level0_iteration(const clb_mg_hierarchy* h, const float* x_in, float* x_out, const float* rhs, int mode,
                            void* stream);

/* multigrid.py:190-220 smooth: `iterations` red-black Gauss-Seidel iterations on one level (level 0
 * uses x and rhs; coarse levels their own p and b). With h->zero_outside = 1 and tile lists built by
 * clb_mg_build_coarse, the caller guarantees that the level's p (x on level 0) is 0 at every cell
 * that is not fluid, and an FP32 level is swept on its fluid tiles only (same values); with 2, level-0
 * x counts as 0 inside the fluid tiles as well. */
int clb_mg_smooth(const clb_mg_hierarchy* h, int level, float* x, const float* rhs, int iterations, void* stream);

/* Process-wide multigrid options (host-side switches, no device work):
 *  option 0: 1 (default) runs each visit of the second-coarsest level, including both coarse solves,
 *            as one single-block launch from shared memory; 0 launches one kernel per sweep as the
 *            reference does. Both give identical results.
 *  option 1: 1 (default) launches the pressure-solve kernels with programmatic dependent launch (a
 *            kernel's blocks are scheduled while its predecessor drains and wait for its completion
 *            on the device); 0 launches them with ordinary stream serialisation. Identical results.
 *  option 2: 1 (default) runs each visit of the third-coarsest level, with its two bottom visits, as
 *            one launch of a thread-block cluster (up to 16 CTAs, distributed shared memory) when the
 *            three levels share their storage type and fit; 0 goes level by level. Identical
 *            results.
 *  option 3: 1 (default) lets clb_mg_ir_step and clb_mg_fcg_step skip the cells that are not
 *            interior fluid cells (neither read nor written); the caller keeps p64_out, d_out and
 *            r_out at 0 there (zero them once per solve: clb_mg_ir_init and clb_mg_residual_norms
 *            with r_out do so for their outputs). 0 writes every cell. Identical results when the
 *            caller keeps that invariant.
 *  option 4: l > 0 makes clb_mg_w_cycle visit every level from l on once per visit of the level above
 *            (a V-cycle below level l - 1; the coarsest level then gets one coarse solve per visit of
 *            the level above), on every path (level by level, bottom and cluster launches); 0 (default)
 *            keeps the reference's two visits. A different preconditioner for the tolerance mode:
 *            values change. Read when a W-cycle is enqueued (and so fixed in a captured graph). */
int clb_mg_set_option(int option, int value);

/* Block-partial count used by clb_mg_residual_norms for a grid of `cells` cells. */
int clb_mg_residual_partials(int64_t cells);

/* FP64 relative-residual pieces over interior fluid cells of level 0: out[0] = sum (b - A p)^2,
 * out[1] = sum b^2 (A = multigrid.cl:25-43 apply_operator). p is float32 (p_is_double = 0) or
 * float64. r_out (nullable) receives the residual rounded to float32 (0 off the fluid). partials:
 * clb_mg_residual_partials(cells) double2 scratch. */
int clb_mg_residual_norms(const void* p, int p_is_double, const float* b, const uint8_t* op0, float delta, int nx,
                          int ny, int nz, float* r_out, void* partials, double* out, void* stream);

/* Iterative-refinement steps (FP64 accumulation of the pressure):
 *  init:   p64 = p32 at interior fluid cells, 0 elsewhere
 *  update: p64 += e
 *  store:  p32 = (float) p64 */
int clb_mg_ir_init(const float* p32, const uint8_t* op0, double* p64, int nx, int ny, int nz, void* stream);
/* One refinement update fused with the next residual: p64_out = p64_in + e, r_out = b - A p64_out
 * (FP64, rounded to float), out = [sum r^2, sum b^2]; p64_out must not alias p64_in. */
int clb_mg_ir_step(const double* p64_in, const float* e, double* p64_out, const float* b, const uint8_t* op0,
                   float delta, int nx, int ny, int nz, float* r_out, void* partials, double* out, void* stream);
int clb_mg_ir_update(double* p64, const float* e, int64_t cells, void* stream);
int clb_mg_ir_store(const double* p64, float* p32, int64_t cells, void* stream);

/* Flexible conjugate gradients preconditioned by one W-cycle (no counterpart in the reference; the
 * same FP64 accumulation as the refinement steps above, with the correction applied along
 * conjugate directions). For z = the W-cycle's correction e of the current residual r (float32,
 * the r_out of the previous step), d_in = the previous direction (float32, zeroed before the
 * first iteration) and state = double[4] {alpha, beta, d.Ad, has_direction} (zeroed before the
 * first iteration):
 *  dots: sums over interior fluid cells of (A z).d, (A z).z, z.r, d.r into partials4
 *        (clb_mg_residual_partials(cells) * 32 bytes), then beta = -(A z).d / d.Ad (0 for the
 *        first direction), d' = z + beta d, alpha = d'.r / d'.Ad' into state.
 *  step: d_out = d' (float32), p64_out = p64_in + alpha d', r_out = b - A p64_out (FP64, rounded
 *        to float), out = [sum r^2, sum b^2]; outputs must not alias inputs.
 * With alpha = 1 and beta = 0 the step is clb_mg_ir_step. */
int clb_mg_fcg_dots(const float* z, const float* d, const float* r, const uint8_t* op0, float delta, int nx, int ny,
                    int nz, void* partials4, double* state, void* stream);
int clb_mg_fcg_step(const double* p64_in, const float* z, const float* d_in, double* p64_out, float* d_out,
                    const double* state, const float* b, const uint8_t* op0, float delta, int nx, int ny, int nz,
                    float* r_out, void* partials, double* out, void* stream);

/* No counterpart in the reference: the tolerance-mode iteration as one CUDA graph that loops on the
 * device. A WHILE conditional node runs refinement after refinement (clb_mg_w_cycle from a zero
 * correction, then clb_mg_fcg_dots + clb_mg_fcg_step for method 0 or clb_mg_ir_step for method 1),
 * the FP64 buffers and directions alternating 0 -> 1 -> 0 ..., until the relative residual
 * sqrt(out[0] / out[1]) of a refinement is <= tol or max_cycles refinements have run; no host
 * round trip inside. After each refinement k (from 1) *cycles = k and history[k] = its relative
 * residual (k < history_len). The caller prepares the system and the initial residual, direction 0,
 * FCG state and the zeroed buffers as for the calls it replaces; after the graph ran the pressure is
 * in p64_0 if *cycles is even, else p64_1. Buffers and settings are fixed at creation (the hierarchy
 * is read then). */
typedef struct clb_solve_loop clb_solve_loop;
int clb_solve_loop_create(const clb_mg_hierarchy* h, float* correction, float* residual, float* direction0,
                          float* direction1, double* p64_0, double* p64_1, const float* rhs, double* fcg_state,
                          void* fcg_partials, void* partials, double* norms, int method, int pre_smooth,
                          int post_smooth, int coarse_iterations, double tol, int max_cycles, int* cycles,
                          double* history, int history_len, clb_solve_loop** out);
/* Resets *cycles to 0 and launches the loop on the stream (asynchronous). */
int clb_solve_loop_launch(clb_solve_loop* loop, int* cycles, void* stream);
/* Kernels one refinement of the loop launches (as clb_launch_count counts them). */
int clb_solve_loop_launches(const clb_solve_loop* loop);
int clb_solve_loop_destroy(clb_solve_loop* loop);

/* ---- tensor cores -------------------------------------------------------------------------- */

/* No counterpart in the reference (the learned warm start is new). Check of the tcgen05 GEMM core
 * used by the 3-D convolutions: c[M][N] (float32) = a * b^T in BF16 with FP32 accumulation.
 * mn_major = 0: a is [M][K] and b is [N][K] (K contiguous); 1: a is [K][M] and b is [K][N].
 * M and K multiples of 8, N one of 16, 32, 64, 128. */
int clb_tc_test_gemm(const void* a, const void* b, float* c, int M, int N, int K, int mn_major, void* stream);

/* Learned warm start (no counterpart in the reference): 3x3x3 convolutions, padding 1, on
 * channels-last BF16 volumes [B][D][H][W][C] as implicit GEMMs on tcgen05 with FP32 accumulation.
 * Taps are ordered (dz, dy, dx), dx fastest. Master weights are FP32 [27 * cin][cout].
 *  arrange_weights: wf[cout][kpad] (forward) and, when wd != NULL, wd[cin][kpad2] (data grad), BF16,
 *                   kpad >= 27*cin and kpad2 >= 27*cout multiples of 64, zero-padded.
 *  forward:  y = act(bias + conv(x)), cin % 8 == 0, cout in {16, 32, 64}, relu = 0/1; bias (nullable)
 *            16-byte aligned. Forward and data gradient stage an input tile in shared memory and read
 *            each tap as a shifted window of it (no per-tap gather).
 *  dgrad:    dx = conv^T(dy) * (mask_x > 0) (mask_x nullable), cout % 8 == 0, cin in {16,32,48,64,96}.
 *  wgrad:    dw[27*cin][cout] += sum over voxels (FP32 atomics; zero dw first), cout in {16, 32, 64};
 *            each block reduces chunks_per_block chunks of 64 voxels. */
int clb_conv3d_arrange_weights(const float* w, void* wf, void* wd, int cin, int cout, int kpad, int kpad2,
                               void* stream);
int clb_conv3d_forward(const void* x, const void* wf, const float* bias, void* y, int B, int D, int H, int W, int cin,
                       int cout, int kpad, int relu, void* stream);
int clb_conv3d_dgrad(const void* dy, const void* wd, const void* mask_x, void* dx, int B, int D, int H, int W, int cout,
                     int cin, int kpad, void* stream);
int clb_conv3d_wgrad(const void* x, const void* dy, float* dw, int B, int D, int H, int W, int cin, int cout,
                     int chunks_per_block, void* stream);
/* U-Net elementwise pieces (BF16 channels-last): 2x2x2 average pooling (extents of the fine volume
 * given) and its backward (adds into dx, then masks by x > 0); nearest 2x upsampling of `coarse`
 * concatenated with `skip` along channels, and its backward (dcoarse written, dskip added into);
 * the 1x1x1 output head (FP32 weights, C <= 16) and its backward (dh masked by h > 0, dw and db
 * accumulated); the bias gradient of a convolution (accumulated); an Adam step on FP32 parameters. */
int clb_unet_avgpool2(const void* x, void* y, int B, int D, int H, int W, int C, void* stream);
int clb_unet_avgpool2_backward(const void* dy, const void* x, void* dx, int B, int D, int H, int W, int C,
                               void* stream);
int clb_unet_upsample_concat(const void* coarse, const void* skip, void* out, int B, int D, int H, int W, int c1,
                             int c2, void* stream);
int clb_unet_upsample_concat_backward(const void* dout, void* dcoarse, void* dskip, int B, int D, int H, int W,
                                      int c1, int c2, void* stream);
int clb_unet_head_forward(const void* h, const float* w, const float* b, float* out, int voxels, int C, void* stream);
int clb_unet_head_backward(const void* h, const float* w, const float* dout, void* dh, float* dw, float* db,
                           int voxels, int C, void* stream);
int clb_unet_bias_grad(const void* dy, float* db, int voxels, int C, void* stream);
int clb_adam_step(float* p, const float* g, float* m, float* v, int64_t n, float lr, float beta1, float beta2, float eps,
                  int step, void* stream);

/* Network input/output next to the solver (no counterpart in the reference): pack_input writes
 * channels (b*scale_b, fluid, solid, p*inv_s, 0, 0, 0, 0) of grid cell (oi+z, oj+y, ok+x) into
 * voxel (z, y, x) of batch slot `slot` of a [B][D][H][W][8] BF16 volume (0 outside the grid; solid
 * nullable); pack_target writes t = (p - p_prev)*inv_s and the loss weight m = fluid;
 * unpack_output writes p = p_prev + out*s at fluid cells (0 elsewhere) from batch slot 0 of a
 * [D][H][W] FP32 volume; mse computes dout = 2 m (out - t) / count and adds
 * sum m (out - t)^2 / count to *loss. */
int clb_unet_pack_input(const float* b, const uint8_t* op0, const uint8_t* solid, const float* p, float scale_b,
                        float inv_s, int nx, int ny, int nz, int oi, int oj, int ok, void* x0, int slot, int D, int H,
                        int W, void* stream);
int clb_unet_pack_target(const float* p, const float* p_prev, const uint8_t* op0, float inv_s, int nx, int ny,
                         int nz, int oi, int oj, int ok, float* t, float* m, int slot, int D, int H, int W,
                         void* stream);
int clb_unet_unpack_output(const float* out, const float* p_prev, const uint8_t* op0, float s, float* p, int nx,
                           int ny, int nz, int D, int H, int W, void* stream);
int clb_unet_mse(const float* out, const float* t, const float* m, float* dout, float* loss, int64_t n, float inv_count,
                 void* stream);

/* ---- collider voxelisation (Solver/Kernel/voxelise_mesh.py, OpenCL/voxelise_mesh.cl) ------- */

/* voxelise_mesh.cl:24-48 voxelise_mesh: ORs 1 into mask for interior cells whose centre ray has an
 * odd hit count (voxelise_mesh.py:111-135 launches it once per mesh on the same mask). triangles:
 * float32 (T,3,3) world space; origin (ox,oy,oz) as voxelise_mesh.py:140. cull = 0 runs the
 * brute-force test over every triangle; 1 skips triangles that lie behind all rays of a block. */
int clb_voxelise_mesh(const float* triangles, uint8_t* mask, int triangle_count, int nx, int ny, int nz, float delta,
                      float ox, float oy, float oz, int cull, void* stream);

/* The ray direction of voxelise_mesh.cl:24 as three floats (host helper). */
int clb_voxelise_direction(float* out3);

/* ---- particle sources (source_particles.py:21-92, which the reference runs on the host) ------
 *
 * Cells are clamp(floor(p / delta), 0, n - 1) per axis (float32 division), as source_particles.py:21-25.
 *  cell_counts: counts[cell] += particles in it (zero counts first).
 *  keep:        keep[q] = 0 if particle q lies in an outflow cell, else 1 (source_particles.py:37-39);
 *               an exclusive scan of keep gives each kept particle's slot and the kept count.
 *  compact:     kept particles (and velocities) to their slots, order preserved.
 *  missing:     missing[c] = max(0, target - counts[c]) in non-solid source cells (solid nullable).
 *  spawn:       source_particles.py:42-75 fill_source: with offsets = exclusive scan of missing, the
 *               g-th new particle (cells in flat order) is placed at (cell + u) * delta, u the host
 *               stream's draws 3g..3g+2 after the PCG64 state (state_hi:state_lo, inc_hi:inc_lo) as
 *               numpy.random.Generator.random gives them (float64, stored as float32); velocity
 *               (vx, vy, vz). particles_out/velocity_out point at the first new record. The caller
 *               advances its generator by 3 * (number of new particles). */
int clb_source_cell_counts(const float* particles, int64_t n, float delta, int nx, int ny, int nz, int32_t* counts,
                           void* stream);
int clb_source_keep(const float* particles, int64_t n, float delta, int nx, int ny, int nz, const uint8_t* outflow,
                    int32_t* keep, void* stream);
int clb_source_compact(const float* particles, const float* velocity, const int32_t* keep, const int32_t* slots,
                       int64_t n, float* particles_out, float* velocity_out, void* stream);
int clb_source_missing(const int32_t* counts, const uint8_t* source, const uint8_t* solid, int target, int64_t cells,
                       int32_t* missing, void* stream);
int clb_source_spawn(const int32_t* missing, const int32_t* offsets, int nx, int ny, int nz, double delta, float vx,
                     float vy, float vz, uint64_t state_hi, uint64_t state_lo, uint64_t inc_hi, uint64_t inc_lo,
                     float* particles_out, float* velocity_out, void* stream);

/* ---- batched scenes (no counterpart in the reference, which bakes one scene at a time) -------
 *
 * Many independent scenes of different grid sizes advance together: every field of a batch holds the
 * scenes' grids back to back (level 0 for the simulation fields, one array per multigrid level for
 * the coarse levels), the particles of all scenes are one array, and each stage is one launch over
 * all scenes. A thread finds its scene from the prefix of the items (cells, particles or blocks) of
 * the scenes in the launch (a clb_batch_list) and runs the single-scene stage's code on that scene's
 * part, so each scene's values equal a single-scene run's. Bin keys are offset by each scene's cell
 * base, so one scan and one stable sort over the whole batch bin every scene at once. */
#define CLB_BATCH_MAX_SCENES 64

typedef struct clb_batch_scene {
    int32_t levels;                         /* multigrid levels of this scene */
    int32_t bottom;                         /* level run as one single-block bottom visit, -1: none */
    int32_t shape[CLB_MG_MAX_LEVELS][3];    /* per level, ghost layer included */
    int64_t base[CLB_MG_MAX_LEVELS];        /* first element of this scene's level-l cells */
    int64_t particle_base;                  /* first particle of this scene */
    int64_t particles;                      /* particle count */
    float delta;                            /* float32(dx), the multigrid spacing */
    float inv_dx;                           /* float32(1/dx) */
    float inv_dx2;                          /* float32(1/dx^2) */
    float rho_over_dt;                      /* float32(rho/dt) */
    float dt_over_rho;                      /* float32(dt/rho) */
    float lower;                            /* particle domain: float32(1.001 dx) */
    float upper[3];                         /* float32((n - 1.001) dx) per axis */
    int32_t pad;
} clb_batch_scene;

typedef struct clb_batch_list {             /* the scenes of one launch and the prefix of their items */
    const int32_t* scene;                   /* device int32[count]: scene indices */
    const int64_t* start;                   /* device int64[count + 1]: item prefix (start[0] = 0) */
    int32_t count;
    int32_t pad;
    int64_t total;                          /* start[count] (host copy) */
} clb_batch_list;

typedef struct clb_batch {
    int32_t scenes;
    int32_t levels;                         /* deepest scene's level count */
    const clb_batch_scene* geom;            /* device [scenes] */
    const clb_batch_scene* geom_host;       /* host copy of the same table */
    clb_batch_list particles;               /* every scene; items = its particles */
    clb_batch_list cells[CLB_MG_MAX_LEVELS];       /* scenes having level l; items = their level-l cells */
    clb_batch_list recurse[CLB_MG_MAX_LEVELS];     /* W-cycle: scenes that smooth and recurse at level l;
                                                      items = level-l cells */
    clb_batch_list recurse_coarse[CLB_MG_MAX_LEVELS]; /* the same scenes; items = level-(l+1) cells */
    clb_batch_list bottom[CLB_MG_MAX_LEVELS];      /* scenes whose bottom visit is at level l; items = 1 each */
    clb_batch_list coarse[CLB_MG_MAX_LEVELS];      /* scenes whose coarsest level l is solved on its own */
    clb_batch_list colour0;                 /* every scene; items = blocks of the level-0 row sweep */
    int32_t sweep0;                         /* level-0 sweep: 1 rows (needs colour0), 4 one thread per cell */
    int32_t vec0;                           /* 4: every scene's nz and level-0 base are multiples of 4 */
    int32_t reduce_blocks;                  /* blocks per scene of the FP64 reductions */
    int32_t bottom_ka, bottom_kb;           /* register tiles of the bottom visit (largest scene) */
    int32_t p2g_tiled;                      /* 1: P2G by the tiled scatter (clb_particle_to_grid_tiled), 0:
                                               the reference-order gather */
    int64_t bottom_smem;                    /* dynamic shared memory of the bottom visit (largest scene) */
    uint8_t* op0;                           /* level-0 packed operator of all scenes */
    float* p[CLB_MG_MAX_LEVELS];            /* levels >= 1 */
    float* b[CLB_MG_MAX_LEVELS];
    uint8_t* mask[CLB_MG_MAX_LEVELS];
    void* op[CLB_MG_MAX_LEVELS];            /* float4 per cell */
    float prolong_scale;                    /* factor of every prolonged correction (0 or 1: the reference's
                                               W-cycle), as clb_mg_hierarchy.prolong_scale */
    int32_t coarse_smoothing;               /* as clb_mg_hierarchy.coarse_smoothing */
    int32_t coarse_pre_smooth;
    int32_t coarse_post_smooth;
} clb_batch;

/* Stage API over a batch (pointers are the batch-wide arrays; per-scene constants come from geom).
 * particle_to_grid: zero-fill, count with scene-offset keys, one scan, one stable sort, P2G
 * (clb_particle_to_grid per scene, or clb_particle_to_grid_tiled when b->p2g_tiled is 1). Workspace as
 * clb_particle_to_grid for the batch totals. */
int clb_batch_particle_to_grid(const clb_batch* b, const float* particles, const float* velocity,
                               float* particles_work, float* velocity_work, float* u, float* v, float* w,
                               float* fluid_fraction, int32_t* bin_counts, int32_t* bin_offsets, int32_t* keys,
                               int32_t* ranks, int32_t* perm, int32_t* slot_keys, void* scan_scratch,
                               int64_t scan_scratch_bytes, float inv_particles_per_cell, void* stream);
int clb_batch_update_velocity(const clb_batch* b, const float* u, const float* v, const float* w, float* result_u,
                              float* result_v, float* result_w, const float* fluid_fraction, float gravity_x,
                              float gravity_y, float gravity_z, float force_x, float force_y, float force_z, float rho,
                              float nu, float dt, void* stream);
int clb_batch_grid_domain_bc(const clb_batch* b, float* u, float* v, float* w, void* stream);
int clb_batch_grid_obstacle_bc(const clb_batch* b, float* u, float* v, float* w, float* fluid_fraction,
                               const uint8_t* obstacle, void* stream);
/* pressure rhs + packed finest operator (clb_mg_rhs_operator), then every coarse operator. */
int clb_batch_rhs_operator(const clb_batch* b, const float* u, const float* v, const float* w,
                           const float* fluid_fraction, float* rhs, void* stream);
/* One W-cycle of every scene (clb_mg_w_cycle per scene). */
int clb_batch_w_cycle(const clb_batch* b, float* x, const float* rhs, int pre_smooth, int post_smooth,
                      int coarse_iterations, void* stream);
/* Per-scene FP64 sums (out[2 s] = sum r^2, out[2 s + 1] = sum b^2) of clb_mg_residual_norms;
 * partials: scenes * reduce_blocks double2. */
int clb_batch_residual_norms(const clb_batch* b, const void* p, int p_is_double, const float* rhs, float* r_out,
                             void* partials, double* out, void* stream);
int clb_batch_ir_init(const clb_batch* b, const float* p32, double* p64, void* stream);
/* p32 = (float) p64, then the Neumann ghost copy of both (clb_mg_ir_store + clb_neumann_domain_bc[_f64]). */
int clb_batch_ir_store(const clb_batch* b, double* p64, float* p32, void* stream);
/* clb_mg_fcg_dots / clb_mg_fcg_step per scene; state: double[4 * scenes]; partials4: scenes *
 * reduce_blocks * 32 bytes; partials: scenes * reduce_blocks double2; out: double[2 * scenes]. */
int clb_batch_fcg_dots(const clb_batch* b, const float* z, const float* d, const float* r, void* partials4,
                       double* state, void* stream);
int clb_batch_fcg_step(const clb_batch* b, const double* p64_in, const float* z, const float* d_in, double* p64_out,
                       float* d_out, const double* state, const float* rhs, float* r_out, void* partials, double* out,
                       void* stream);
/* pressure_correction (FP32 pressure, p_is_double = 0) or clb_pressure_correction_f64 per scene, and
 * the FP32 Neumann ghost copy (parity mode). */
int clb_batch_pressure_correction(const clb_batch* b, float* u, float* v, float* w, const void* pressure,
                                  int p_is_double, void* stream);
int clb_batch_neumann_domain_bc(const clb_batch* b, float* pressure, void* stream);
/* clb_particle_update per scene (obstacle may be an all-zero mask for scenes without a collider). */
int clb_batch_particle_update(const clb_batch* b, float* particles, float* velocity, const float* u, const float* v,
                              const float* w, const float* u_old, const float* v_old, const float* w_old,
                              const uint8_t* obstacle, float flip_ratio, float dt, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* CLB200_H */
