// ORACLE — test infrastructure only. Nothing in the product path links, loads or calls this file.
//
// CPU restatement of Continuum Liquid's OpenCL FLIP kernels (Solver/Kernel/OpenCL/*.cl). Each function
// follows one reference kernel and cites the file:line it restates. Work-group algorithms are restated
// serially with the reference's reduction order (particles.cl:166-211 lane striding and tree;
// particles.cl:61-99 Blelloch up/down sweep).
//
// Floating-point semantics: built with -ffp-contract=off and no fast-math, so every + - * / is a
// separately rounded IEEE binary32 (or binary64) operation, sqrt is correctly rounded, and the
// OpenCL vector builtins are restated as plain left-to-right expressions:
//   dot(a,b)   = a.x*b.x + a.y*b.y + a.z*b.z
//   cross(a,b) = (a.y*b.z - a.z*b.y, a.z*b.x - a.x*b.z, a.x*b.y - a.y*b.x)
//   length(a)  = sqrt(dot(a,a)),  normalize(a) = a / length(a) per component.
// The reference runs on whatever OpenCL compiler the user has; what contraction or division precision
// that compiler would apply cannot be known here, so this restatement defines the semantics.
//
// Parity status: unpinned by the reference itself. The reference has no tests, fixtures or golden
// vectors, and it cannot run in this environment (no OpenCL runtime). The restatement is pinned
// instead by hand-derived known-answer tests of the reference's documented semantics (tests/).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

typedef int64_t i64;

namespace {

// helper.cl:4-6 grid_index (k fastest). 64-bit so grids up to 1024^3 do not overflow.
inline i64 gidx(int i, int j, int k, int ny, int nz) { return ((i64)i * ny + j) * nz + k; }

// helper.cl:8-15 grid_coordinates
inline void gcoord(i64 index, int ny, int nz, int& i, int& j, int& k) {
    const i64 yz = (i64)ny * nz;
    i = (int)(index / yz);
    const i64 rem = index - (i64)i * yz;
    j = (int)(rem / nz);
    k = (int)(rem - (i64)j * nz);
}

// helper.cl:21-23 is_interior_cell
inline bool interior(int i, int j, int k, int nx, int ny, int nz) {
    return i > 0 && j > 0 && k > 0 && i < nx - 1 && j < ny - 1 && k < nz - 1;
}

inline int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// particles.cl:3-6 interpolation_base: clamp(convert_int3_rtn(p*inv_dx - 0.5f), 0, n-2)
inline void interpolation_base(const float* p, float inv_dx, int nx, int ny, int nz, int b[3]) {
    const float x = p[0] * inv_dx - 0.5f;
    const float y = p[1] * inv_dx - 0.5f;
    const float z = p[2] * inv_dx - 0.5f;
    b[0] = clampi((int)std::floor(x), 0, nx - 2);
    b[1] = clampi((int)std::floor(y), 0, ny - 2);
    b[2] = clampi((int)std::floor(z), 0, nz - 2);
}

inline float fmaxf_(float a, float b) { return a > b ? a : b; }

// particles.cl:12-42 staggered_interpolation_base / fraction / weight / sample_field
inline void staggered_base_fraction(const float* p, float inv_dx, const float off[3], int nx, int ny, int nz,
                                    int base[3], float frac[3]) {
    const int lim[3] = {nx - 2, ny - 2, nz - 2};
    for (int a = 0; a < 3; ++a) {
        const float s = p[a] * inv_dx - off[a];
        base[a] = clampi((int)std::floor(s), 0, lim[a]);
        float f = p[a] * inv_dx - off[a] - (float)base[a];
        f = f < 0.0f ? 0.0f : (f > 1.0f ? 1.0f : f);
        frac[a] = f;
    }
}

inline float sample_field(const float* field, const int base[3], const float frac[3], int ny, int nz) {
    float value = 0.0f;
    for (int ox = 0; ox <= 1; ++ox)
        for (int oy = 0; oy <= 1; ++oy)
            for (int oz = 0; oz <= 1; ++oz) {
                const float wx = ox ? frac[0] : 1.0f - frac[0];
                const float wy = oy ? frac[1] : 1.0f - frac[1];
                const float wz = oz ? frac[2] : 1.0f - frac[2];
                const float wgt = wx * wy * wz;
                value += wgt * field[gidx(base[0] + ox, base[1] + oy, base[2] + oz, ny, nz)];
            }
    return value;
}

}  // namespace

extern "C" {

// ---------------------------------------------------------------------------------------------
// Particles (particles.cl)
// ---------------------------------------------------------------------------------------------

// Bin key per particle (particles.cl:3-6 + helper.cl:4-6); not a reference kernel, a test helper.
void orc_bin_keys(const float* pos, int32_t* keys, i64 n, float inv_dx, int nx, int ny, int nz) {
#pragma omp parallel for schedule(static)
    for (i64 p = 0; p < n; ++p) {
        int b[3];
        interpolation_base(pos + 3 * p, inv_dx, nx, ny, nz, b);
        keys[p] = (int32_t)gidx(b[0], b[1], b[2], ny, nz);
    }
}

// particles.cl:44-59 count_particles_per_cell (accumulates; the caller zero-fills first as
// particles.py:146 does).
void orc_count_particles_per_cell(const float* pos, int32_t* counts, i64 n, float inv_dx, int nx, int ny, int nz) {
    for (i64 p = 0; p < n; ++p) {
        int b[3];
        interpolation_base(pos + 3 * p, inv_dx, nx, ny, nz, b);
        counts[gidx(b[0], b[1], b[2], ny, nz)] += 1;
    }
}

// particles.cl:61-99 scan_blocks_exclusive: one work-group of L lanes scans 2L elements (Blelloch
// up-sweep, clear, down-sweep) and writes the block total to block_sums[group].
void orc_scan_blocks_exclusive(const int32_t* input, int32_t* output, int32_t* block_sums, i64 count, int L) {
    const int S = 2 * L;
    const i64 groups = (count + S - 1) / S;
    std::vector<int32_t> scratch(S);
    for (i64 g = 0; g < groups; ++g) {
        const i64 start = g * S;
        for (int l = 0; l < L; ++l) {
            const i64 first = start + l, second = first + L;
            scratch[l] = first < count ? input[first] : 0;
            scratch[l + L] = second < count ? input[second] : 0;
        }
        for (int offset = 1; offset < S; offset <<= 1)
            for (int l = 0; l < L; ++l) {
                const i64 target = (i64)(l + 1) * offset * 2 - 1;
                if (target < S) scratch[target] += scratch[target - offset];
            }
        block_sums[g] = scratch[S - 1];
        scratch[S - 1] = 0;
        for (int offset = S >> 1; offset > 0; offset >>= 1)
            for (int l = 0; l < L; ++l) {
                const i64 target = (i64)(l + 1) * offset * 2 - 1;
                if (target < S) {
                    const int32_t left = scratch[target - offset];
                    scratch[target - offset] = scratch[target];
                    scratch[target] += left;
                }
            }
        for (int l = 0; l < L; ++l) {
            const i64 first = start + l, second = first + L;
            if (first < count) output[first] = scratch[l];
            if (second < count) output[second] = scratch[l + L];
        }
    }
}

// particles.cl:101-108 add_scanned_block_offsets
void orc_add_scanned_block_offsets(int32_t* values, const int32_t* block_offsets, i64 count, int elements_per_block) {
    for (i64 i = 0; i < count; ++i) values[i] += block_offsets[i / elements_per_block];
}

// particles.py:39-70 exclusive_prefix_sum: levels of scan_blocks_exclusive going up, then
// add_scanned_block_offsets going down. Writes the full exclusive scan into `output` and the
// top-level total into *total. L = REDUCTION_THREADS_PER_BLOCK (kernel_config.py:7, 256 on GPU).
void orc_exclusive_prefix_sum(const int32_t* values, int32_t* output, i64 count, int L, int32_t* total) {
    const i64 S = 2 * (i64)L;
    std::vector<std::vector<int32_t>> outs, sums;
    std::vector<const int32_t*> inputs;
    std::vector<i64> counts;
    i64 level_count = count;
    const int32_t* in = values;
    while (true) {
        const i64 blocks = (level_count + S - 1) / S;
        outs.emplace_back(level_count);
        sums.emplace_back(std::max<i64>(blocks, 1));
        counts.push_back(level_count);
        orc_scan_blocks_exclusive(in, outs.back().data(), sums.back().data(), level_count, L);
        if (blocks <= 1) break;
        in = sums.back().data();
        level_count = blocks;
    }
    for (int level = (int)outs.size() - 2; level >= 0; --level)
        orc_add_scanned_block_offsets(outs[level].data(), outs[level + 1].data(), counts[level], (int)S);
    std::memcpy(output, outs[0].data(), sizeof(int32_t) * count);
    if (total) *total = sums.back()[0];
}

// particles.cl:110-133 sort_particles. The reference's atomic cursor makes the order within a bin
// nondeterministic on a parallel device; restated serially in particle-index order, which is the
// stable counting-sort order.
void orc_sort_particles(const float* pos, const float* vel, float* pos_sorted, float* vel_sorted,
                        const int32_t* offsets, int32_t* cursors, i64 n, float inv_dx, int nx, int ny, int nz) {
    for (i64 p = 0; p < n; ++p) {
        int b[3];
        interpolation_base(pos + 3 * p, inv_dx, nx, ny, nz, b);
        const i64 bin = gidx(b[0], b[1], b[2], ny, nz);
        const i64 local = cursors[bin]++;
        const i64 dst = 3 * ((i64)offsets[bin] + local);
        for (int a = 0; a < 3; ++a) {
            pos_sorted[dst + a] = pos[3 * p + a];
            vel_sorted[dst + a] = vel[3 * p + a];
        }
    }
}

// particles.cl:135-227 particle_to_grid_gather. One work-group of `lanes` lanes per cell; lane l
// visits neighbour bins l, l+lanes, ...; partial sums are tree-reduced with offsets lanes/2 ... 1.
void orc_particle_to_grid_gather(const float* pos, const float* vel, const int32_t* offsets, const int32_t* counts,
                                 float* u, float* v, float* w, float* ff, float inv_dx, float inv_ppc, int nx, int ny,
                                 int nz, int lanes) {
    const i64 C = (i64)nx * ny * nz;
#pragma omp parallel for schedule(dynamic, 4096)
    for (i64 index = 0; index < C; ++index) {
        int ci, cj, ck;
        gcoord(index, ny, nz, ci, cj, ck);
        float vs[64][3], ws[64][3];
        int cnt[64];
        const float gx = (float)ci, gy = (float)cj, gz = (float)ck;
        const float up[3] = {gx + 1.0f, gy + 0.5f, gz + 0.5f};
        const float vp[3] = {gx + 0.5f, gy + 1.0f, gz + 0.5f};
        const float wp[3] = {gx + 0.5f, gy + 0.5f, gz + 1.0f};
        for (int lane = 0; lane < lanes; ++lane) {
            float vsum[3] = {0.0f, 0.0f, 0.0f}, wsum[3] = {0.0f, 0.0f, 0.0f};
            int inside = 0;
            for (int nb = lane; nb < 27; nb += lanes) {
                const int ox = nb / 9 - 1, oy = (nb / 3) % 3 - 1, oz = nb % 3 - 1;
                const int bx = ci + ox;
                if (bx < 0 || bx >= nx - 1) continue;
                const int by = cj + oy;
                if (by < 0 || by >= ny - 1) continue;
                const int bz = ck + oz;
                if (bz < 0 || bz >= nz - 1) continue;
                const i64 bin = gidx(bx, by, bz, ny, nz);
                const i64 begin = offsets[bin], end = begin + counts[bin];
                for (i64 q = begin; q < end; ++q) {
                    const float* P = pos + 3 * q;
                    const float* V = vel + 3 * q;
                    const float s0 = P[0] * inv_dx, s1 = P[1] * inv_dx, s2 = P[2] * inv_dx;
                    const int pc0 = clampi((int)s0, 1, nx - 2);
                    const int pc1 = clampi((int)s1, 1, ny - 2);
                    const int pc2 = clampi((int)s2, 1, nz - 2);
                    inside += (pc0 == ci && pc1 == cj && pc2 == ck) ? 1 : 0;
                    const float s[3] = {s0, s1, s2};
                    float wu[3], wv[3], ww[3];
                    for (int a = 0; a < 3; ++a) {
                        wu[a] = fmaxf_(0.0f, 1.0f - std::fabs(s[a] - up[a]));
                        wv[a] = fmaxf_(0.0f, 1.0f - std::fabs(s[a] - vp[a]));
                        ww[a] = fmaxf_(0.0f, 1.0f - std::fabs(s[a] - wp[a]));
                    }
                    const float wgt[3] = {wu[0] * wu[1] * wu[2], wv[0] * wv[1] * wv[2], ww[0] * ww[1] * ww[2]};
                    for (int a = 0; a < 3; ++a) {
                        vsum[a] += wgt[a] * V[a];
                        wsum[a] += wgt[a];
                    }
                }
            }
            for (int a = 0; a < 3; ++a) {
                vs[lane][a] = vsum[a];
                ws[lane][a] = wsum[a];
            }
            cnt[lane] = inside;
        }
        for (int offset = lanes >> 1; offset > 0; offset >>= 1)
            for (int lane = 0; lane < offset; ++lane) {
                for (int a = 0; a < 3; ++a) {
                    vs[lane][a] += vs[lane + offset][a];
                    ws[lane][a] += ws[lane + offset][a];
                }
                cnt[lane] += cnt[lane + offset];
            }
        u[index] = ws[0][0] > 0.0f ? vs[0][0] / ws[0][0] : 0.0f;
        v[index] = ws[0][1] > 0.0f ? vs[0][1] / ws[0][1] : 0.0f;
        w[index] = ws[0][2] > 0.0f ? vs[0][2] / ws[0][2] : 0.0f;
        ff[index] = (float)cnt[0] * inv_ppc;
    }
}

// particles.cl:229-262 grid_to_particle, extended by a FLIP/PIC blend. flip_ratio == 1 is exactly
// the reference (v += I(u) - I(u_old)); otherwise v = a*(v + I(u) - I(u_old)) + (1-a)*I(u).
void orc_grid_to_particle(float* vel, const float* pos, const float* u, const float* v, const float* w,
                          const float* ou, const float* ov, const float* ow, i64 n, float inv_dx, int nx, int ny,
                          int nz, float flip_ratio) {
    const float offs[3][3] = {{1.0f, 0.5f, 0.5f}, {0.5f, 1.0f, 0.5f}, {0.5f, 0.5f, 1.0f}};
    const float* nf[3] = {u, v, w};
    const float* of[3] = {ou, ov, ow};
#pragma omp parallel for schedule(static)
    for (i64 p = 0; p < n; ++p) {
        const float* P = pos + 3 * p;
        float cur[3], chg[3];
        for (int a = 0; a < 3; ++a) {
            int base[3];
            float frac[3];
            staggered_base_fraction(P, inv_dx, offs[a], nx, ny, nz, base, frac);
            cur[a] = sample_field(nf[a], base, frac, ny, nz);
            chg[a] = cur[a] - sample_field(of[a], base, frac, ny, nz);
        }
        for (int a = 0; a < 3; ++a) {
            const float flip = vel[3 * p + a] + chg[a];
            vel[3 * p + a] = flip_ratio == 1.0f ? flip : flip_ratio * flip + (1.0f - flip_ratio) * cur[a];
        }
    }
}

// particles.cl:264-276 advect_particles
void orc_advect_particles(float* pos, const float* vel, i64 n, float dt) {
#pragma omp parallel for schedule(static)
    for (i64 i = 0; i < 3 * n; ++i) pos[i] = pos[i] + dt * vel[i];
}

// ---------------------------------------------------------------------------------------------
// Voxelisation (voxelise_mesh.cl)
// ---------------------------------------------------------------------------------------------

// voxelise_mesh.cl:24 direction = normalize((1, 0.3713907, 0.2178311)), restated as v / sqrt(dot(v,v)).
void orc_voxelise_direction(float out[3]) {
    const float x = 1.0f, y = 0.3713907f, z = 0.2178311f;
    const float len = std::sqrt(x * x + y * y + z * z);
    out[0] = x / len;
    out[1] = y / len;
    out[2] = z / len;
}

// voxelise_mesh.cl:5-22 ray_hit (Moller-Trumbore; det guard 1e-7, t > 1e-6, inclusive u/v bounds).
static inline int ray_hit(const float o[3], const float d[3], const float* A, const float* B, const float* Cv) {
    const float e1[3] = {B[0] - A[0], B[1] - A[1], B[2] - A[2]};
    const float e2[3] = {Cv[0] - A[0], Cv[1] - A[1], Cv[2] - A[2]};
    const float p[3] = {d[1] * e2[2] - d[2] * e2[1], d[2] * e2[0] - d[0] * e2[2], d[0] * e2[1] - d[1] * e2[0]};
    const float det = e1[0] * p[0] + e1[1] * p[1] + e1[2] * p[2];
    if (std::fabs(det) < 1.0e-7f) return 0;
    const float inv = 1.0f / det;
    const float t[3] = {o[0] - A[0], o[1] - A[1], o[2] - A[2]};
    const float uu = (t[0] * p[0] + t[1] * p[1] + t[2] * p[2]) * inv;
    if (uu < 0.0f || uu > 1.0f) return 0;
    const float q[3] = {t[1] * e1[2] - t[2] * e1[1], t[2] * e1[0] - t[0] * e1[2], t[0] * e1[1] - t[1] * e1[0]};
    const float vv = (d[0] * q[0] + d[1] * q[1] + d[2] * q[2]) * inv;
    if (vv < 0.0f || uu + vv > 1.0f) return 0;
    return (e2[0] * q[0] + e2[1] * q[1] + e2[2] * q[2]) * inv > 1.0e-6f;
}

// voxelise_mesh.cl:24-48 voxelise_mesh: interior cells only; odd hit count sets mask=1 (OR, no clear).
void orc_voxelise_mesh(const float* tris, uint8_t* mask, int T, int nx, int ny, int nz, float delta, float ox,
                       float oy, float oz) {
    float dir[3];
    orc_voxelise_direction(dir);
#pragma omp parallel for collapse(2) schedule(dynamic, 1)
    for (int i = 1; i < nx - 1; ++i)
        for (int j = 1; j < ny - 1; ++j)
            for (int k = 1; k < nz - 1; ++k) {
                const float o[3] = {ox + ((float)i + 0.5f) * delta, oy + ((float)j + 0.5f) * delta,
                                    oz + ((float)k + 0.5f) * delta};
                int hits = 0;
                for (int t = 0; t < T; ++t)
                    hits += ray_hit(o, dir, tris + 9 * (i64)t, tris + 9 * (i64)t + 3, tris + 9 * (i64)t + 6);
                if (hits & 1) mask[gidx(i, j, k, ny, nz)] = 1;
            }
}

// ---------------------------------------------------------------------------------------------
// Grid kernels (velocity_update.cl, boundary_conditions.cl, pressure_solve.cl)
// ---------------------------------------------------------------------------------------------

// helper.cl:54-66 laplacian
static inline float laplacian(const float* f, int i, int j, int k, float inv_dx2, int ny, int nz) {
    const float c = f[gidx(i, j, k, ny, nz)];
    const float s = f[gidx(i + 1, j, k, ny, nz)] + f[gidx(i - 1, j, k, ny, nz)] + f[gidx(i, j + 1, k, ny, nz)] +
                    f[gidx(i, j - 1, k, ny, nz)] + f[gidx(i, j, k + 1, ny, nz)] + f[gidx(i, j, k - 1, ny, nz)];
    return (s - 6.0f * c) * inv_dx2;
}

// velocity_update.cl:3-43 update_velocity
void orc_update_velocity(const float* u, const float* v, const float* w, float* ru, float* rv, float* rw,
                         const float* ff, float gx, float gy, float gz, float fx, float fy, float fz, float rho,
                         float nu, float inv_dx2, float dt, int nx, int ny, int nz) {
    const i64 C = (i64)nx * ny * nz;
#pragma omp parallel for schedule(static)
    for (i64 index = 0; index < C; ++index) {
        int i, j, k;
        gcoord(index, ny, nz, i, j, k);
        float r0 = u[index], r1 = v[index], r2 = w[index];
        if (ff[index] > 0.0f) {
            r0 += dt * (gx + fx / rho);
            r1 += dt * (gy + fy / rho);
            r2 += dt * (gz + fz / rho);
        }
        if (interior(i, j, k, nx, ny, nz)) {
            r0 += nu * dt * laplacian(u, i, j, k, inv_dx2, ny, nz);
            r1 += nu * dt * laplacian(v, i, j, k, inv_dx2, ny, nz);
            r2 += nu * dt * laplacian(w, i, j, k, inv_dx2, ny, nz);
        }
        ru[index] = r0;
        rv[index] = r1;
        rw[index] = r2;
    }
}

// boundary_conditions.cl:33-67 grid_domain_bc
void orc_grid_domain_bc(float* u, float* v, float* w, int nx, int ny, int nz) {
    const i64 C = (i64)nx * ny * nz;
    // Ghost cells copy from interior cells whose copied component is never modified by the same
    // launch (the wall flags of a ghost and its interior source agree), so one pass is exact.
#pragma omp parallel for schedule(static)
    for (i64 index = 0; index < C; ++index) {
        int i, j, k;
        gcoord(index, ny, nz, i, j, k);
        const bool ghost = !interior(i, j, k, nx, ny, nz);
        const bool wu = i == 0 || i >= nx - 2, wv = j == 0 || j >= ny - 2, ww = k == 0 || k >= nz - 2;
        if (!ghost && !wu && !wv && !ww) continue;
        if (ghost) {
            const i64 src = gidx(clampi(i, 1, nx - 2), clampi(j, 1, ny - 2), clampi(k, 1, nz - 2), ny, nz);
            u[index] = wu ? 0.0f : u[src];
            v[index] = wv ? 0.0f : v[src];
            w[index] = ww ? 0.0f : w[src];
            continue;
        }
        if (wu) u[index] = 0.0f;
        if (wv) v[index] = 0.0f;
        if (ww) w[index] = 0.0f;
    }
}

// boundary_conditions.cl:99-119 grid_obstacle_bc
void orc_grid_obstacle_bc(float* u, float* v, float* w, float* ff, const uint8_t* obs, int nx, int ny, int nz) {
    const i64 C = (i64)nx * ny * nz;
#pragma omp parallel for schedule(static)
    for (i64 index = 0; index < C; ++index) {
        int i, j, k;
        gcoord(index, ny, nz, i, j, k);
        if (obs[index]) ff[index] = 0.0f;
        const bool xs = obs[index] || (i + 1 < nx && obs[gidx(i + 1, j, k, ny, nz)]);
        const bool ys = obs[index] || (j + 1 < ny && obs[gidx(i, j + 1, k, ny, nz)]);
        const bool zs = obs[index] || (k + 1 < nz && obs[gidx(i, j, k + 1, ny, nz)]);
        if (xs) u[index] = 0.0f;
        if (ys) v[index] = 0.0f;
        if (zs) w[index] = 0.0f;
    }
}

// boundary_conditions.cl:121-173 extrapolate_obstacle_velocity (reads only non-obstacle cells,
// writes only obstacle cells, so a single pass is race-free).
void orc_extrapolate_obstacle_velocity(float* u, float* v, float* w, const uint8_t* obs, int nx, int ny, int nz) {
    const i64 C = (i64)nx * ny * nz;
#pragma omp parallel for schedule(static)
    for (i64 index = 0; index < C; ++index) {
        if (!obs[index]) continue;
        int i, j, k;
        gcoord(index, ny, nz, i, j, k);
        float t0 = 0.0f, t1 = 0.0f, t2 = 0.0f;
        int n = 0;
        int ax = 0, ay = 0, az = 0;
        auto acc = [&](int a, int b, int c, int& axis) {
            const i64 q = gidx(a, b, c, ny, nz);
            if (!obs[q]) {
                t0 += u[q];
                t1 += v[q];
                t2 += w[q];
                n += 1;
                axis = 1;
            }
        };
        if (i > 0) acc(i - 1, j, k, ax);
        if (i + 1 < nx) acc(i + 1, j, k, ax);
        if (j > 0) acc(i, j - 1, k, ay);
        if (j + 1 < ny) acc(i, j + 1, k, ay);
        if (k > 0) acc(i, j, k - 1, az);
        if (k + 1 < nz) acc(i, j, k + 1, az);
        if (n == 0) continue;
        const float fn = (float)n;
        t0 /= fn;
        t1 /= fn;
        t2 /= fn;
        u[index] = ax ? 0.0f : t0;
        v[index] = ay ? 0.0f : t1;
        w[index] = az ? 0.0f : t2;
    }
}

// boundary_conditions.cl:69-97 particle_domain_bc
void orc_particle_domain_bc(float* pos, float* vel, i64 n, float lower, float ux, float uy, float uz) {
    const float up[3] = {ux, uy, uz};
#pragma omp parallel for schedule(static)
    for (i64 p = 0; p < n; ++p) {
        float* P = pos + 3 * p;
        float* V = vel + 3 * p;
        bool hit = false;
        float q[3];
        for (int a = 0; a < 3; ++a) {
            const bool lo = P[a] < lower, hi = P[a] > up[a];
            float x = P[a];
            if (lo) x = 2.0f * lower - P[a];
            if (hi) x = 2.0f * up[a] - x;
            x = x < lower ? lower : (x > up[a] ? up[a] : x);
            q[a] = x;
            hit = hit || lo || hi;
            if (lo || hi) V[a] = 0.0f;
        }
        for (int a = 0; a < 3; ++a) P[a] = q[a];
        (void)hit;
    }
}

// boundary_conditions.cl:175-264 particle_obstacle_bc
void orc_particle_obstacle_bc(float* pos, const float* prev, float* vel, const uint8_t* obs, i64 n, float inv_dx,
                              int nx, int ny, int nz) {
#pragma omp parallel for schedule(static)
    for (i64 p = 0; p < n; ++p) {
        float* P = pos + 3 * p;
        const float* Q = prev + 3 * p;
        float* V = vel + 3 * p;
        const int c0 = clampi((int)(P[0] * inv_dx), 0, nx - 1);
        const int c1 = clampi((int)(P[1] * inv_dx), 0, ny - 1);
        const int c2 = clampi((int)(P[2] * inv_dx), 0, nz - 1);
        if (!obs[gidx(c0, c1, c2, ny, nz)]) continue;
        const int p0 = clampi((int)(Q[0] * inv_dx), 0, nx - 1);
        const int p1 = clampi((int)(Q[1] * inv_dx), 0, ny - 1);
        const int p2 = clampi((int)(Q[2] * inv_dx), 0, nz - 1);
        float nrm[3] = {0.0f, 0.0f, 0.0f};
        if ((p0 != c0 || p1 != c1 || p2 != c2) && !obs[gidx(p0, p1, p2, ny, nz)]) {
            nrm[0] = (float)(p0 - c0);
            nrm[1] = (float)(p1 - c1);
            nrm[2] = (float)(p2 - c2);
        } else {
            if (c0 > 0 && !obs[gidx(c0 - 1, c1, c2, ny, nz)]) nrm[0] -= 1.0f;
            if (c0 + 1 < nx && !obs[gidx(c0 + 1, c1, c2, ny, nz)]) nrm[0] += 1.0f;
            if (c1 > 0 && !obs[gidx(c0, c1 - 1, c2, ny, nz)]) nrm[1] -= 1.0f;
            if (c1 + 1 < ny && !obs[gidx(c0, c1 + 1, c2, ny, nz)]) nrm[1] += 1.0f;
            if (c2 > 0 && !obs[gidx(c0, c1, c2 - 1, ny, nz)]) nrm[2] -= 1.0f;
            if (c2 + 1 < nz && !obs[gidx(c0, c1, c2 + 1, ny, nz)]) nrm[2] += 1.0f;
        }
        const float len = std::sqrt(nrm[0] * nrm[0] + nrm[1] * nrm[1] + nrm[2] * nrm[2]);
        if (len > 0.0f) {
            nrm[0] /= len;
            nrm[1] /= len;
            nrm[2] /= len;
        } else {
            const float fb[3] = {Q[0] - P[0], Q[1] - P[1], Q[2] - P[2]};
            const float fl = std::sqrt(fb[0] * fb[0] + fb[1] * fb[1] + fb[2] * fb[2]);
            if (fl > 0.0f) {
                nrm[0] = fb[0] / fl;
                nrm[1] = fb[1] / fl;
                nrm[2] = fb[2] / fl;
            } else {
                nrm[0] = 0.0f;
                nrm[1] = 0.0f;
                nrm[2] = 1.0f;
            }
        }
        const float vn = V[0] * nrm[0] + V[1] * nrm[1] + V[2] * nrm[2];
        if (vn < 0.0f) {
            V[0] -= vn * nrm[0];
            V[1] -= vn * nrm[1];
            V[2] -= vn * nrm[2];
        }
        const float dx = 1.0f / inv_dx;
        const int cc[3] = {c0, c1, c2};
        float cor[3] = {P[0], P[1], P[2]};
        for (int a = 0; a < 3; ++a) {
            if (nrm[a] < 0.0f)
                cor[a] = 2.0f * ((float)cc[a] * dx) - P[a];
            else if (nrm[a] > 0.0f)
                cor[a] = 2.0f * ((float)(cc[a] + 1) * dx) - P[a];
        }
        const int k0 = clampi((int)(cor[0] * inv_dx), 0, nx - 1);
        const int k1 = clampi((int)(cor[1] * inv_dx), 0, ny - 1);
        const int k2 = clampi((int)(cor[2] * inv_dx), 0, nz - 1);
        if (obs[gidx(k0, k1, k2, ny, nz)]) {
            cor[0] = Q[0];
            cor[1] = Q[1];
            cor[2] = Q[2];
        }
        P[0] = cor[0];
        P[1] = cor[1];
        P[2] = cor[2];
    }
}

// ---- moving colliders (no counterpart in the reference, whose colliders are static) ------------
// A rigid motion m[9] = (V, W, C) in grid-local coordinates: velocity, angular velocity (rad/s) and
// pivot. The solid's velocity at x is V + W x (x - C), evaluated in this order (separately rounded).
static inline void rigid_velocity(const float* m, float x, float y, float z, float out[3]) {
    const float rx = x - m[6], ry = y - m[7], rz = z - m[8];
    out[0] = m[0] + (m[4] * rz - m[5] * ry);
    out[1] = m[1] + (m[5] * rx - m[3] * rz);
    out[2] = m[2] + (m[3] * ry - m[4] * rx);
}

// grid_obstacle_bc with a moving solid: a solid face takes the solid's velocity component at the face
// centre (u face of cell (i, j, k) at ((i+1) dx, (j+0.5) dx, (k+0.5) dx), v and w likewise) instead of 0.
void orc_grid_obstacle_bc_moving(float* u, float* v, float* w, float* ff, const uint8_t* obs, int nx, int ny, int nz,
                                 const float* m, float dx) {
    const i64 C = (i64)nx * ny * nz;
#pragma omp parallel for schedule(static)
    for (i64 index = 0; index < C; ++index) {
        int i, j, k;
        gcoord(index, ny, nz, i, j, k);
        if (obs[index]) ff[index] = 0.0f;
        const bool xs = obs[index] || (i + 1 < nx && obs[gidx(i + 1, j, k, ny, nz)]);
        const bool ys = obs[index] || (j + 1 < ny && obs[gidx(i, j + 1, k, ny, nz)]);
        const bool zs = obs[index] || (k + 1 < nz && obs[gidx(i, j, k + 1, ny, nz)]);
        const float fi = (float)i, fj = (float)j, fk = (float)k;
        float sv[3];
        if (xs) {
            rigid_velocity(m, (fi + 1.0f) * dx, (fj + 0.5f) * dx, (fk + 0.5f) * dx, sv);
            u[index] = sv[0];
        }
        if (ys) {
            rigid_velocity(m, (fi + 0.5f) * dx, (fj + 1.0f) * dx, (fk + 0.5f) * dx, sv);
            v[index] = sv[1];
        }
        if (zs) {
            rigid_velocity(m, (fi + 0.5f) * dx, (fj + 0.5f) * dx, (fk + 1.0f) * dx, sv);
            w[index] = sv[2];
        }
    }
}

// extrapolate_obstacle_velocity with a moving solid: a solid cell next to fluid keeps the fluid's
// averaged tangential velocity and takes the solid's normal component at its face centre.
void orc_extrapolate_obstacle_velocity_moving(float* u, float* v, float* w, const uint8_t* obs, int nx, int ny,
                                              int nz, const float* m, float dx) {
    const i64 C = (i64)nx * ny * nz;
#pragma omp parallel for schedule(static)
    for (i64 index = 0; index < C; ++index) {
        if (!obs[index]) continue;
        int i, j, k;
        gcoord(index, ny, nz, i, j, k);
        float t0 = 0.0f, t1 = 0.0f, t2 = 0.0f;
        int n = 0;
        int ax = 0, ay = 0, az = 0;
        auto acc = [&](int a, int b, int c, int& axis) {
            const i64 q = gidx(a, b, c, ny, nz);
            if (!obs[q]) {
                t0 += u[q];
                t1 += v[q];
                t2 += w[q];
                n += 1;
                axis = 1;
            }
        };
        if (i > 0) acc(i - 1, j, k, ax);
        if (i + 1 < nx) acc(i + 1, j, k, ax);
        if (j > 0) acc(i, j - 1, k, ay);
        if (j + 1 < ny) acc(i, j + 1, k, ay);
        if (k > 0) acc(i, j, k - 1, az);
        if (k + 1 < nz) acc(i, j, k + 1, az);
        if (n == 0) continue;
        const float fn = (float)n;
        t0 /= fn;
        t1 /= fn;
        t2 /= fn;
        const float fi = (float)i, fj = (float)j, fk = (float)k;
        float sv[3];
        if (ax) rigid_velocity(m, (fi + 1.0f) * dx, (fj + 0.5f) * dx, (fk + 0.5f) * dx, sv);
        u[index] = ax ? sv[0] : t0;
        if (ay) rigid_velocity(m, (fi + 0.5f) * dx, (fj + 1.0f) * dx, (fk + 0.5f) * dx, sv);
        v[index] = ay ? sv[1] : t1;
        if (az) rigid_velocity(m, (fi + 0.5f) * dx, (fj + 0.5f) * dx, (fk + 1.0f) * dx, sv);
        w[index] = az ? sv[2] : t2;
    }
}

// particle_obstacle_bc with a moving solid: the same normal and push-out, but only the particle's
// velocity relative to the solid (at the particle's position) loses its inward normal component.
void orc_particle_obstacle_bc_moving(float* pos, const float* prev, float* vel, const uint8_t* obs, i64 n,
                                     float inv_dx, int nx, int ny, int nz, const float* m) {
#pragma omp parallel for schedule(static)
    for (i64 p = 0; p < n; ++p) {
        float* P = pos + 3 * p;
        const float* Q = prev + 3 * p;
        float* V = vel + 3 * p;
        const int c0 = clampi((int)(P[0] * inv_dx), 0, nx - 1);
        const int c1 = clampi((int)(P[1] * inv_dx), 0, ny - 1);
        const int c2 = clampi((int)(P[2] * inv_dx), 0, nz - 1);
        if (!obs[gidx(c0, c1, c2, ny, nz)]) continue;
        const int p0 = clampi((int)(Q[0] * inv_dx), 0, nx - 1);
        const int p1 = clampi((int)(Q[1] * inv_dx), 0, ny - 1);
        const int p2 = clampi((int)(Q[2] * inv_dx), 0, nz - 1);
        float nrm[3] = {0.0f, 0.0f, 0.0f};
        if ((p0 != c0 || p1 != c1 || p2 != c2) && !obs[gidx(p0, p1, p2, ny, nz)]) {
            nrm[0] = (float)(p0 - c0);
            nrm[1] = (float)(p1 - c1);
            nrm[2] = (float)(p2 - c2);
        } else {
            if (c0 > 0 && !obs[gidx(c0 - 1, c1, c2, ny, nz)]) nrm[0] -= 1.0f;
            if (c0 + 1 < nx && !obs[gidx(c0 + 1, c1, c2, ny, nz)]) nrm[0] += 1.0f;
            if (c1 > 0 && !obs[gidx(c0, c1 - 1, c2, ny, nz)]) nrm[1] -= 1.0f;
            if (c1 + 1 < ny && !obs[gidx(c0, c1 + 1, c2, ny, nz)]) nrm[1] += 1.0f;
            if (c2 > 0 && !obs[gidx(c0, c1, c2 - 1, ny, nz)]) nrm[2] -= 1.0f;
            if (c2 + 1 < nz && !obs[gidx(c0, c1, c2 + 1, ny, nz)]) nrm[2] += 1.0f;
        }
        const float len = std::sqrt(nrm[0] * nrm[0] + nrm[1] * nrm[1] + nrm[2] * nrm[2]);
        if (len > 0.0f) {
            nrm[0] /= len;
            nrm[1] /= len;
            nrm[2] /= len;
        } else {
            const float fb[3] = {Q[0] - P[0], Q[1] - P[1], Q[2] - P[2]};
            const float fl = std::sqrt(fb[0] * fb[0] + fb[1] * fb[1] + fb[2] * fb[2]);
            if (fl > 0.0f) {
                nrm[0] = fb[0] / fl;
                nrm[1] = fb[1] / fl;
                nrm[2] = fb[2] / fl;
            } else {
                nrm[0] = 0.0f;
                nrm[1] = 0.0f;
                nrm[2] = 1.0f;
            }
        }
        float sv[3];
        rigid_velocity(m, P[0], P[1], P[2], sv);
        const float r0 = V[0] - sv[0], r1 = V[1] - sv[1], r2 = V[2] - sv[2];
        const float vn = r0 * nrm[0] + r1 * nrm[1] + r2 * nrm[2];
        if (vn < 0.0f) {
            V[0] -= vn * nrm[0];
            V[1] -= vn * nrm[1];
            V[2] -= vn * nrm[2];
        }
        const float dx = 1.0f / inv_dx;
        const int cc[3] = {c0, c1, c2};
        float cor[3] = {P[0], P[1], P[2]};
        for (int a = 0; a < 3; ++a) {
            if (nrm[a] < 0.0f)
                cor[a] = 2.0f * ((float)cc[a] * dx) - P[a];
            else if (nrm[a] > 0.0f)
                cor[a] = 2.0f * ((float)(cc[a] + 1) * dx) - P[a];
        }
        const int k0 = clampi((int)(cor[0] * inv_dx), 0, nx - 1);
        const int k1 = clampi((int)(cor[1] * inv_dx), 0, ny - 1);
        const int k2 = clampi((int)(cor[2] * inv_dx), 0, nz - 1);
        if (obs[gidx(k0, k1, k2, ny, nz)]) {
            cor[0] = Q[0];
            cor[1] = Q[1];
            cor[2] = Q[2];
        }
        P[0] = cor[0];
        P[1] = cor[1];
        P[2] = cor[2];
    }
}

// pressure_solve.cl:3-24 pressure_rhs
void orc_pressure_rhs(const float* u, const float* v, const float* w, const float* ff, float* rhs, float rho_over_dt,
                      float inv_dx, int nx, int ny, int nz) {
    const i64 C = (i64)nx * ny * nz;
#pragma omp parallel for schedule(static)
    for (i64 index = 0; index < C; ++index) {
        int i, j, k;
        gcoord(index, ny, nz, i, j, k);
        if (!interior(i, j, k, nx, ny, nz) || ff[index] <= 0.0f) {
            rhs[index] = 0.0f;
            continue;
        }
        const float du = u[index] - u[gidx(i - 1, j, k, ny, nz)];
        const float dv = v[index] - v[gidx(i, j - 1, k, ny, nz)];
        const float dw = w[index] - w[gidx(i, j, k - 1, ny, nz)];
        rhs[index] = rho_over_dt * ((du + dv + dw) * inv_dx);
    }
}

// pressure_solve.cl:26-47 pressure_correction (helper.cl:25-37 gradient)
void orc_pressure_correction(float* u, float* v, float* w, const float* p, float dt_over_rho, float inv_dx, int nx,
                             int ny, int nz) {
    const i64 C = (i64)nx * ny * nz;
#pragma omp parallel for schedule(static)
    for (i64 index = 0; index < C; ++index) {
        int i, j, k;
        gcoord(index, ny, nz, i, j, k);
        if (!interior(i, j, k, nx, ny, nz)) continue;
        const float c = p[index];
        const float gx = (p[gidx(i + 1, j, k, ny, nz)] - c) * inv_dx;
        const float gy = (p[gidx(i, j + 1, k, ny, nz)] - c) * inv_dx;
        const float gz = (p[gidx(i, j, k + 1, ny, nz)] - c) * inv_dx;
        u[index] -= dt_over_rho * gx;
        v[index] -= dt_over_rho * gy;
        w[index] -= dt_over_rho * gz;
    }
}

// boundary_conditions.cl:18-31 neumann_domain_bc (ghosts read interior cells only)
void orc_neumann_domain_bc(float* p, int nx, int ny, int nz) {
    const i64 C = (i64)nx * ny * nz;
#pragma omp parallel for schedule(static)
    for (i64 index = 0; index < C; ++index) {
        int i, j, k;
        gcoord(index, ny, nz, i, j, k);
        if (interior(i, j, k, nx, ny, nz)) continue;
        p[index] = p[gidx(clampi(i, 1, nx - 2), clampi(j, 1, ny - 2), clampi(k, 1, nz - 2), ny, nz)];
    }
}

}  // extern "C"

// ---------------------------------------------------------------------------------------------
// Multigrid (multigrid.cl, multigrid.py), templated so the same code gives the FP64 oracle solve
// ---------------------------------------------------------------------------------------------
namespace {

template <typename T>
inline T domain_diagonal(int i, int j, int k, int nx, int ny, int nz) {  // multigrid.cl:3-5
    return (T)6 - (T)(i == 1) - (T)(i == nx - 2) - (T)(j == 1) - (T)(j == ny - 2) - (T)(k == 1) - (T)(k == nz - 2);
}

template <typename T>
inline T wsum(const T* p, const T* wx, const T* wy, const T* wz, int i, int j, int k, int ny, int nz) {
    const i64 c = gidx(i, j, k, ny, nz);  // multigrid.cl:7-23 weighted_neighbor_sum
    return wx[c] * p[gidx(i + 1, j, k, ny, nz)] + wx[gidx(i - 1, j, k, ny, nz)] * p[gidx(i - 1, j, k, ny, nz)] +
           wy[c] * p[gidx(i, j + 1, k, ny, nz)] + wy[gidx(i, j - 1, k, ny, nz)] * p[gidx(i, j - 1, k, ny, nz)] +
           wz[c] * p[gidx(i, j, k + 1, ny, nz)] + wz[gidx(i, j, k - 1, ny, nz)] * p[gidx(i, j, k - 1, ny, nz)];
}

template <typename T>  // multigrid.cl:25-61 apply_operator / residual
inline T residual_at(const T* p, const T* b, const T* mask, const T* d, const T* wx, const T* wy, const T* wz,
                     T inv_delta2, int i, int j, int k, int nx, int ny, int nz) {
    const i64 c = gidx(i, j, k, ny, nz);
    T ap = 0;
    if (interior(i, j, k, nx, ny, nz) && !(mask[c] <= (T)0))
        ap = (wsum(p, wx, wy, wz, i, j, k, ny, nz) - d[c] * p[c]) * inv_delta2;
    return b[c] - ap;
}

template <typename T>  // multigrid.cl:63-88 build_finest_operator
void build_finest_operator(const T* mask, T* d, T* wx, T* wy, T* wz, int nx, int ny, int nz) {
    const i64 C = (i64)nx * ny * nz;
#pragma omp parallel for schedule(static)
    for (i64 index = 0; index < C; ++index) {
        d[index] = 0;
        wx[index] = 0;
        wy[index] = 0;
        wz[index] = 0;
        int i, j, k;
        gcoord(index, ny, nz, i, j, k);
        if (!interior(i, j, k, nx, ny, nz) || mask[index] <= (T)0) continue;
        d[index] = domain_diagonal<T>(i, j, k, nx, ny, nz);
        if (i < nx - 2) wx[index] = mask[gidx(i + 1, j, k, ny, nz)] > (T)0 ? (T)1 : (T)0;
        if (j < ny - 2) wy[index] = mask[gidx(i, j + 1, k, ny, nz)] > (T)0 ? (T)1 : (T)0;
        if (k < nz - 2) wz[index] = mask[gidx(i, j, k + 1, ny, nz)] > (T)0 ? (T)1 : (T)0;
    }
}

template <typename T>  // multigrid.cl:90-180 restrict_residual
void restrict_residual(const T* fp, const T* fb, const T* fm, const T* fd, const T* fwx, const T* fwy, const T* fwz,
                       T* cp, T* cb, T* cm, T* cd, T* cwx, T* cwy, T* cwz, T delta, int fnx, int fny, int fnz,
                       int cnx, int cny, int cnz) {
    const i64 C = (i64)cnx * cny * cnz;
    const T inv_delta2 = (T)1 / (delta * delta);
#pragma omp parallel for schedule(static)
    for (i64 ci = 0; ci < C; ++ci) {
        cp[ci] = 0;
        cb[ci] = 0;
        cm[ci] = 0;
        cd[ci] = 0;
        cwx[ci] = 0;
        cwy[ci] = 0;
        cwz[ci] = 0;
        int I, J, K;
        gcoord(ci, cny, cnz, I, J, K);
        if (!interior(I, J, K, cnx, cny, cnz)) continue;
        const int si = 1 + 2 * (I - 1), sj = 1 + 2 * (J - 1), sk = 1 + 2 * (K - 1);
        T rhs = 0, dsum = 0, cx = 0, cy = 0, cz = 0;
        int active = 0;
        for (int di = 0; di < 2; ++di)
            for (int dj = 0; dj < 2; ++dj)
                for (int dk = 0; dk < 2; ++dk) {
                    const int i = si + di, j = sj + dj, k = sk + dk;
                    if (!interior(i, j, k, fnx, fny, fnz)) continue;
                    const i64 f = gidx(i, j, k, fny, fnz);
                    if (fm[f] <= (T)0) continue;
                    ++active;
                    rhs += residual_at(fp, fb, fm, fd, fwx, fwy, fwz, inv_delta2, i, j, k, fnx, fny, fnz);
                    dsum += fd[f];
                    const T wx = fwx[f], wy = fwy[f], wz = fwz[f];
                    if (wx > (T)0) {
                        if (di == 0) dsum -= (T)2 * wx; else cx += wx;
                    }
                    if (wy > (T)0) {
                        if (dj == 0) dsum -= (T)2 * wy; else cy += wy;
                    }
                    if (wz > (T)0) {
                        if (dk == 0) dsum -= (T)2 * wz; else cz += wz;
                    }
                }
        if (active > 0) {
            cb[ci] = rhs;
            cm[ci] = 1;
            cd[ci] = dsum;
            cwx[ci] = cx;
            cwy[ci] = cy;
            cwz[ci] = cz;
        }
    }
}

// multigrid.cl:182-201 prolongate. w multiplies the prolonged correction (no counterpart in the
// reference, whose prolongation is w = 1: 1 * e = e, so w = 1 is the reference bit for bit).
template <typename T>
void prolongate(const T* ce, T* fp, const T* fm, int cnx, int cny, int cnz, int fnx, int fny, int fnz, T w = 1) {
    const i64 C = (i64)fnx * fny * fnz;
#pragma omp parallel for schedule(static)
    for (i64 f = 0; f < C; ++f) {
        int i, j, k;
        gcoord(f, fny, fnz, i, j, k);
        if (!interior(i, j, k, fnx, fny, fnz) || fm[f] <= (T)0) continue;
        const int I = std::min((i - 1) / 2 + 1, cnx - 2);
        const int J = std::min((j - 1) / 2 + 1, cny - 2);
        const int K = std::min((k - 1) / 2 + 1, cnz - 2);
        fp[f] += w * ce[gidx(I, J, K, cny, cnz)];
    }
}

// multigrid.cl:203-230 rbgs_step (one colour). The reference zeroes p at mask <= 0 cells in the same
// launch that updates the colour; a cell being updated can read such a neighbour before or after it
// is zeroed, but every such neighbour has weight 0, so only the sign of a zero product can differ.
// Restated deterministically as a zeroing pass followed by the colour update.
template <typename T>
void rbgs_step(T* p, const T* b, const T* m, const T* d, const T* wx, const T* wy, const T* wz, T delta, int parity,
               int nx, int ny, int nz) {
    const i64 C = (i64)nx * ny * nz;
    const T d2 = delta * delta;
#pragma omp parallel for schedule(static)
    for (i64 index = 0; index < C; ++index)
        if (m[index] <= (T)0) p[index] = 0;
#pragma omp parallel for schedule(static)
    for (i64 index = 0; index < C; ++index) {
        int i, j, k;
        gcoord(index, ny, nz, i, j, k);
        if (!interior(i, j, k, nx, ny, nz) || m[index] <= (T)0 || ((i + j + k) & 1) != parity) continue;
        const T dd = d[index];
        if (dd > (T)0) p[index] = (wsum(p, wx, wy, wz, i, j, k, ny, nz) - d2 * b[index]) / dd;
    }
}

template <typename T>  // multigrid.cl:232-264 coarse_smooth
void coarse_smooth(T* p, const T* b, const T* m, const T* d, const T* wx, const T* wy, const T* wz, T delta,
                   int iterations, int nx, int ny, int nz) {
    const i64 C = (i64)nx * ny * nz;
    const T d2 = delta * delta;
    for (int it = 0; it < iterations; ++it)
        for (int parity = 0; parity < 2; ++parity)
            for (i64 index = 0; index < C; ++index) {
                int i, j, k;
                gcoord(index, ny, nz, i, j, k);
                if (!interior(i, j, k, nx, ny, nz) || m[index] <= (T)0 || ((i + j + k) & 1) != parity) continue;
                const T dd = d[index];
                if (dd > (T)0) p[index] = (wsum(p, wx, wy, wz, i, j, k, ny, nz) - d2 * b[index]) / dd;
            }
}

template <typename T>
struct Levels {
    T** p;
    T** b;
    T** m;
    T** d;
    T** wx;
    T** wy;
    T** wz;
    const int* shape;  // 3 ints per level
    int count;         // number of levels including level 0
};

// multigrid.py:53-187 w_cycle (recursive). Level 0 is the fine grid; level count-1 is the coarsest.
// single_from > 0 (no counterpart in the reference): levels from single_from on are visited once per
// visit of the level above instead of twice (the solver's clb_mg_set_option 4).
template <typename T>
void w_cycle(const Levels<T>& L, int level, T delta, int pre, int post, int coarse_iters, int single_from = 0,
             T prolong_scale = 1, int pre_coarse = -1, int post_coarse = -1) {
    const int* s = L.shape + 3 * level;
    // pre_coarse / post_coarse >= 0 (no counterpart in the reference): the smoothing counts of levels >= 1,
    // the coarsest level's solve included (pre + coarse_iters iterations)
    if (level > 0 && pre_coarse >= 0) pre = pre_coarse;
    if (level > 0 && post_coarse >= 0) post = post_coarse;
    if (level == L.count - 1) {
        coarse_smooth<T>(L.p[level], L.b[level], L.m[level], L.d[level], L.wx[level], L.wy[level], L.wz[level], delta,
                         pre + coarse_iters, s[0], s[1], s[2]);
        return;
    }
    for (int it = 0; it < pre; ++it)
        for (int parity = 0; parity < 2; ++parity)
            rbgs_step<T>(L.p[level], L.b[level], L.m[level], L.d[level], L.wx[level], L.wy[level], L.wz[level], delta,
                         parity, s[0], s[1], s[2]);
    const int c = level + 1;
    const int* cs = L.shape + 3 * c;
    restrict_residual<T>(L.p[level], L.b[level], L.m[level], L.d[level], L.wx[level], L.wy[level], L.wz[level], L.p[c],
                         L.b[c], L.m[c], L.d[c], L.wx[c], L.wy[c], L.wz[c], delta, s[0], s[1], s[2], cs[0], cs[1],
                         cs[2]);
    const int visits = single_from > 0 && c >= single_from ? 1 : 2;
    for (int v = 0; v < visits; ++v)
        w_cycle<T>(L, c, delta, pre, post, coarse_iters, single_from, prolong_scale, pre_coarse, post_coarse);
    prolongate<T>(L.p[c], L.p[level], L.m[level], cs[0], cs[1], cs[2], s[0], s[1], s[2], prolong_scale);
    for (int it = 0; it < post; ++it)
        for (int parity = 0; parity < 2; ++parity)
            rbgs_step<T>(L.p[level], L.b[level], L.m[level], L.d[level], L.wx[level], L.wy[level], L.wz[level], delta,
                         parity, s[0], s[1], s[2]);
}

// FP64 residual norm over interior fluid cells of the finest level: returns (sum r^2, sum b^2).
template <typename T>
void residual_norms(const T* p, const T* b, const T* m, const T* d, const T* wx, const T* wy, const T* wz, T delta,
                    int nx, int ny, int nz, double* rr, double* bb) {
    const i64 C = (i64)nx * ny * nz;
    const T inv_delta2 = (T)1 / (delta * delta);
    double sr = 0.0, sb = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : sr, sb)
    for (i64 index = 0; index < C; ++index) {
        int i, j, k;
        gcoord(index, ny, nz, i, j, k);
        if (!interior(i, j, k, nx, ny, nz) || m[index] <= (T)0) continue;
        const double r = (double)residual_at(p, b, m, d, wx, wy, wz, inv_delta2, i, j, k, nx, ny, nz);
        sr += r * r;
        sb += (double)b[index] * (double)b[index];
    }
    *rr = sr;
    *bb = sb;
}

}  // namespace

extern "C" {

void orc_build_finest_operator_f32(const float* m, float* d, float* wx, float* wy, float* wz, int nx, int ny, int nz) {
    build_finest_operator<float>(m, d, wx, wy, wz, nx, ny, nz);
}
void orc_build_finest_operator_f64(const double* m, double* d, double* wx, double* wy, double* wz, int nx, int ny,
                                   int nz) {
    build_finest_operator<double>(m, d, wx, wy, wz, nx, ny, nz);
}
void orc_restrict_residual_f32(const float* fp, const float* fb, const float* fm, const float* fd, const float* fwx,
                               const float* fwy, const float* fwz, float* cp, float* cb, float* cm, float* cd,
                               float* cwx, float* cwy, float* cwz, float delta, int fnx, int fny, int fnz, int cnx,
                               int cny, int cnz) {
    restrict_residual<float>(fp, fb, fm, fd, fwx, fwy, fwz, cp, cb, cm, cd, cwx, cwy, cwz, delta, fnx, fny, fnz, cnx,
                             cny, cnz);
}
void orc_prolongate_f32(const float* ce, float* fp, const float* fm, int cnx, int cny, int cnz, int fnx, int fny,
                        int fnz) {
    prolongate<float>(ce, fp, fm, cnx, cny, cnz, fnx, fny, fnz);
}
void orc_rbgs_step_f32(float* p, const float* b, const float* m, const float* d, const float* wx, const float* wy,
                       const float* wz, float delta, int parity, int nx, int ny, int nz) {
    rbgs_step<float>(p, b, m, d, wx, wy, wz, delta, parity, nx, ny, nz);
}
void orc_coarse_smooth_f32(float* p, const float* b, const float* m, const float* d, const float* wx, const float* wy,
                           const float* wz, float delta, int iterations, int nx, int ny, int nz) {
    coarse_smooth<float>(p, b, m, d, wx, wy, wz, delta, iterations, nx, ny, nz);
}

// W-cycle over a level list whose arrays are given as pointer tables (level 0 = finest).
void orc_w_cycle_f32(float** p, float** b, float** m, float** d, float** wx, float** wy, float** wz, const int* shapes,
                     int levels, float delta, int pre, int post, int coarse_iters, int single_from,
                     float prolong_scale, int pre_coarse, int post_coarse) {
    Levels<float> L{p, b, m, d, wx, wy, wz, shapes, levels};
    w_cycle<float>(L, 0, delta, pre, post, coarse_iters, single_from, prolong_scale, pre_coarse, post_coarse);
}
void orc_w_cycle_f64(double** p, double** b, double** m, double** d, double** wx, double** wy, double** wz,
                     const int* shapes, int levels, double delta, int pre, int post, int coarse_iters, int single_from,
                     double prolong_scale, int pre_coarse, int post_coarse) {
    Levels<double> L{p, b, m, d, wx, wy, wz, shapes, levels};
    w_cycle<double>(L, 0, delta, pre, post, coarse_iters, single_from, prolong_scale, pre_coarse, post_coarse);
}
void orc_residual_norms_f32(const float* p, const float* b, const float* m, const float* d, const float* wx,
                            const float* wy, const float* wz, float delta, int nx, int ny, int nz, double* rr,
                            double* bb) {
    residual_norms<float>(p, b, m, d, wx, wy, wz, delta, nx, ny, nz, rr, bb);
}
void orc_residual_norms_f64(const double* p, const double* b, const double* m, const double* d, const double* wx,
                            const double* wy, const double* wz, double delta, int nx, int ny, int nz, double* rr,
                            double* bb) {
    residual_norms<double>(p, b, m, d, wx, wy, wz, delta, nx, ny, nz, rr, bb);
}
// One flexible-CG update of the tolerance-mode iteration (oracle.fcg_solve), in FP64 with OpenMP:
// z = the W-cycle correction e at interior fluid cells (mask > 0), 0 elsewhere; with `flexible`
// the four dot products of Notay's truncated flexible CG (A z . d, A z . z, z . r32, d . r32), the
// scalars beta, d.Ad (*dad, carried between calls, 0 = no direction yet) and alpha, the new float32
// direction d = z + beta d and x += alpha d; without it x += z. Then r = b - A x (FP64), r32 = r
// rounded to float32 and *rr = sum r^2. A is the FP64 finest operator (d, wx, wy, wz).
void orc_fcg_update(const float* e, float* dir, double* x, double* r, float* r32, const double* b, const float* m,
                    const double* dg, const double* wx, const double* wy, const double* wz, double dx, int nx, int ny,
                    int nz, int flexible, double* dad, double* rr) {
    const i64 C = (i64)nx * ny * nz, syz = (i64)ny * nz;
    const double inv = 1.0 / (dx * dx);
    auto fluid = [&](i64 c, int i, int j, int k) { return interior(i, j, k, nx, ny, nz) && m[c] > 0.0f; };
    auto zval = [&](i64 c) {
        int i, j, k;
        gcoord(c, ny, nz, i, j, k);
        return fluid(c, i, j, k) ? (double)e[c] : 0.0;
    };
    auto apply = [&](auto&& val, i64 c) {
        const double ws = wx[c] * val(c + syz) + wx[c - syz] * val(c - syz) + wy[c] * val(c + nz) +
                          wy[c - nz] * val(c - nz) + wz[c] * val(c + 1) + wz[c - 1] * val(c - 1);
        return (ws - dg[c] * val(c)) * inv;
    };
    if (flexible) {
        double sx = 0.0, sy = 0.0, sz = 0.0, sw = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : sx, sy, sz, sw)
        for (i64 c = 0; c < C; ++c) {
            int i, j, k;
            gcoord(c, ny, nz, i, j, k);
            if (!fluid(c, i, j, k)) continue;
            const double z = (double)e[c];
            const double az = apply(zval, c);
            sx += az * (double)dir[c];
            sy += az * z;
            sz += z * (double)r32[c];
            sw += (double)dir[c] * (double)r32[c];
        }
        double beta, dr;
        if (*dad != 0.0) {
            beta = -sx / *dad;
            dr = sz + beta * sw;
            *dad = sy + 2.0 * beta * sx + beta * beta * *dad;
        } else {
            beta = 0.0;
            *dad = sy;
            dr = sz;
        }
        const double alpha = *dad != 0.0 ? dr / *dad : 0.0;
#pragma omp parallel for schedule(static)
        for (i64 c = 0; c < C; ++c) {
            const float dn = (float)(zval(c) + beta * (double)dir[c]);
            dir[c] = dn;
            x[c] = x[c] + alpha * (double)dn;
        }
    } else {
#pragma omp parallel for schedule(static)
        for (i64 c = 0; c < C; ++c) x[c] = x[c] + zval(c);
    }
    auto xval = [&](i64 c) { return x[c]; };
    double sr = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : sr)
    for (i64 c = 0; c < C; ++c) {
        int i, j, k;
        gcoord(c, ny, nz, i, j, k);
        const double rc = fluid(c, i, j, k) ? b[c] - apply(xval, c) : 0.0;
        r[c] = rc;
        r32[c] = (float)rc;
        sr += rc * rc;
    }
    *rr = sr;
}

int orc_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

}  // extern "C"
