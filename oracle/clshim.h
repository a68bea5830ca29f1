// OpenCL C, the subset the reference's kernels use, as C++17 on the host. Test infrastructure only.
//
// oracle/ref_build.py rewrites the reference's Solver/Kernel/OpenCL/*.cl into C++ that includes this
// header (vector literals become function calls, includes are inlined, a registration line per
// kernel is appended) and compiles it into oracle/_ref/. oracle/pyopencl_shim/ then runs the
// reference's own Python host code (Solver/Kernel/*.py) on those kernels, so the reference solver
// produces outputs here although no OpenCL device exists.
//
// Semantics (the ones the oracle restatement uses too; OpenCL leaves them to the implementation):
//   * every float operation separately rounded (built with -ffp-contract=off), division and sqrt
//     correctly rounded;
//   * dot(a,b) = a.x*b.x + a.y*b.y + a.z*b.z left to right, length(a) = sqrt(dot(a,a)),
//     normalize(a) = a / length(a) per component, cross as the textbook determinant;
//   * work-items run one after another in index order (so atomic_inc hands out slots in index
//     order, which makes sort_particles stable); a work-group whose kernel calls barrier() runs its
//     work-items as cooperative fibers that switch at every barrier.
#pragma once

#include <math.h>
#include <stddef.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>

#include <type_traits>
#include <utility>

#define __kernel
#define __global
#define __local
#define __private
#define __constant const
#define CLK_LOCAL_MEM_FENCE 1
#define CLK_GLOBAL_MEM_FENCE 2

typedef unsigned int uint;
typedef unsigned char uchar;

// ---- vector types --------------------------------------------------------------------------------
struct float3 {
    float x, y, z;
};
struct int3 {
    int x, y, z;
};
struct float4 {
    union {
        struct {
            float x, y, z, w;
        };
        float3 xyz;
    };
};

static inline float3 clshim_float3(float a) { return float3{a, a, a}; }
static inline float3 clshim_float3(float a, float b, float c) { return float3{a, b, c}; }
static inline int3 clshim_int3(int a) { return int3{a, a, a}; }
static inline int3 clshim_int3(int a, int b, int c) { return int3{a, b, c}; }
static inline float4 clshim_float4(float a) {
    float4 r;
    r.x = r.y = r.z = r.w = a;
    return r;
}
static inline float4 clshim_float4(float3 a, float w) {
    float4 r;
    r.x = a.x;
    r.y = a.y;
    r.z = a.z;
    r.w = w;
    return r;
}

#define CLSHIM_BINARY(T, S, OP)                                                                            \
    static inline T operator OP(T a, T b) { return T{a.x OP b.x, a.y OP b.y, a.z OP b.z}; }                \
    static inline T operator OP(T a, S b) { return T{a.x OP b, a.y OP b, a.z OP b}; }                      \
    static inline T operator OP(S a, T b) { return T{a OP b.x, a OP b.y, a OP b.z}; }                      \
    static inline T& operator OP##=(T & a, T b) { return a = a OP b; }                                     \
    static inline T& operator OP##=(T & a, S b) { return a = a OP b; }
CLSHIM_BINARY(float3, float, +)
CLSHIM_BINARY(float3, float, -)
CLSHIM_BINARY(float3, float, *)
CLSHIM_BINARY(float3, float, /)
CLSHIM_BINARY(int3, int, +)
CLSHIM_BINARY(int3, int, -)
CLSHIM_BINARY(int3, int, *)
CLSHIM_BINARY(int3, int, /)
CLSHIM_BINARY(int3, int, |)
CLSHIM_BINARY(int3, int, &)
#undef CLSHIM_BINARY

static inline float3 operator-(float3 a) { return float3{-a.x, -a.y, -a.z}; }
static inline int3 operator-(int3 a) { return int3{-a.x, -a.y, -a.z}; }
static inline float4 operator+(float4 a, float4 b) {
    float4 r;
    r.x = a.x + b.x;
    r.y = a.y + b.y;
    r.z = a.z + b.z;
    r.w = a.w + b.w;
    return r;
}
static inline float4& operator+=(float4& a, float4 b) { return a = a + b; }

// Relational operators of vectors give -1 (all bits set) where true and 0 where false.
#define CLSHIM_RELATION(T, S, OP)                                                                          \
    static inline int3 operator OP(T a, T b) {                                                            \
        return int3{-(int)(a.x OP b.x), -(int)(a.y OP b.y), -(int)(a.z OP b.z)};                          \
    }                                                                                                      \
    static inline int3 operator OP(T a, S b) {                                                            \
        return int3{-(int)(a.x OP b), -(int)(a.y OP b), -(int)(a.z OP b)};                                \
    }                                                                                                      \
    static inline int3 operator OP(S a, T b) {                                                            \
        return int3{-(int)(a OP b.x), -(int)(a OP b.y), -(int)(a OP b.z)};                                \
    }
CLSHIM_RELATION(float3, float, <)
CLSHIM_RELATION(float3, float, >)
CLSHIM_RELATION(float3, float, <=)
CLSHIM_RELATION(float3, float, >=)
CLSHIM_RELATION(float3, float, ==)
CLSHIM_RELATION(float3, float, !=)
CLSHIM_RELATION(int3, int, <)
CLSHIM_RELATION(int3, int, >)
CLSHIM_RELATION(int3, int, ==)
CLSHIM_RELATION(int3, int, !=)
#undef CLSHIM_RELATION

static inline int any(int3 a) { return (a.x < 0) || (a.y < 0) || (a.z < 0); }
static inline int all(int3 a) { return (a.x < 0) && (a.y < 0) && (a.z < 0); }

// select(a, b, c): b where the most significant bit of c is set, else a.
static inline float3 select(float3 a, float3 b, int3 c) {
    return float3{c.x < 0 ? b.x : a.x, c.y < 0 ? b.y : a.y, c.z < 0 ? b.z : a.z};
}

// ---- conversions ---------------------------------------------------------------------------------
static inline int3 convert_int3_rtn(float3 a) { return int3{(int)floorf(a.x), (int)floorf(a.y), (int)floorf(a.z)}; }
static inline int3 convert_int3_rtz(float3 a) { return int3{(int)a.x, (int)a.y, (int)a.z}; }
static inline float3 convert_float3(int3 a) { return float3{(float)a.x, (float)a.y, (float)a.z}; }
static inline float convert_float(int a) { return (float)a; }

// ---- common and geometric functions ------------------------------------------------------------
static inline float clshim_fmin(float a, float b) { return b < a ? b : a; }
static inline float clshim_fmax(float a, float b) { return a < b ? b : a; }
static inline int clamp(int x, int lo, int hi) { return x < lo ? lo : (x > hi ? hi : x); }
static inline float clamp(float x, float lo, float hi) { return clshim_fmin(clshim_fmax(x, lo), hi); }
static inline int3 clamp(int3 x, int3 lo, int3 hi) {
    return int3{clamp(x.x, lo.x, hi.x), clamp(x.y, lo.y, hi.y), clamp(x.z, lo.z, hi.z)};
}
static inline float3 clamp(float3 x, float lo, float hi) {
    return float3{clamp(x.x, lo, hi), clamp(x.y, lo, hi), clamp(x.z, lo, hi)};
}
static inline float3 clamp(float3 x, float3 lo, float3 hi) {
    return float3{clamp(x.x, lo.x, hi.x), clamp(x.y, lo.y, hi.y), clamp(x.z, lo.z, hi.z)};
}
static inline int3 min(int3 a, int3 b) {
    return int3{b.x < a.x ? b.x : a.x, b.y < a.y ? b.y : a.y, b.z < a.z ? b.z : a.z};
}
static inline int3 max(int3 a, int3 b) {
    return int3{a.x < b.x ? b.x : a.x, a.y < b.y ? b.y : a.y, a.z < b.z ? b.z : a.z};
}
static inline float3 max(float3 a, float3 b) {
    return float3{clshim_fmax(a.x, b.x), clshim_fmax(a.y, b.y), clshim_fmax(a.z, b.z)};
}
static inline float3 min(float3 a, float3 b) {
    return float3{clshim_fmin(a.x, b.x), clshim_fmin(a.y, b.y), clshim_fmin(a.z, b.z)};
}
static inline float3 fabs(float3 a) { return float3{fabsf(a.x), fabsf(a.y), fabsf(a.z)}; }
static inline float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline float3 cross(float3 a, float3 b) {
    return float3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
static inline float length(float3 a) { return sqrtf(dot(a, a)); }
static inline float3 normalize(float3 a) { return a / length(a); }

static inline float3 vload3(size_t offset, const float* p) {
    return float3{p[3 * offset], p[3 * offset + 1], p[3 * offset + 2]};
}
static inline void vstore3(float3 v, size_t offset, float* p) {
    p[3 * offset] = v.x;
    p[3 * offset + 1] = v.y;
    p[3 * offset + 2] = v.z;
}

static inline uint atomic_inc(volatile uint* p) { return __atomic_fetch_add(p, 1u, __ATOMIC_RELAXED); }
static inline int atomic_inc(volatile int* p) { return __atomic_fetch_add(p, 1, __ATOMIC_RELAXED); }

// ---- work-items ----------------------------------------------------------------------------------
struct clshim_item {
    size_t global_id[3], local_id[3], group_id[3];
};
struct clshim_range {
    int dims;
    size_t global_size[3], local_size[3];
};
extern thread_local const clshim_item* clshim_current_item;
extern thread_local const clshim_range* clshim_current_range;

static inline size_t get_global_id(int d) { return clshim_current_item->global_id[d]; }
static inline size_t get_local_id(int d) { return clshim_current_item->local_id[d]; }
static inline size_t get_group_id(int d) { return clshim_current_item->group_id[d]; }
static inline size_t get_local_size(int d) { return clshim_current_range->local_size[d]; }
static inline size_t get_global_size(int d) { return clshim_current_range->global_size[d]; }
static inline size_t get_num_groups(int d) {
    return clshim_current_range->global_size[d] / clshim_current_range->local_size[d];
}
static inline uint get_work_dim() { return (uint)clshim_current_range->dims; }

void barrier(int flags);

// ---- kernel registration -------------------------------------------------------------------------
// A kernel is invoked through a type-erased entry: argv[i] points at the storage of argument i (a
// pointer value for buffers and local memory, the scalar itself otherwise).
typedef void (*clshim_entry)(void** argv);

template <typename... A, size_t... I>
static inline void clshim_call(void (*f)(A...), void** argv, std::index_sequence<I...>) {
    f(*reinterpret_cast<std::remove_cv_t<std::remove_reference_t<A>>*>(argv[I])...);
}
template <typename... A>
static inline int clshim_arity(void (*)(A...)) {
    return (int)sizeof...(A);
}
template <typename... A>
static inline void clshim_invoke(void (*f)(A...), void** argv) {
    clshim_call(f, argv, std::index_sequence_for<A...>{});
}

void clshim_register(const char* name, clshim_entry entry, int arity, int uses_barrier);

// Appended by oracle/ref_build.py once per __kernel of a translated file.
#define CLSHIM_REGISTER(NAME, USES_BARRIER)                                                                \
    static void clshim_entry_##NAME(void** argv) { clshim_invoke(NAME, argv); }                           \
    static const int clshim_registered_##NAME =                                                           \
        (clshim_register(#NAME, clshim_entry_##NAME, clshim_arity(NAME), USES_BARRIER), 0);
