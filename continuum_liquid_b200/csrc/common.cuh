// Shared definitions for the Continuum Liquid B200 kernels.
//
// The whole library is compiled with -fmad=false, so every floating-point + - * / in these kernels is
// a separately rounded IEEE operation (division and sqrt are correctly rounded: -prec-div/-prec-sqrt
// stay at their defaults). Together with the reference's evaluation orders, restated per kernel, this
// makes the bin keys, sort, P2G, G2P, boundary conditions and red-black Gauss-Seidel sweeps
// reproduce the CPU restatement bit for bit.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <atomic>
#include <stdarg.h>
#include <stdio.h>

namespace clb {

typedef int64_t i64;

// helper.cl:4-6 grid_index (k fastest); 64-bit so that 1024^3 grids do not overflow.
__host__ __device__ __forceinline__ i64 gidx(int i, int j, int k, int ny, int nz) {
    return ((i64)i * ny + j) * nz + k;
}

// helper.cl:8-15 grid_coordinates. Every grid has fewer than 2^31 cells (checked at each entry
// point), so the decode uses 32-bit unsigned division.
__device__ __forceinline__ void gcoord(i64 index, int ny, int nz, int& i, int& j, int& k) {
    const uint32_t yz = (uint32_t)ny * (uint32_t)nz;
    const uint32_t c = (uint32_t)index;
    const uint32_t ii = c / yz;
    const uint32_t rem = c - ii * yz;
    const uint32_t jj = rem / (uint32_t)nz;
    i = (int)ii;
    j = (int)jj;
    k = (int)(rem - jj * (uint32_t)nz);
}

// helper.cl:21-23 is_interior_cell
__host__ __device__ __forceinline__ bool interior(int i, int j, int k, int nx, int ny, int nz) {
    return i > 0 && j > 0 && k > 0 && i < nx - 1 && j < ny - 1 && k < nz - 1;
}

__host__ __device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// Error word written by kernels whose bounded waits ran out (read and cleared by clb_device_error).
// Codes: 1 = scan look-back gave up, 2 = bounded wait elsewhere gave up, 3 = index out of range.
__device__ unsigned int g_device_error = 0;

__device__ __forceinline__ void raise_device_error(unsigned int code) { atomicCAS(&g_device_error, 0u, code); }

// Thread-local last error text (clb_last_error).
static thread_local char t_last_error[512] = {0};

static inline int set_error(const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(t_last_error, sizeof(t_last_error), fmt, ap);
    va_end(ap);
    return 1;
}

// Kernels launched by this library since load (host side; graph replays are not counted).
static std::atomic<long long> g_launches{0};

static inline int check_launch(const char* what) {
    g_launches.fetch_add(1, std::memory_order_relaxed);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return set_error("%s: %s", what, cudaGetErrorString(e));
    return 0;
}

static inline int check_call(cudaError_t e, const char* what) {
    if (e != cudaSuccess) return set_error("%s: %s", what, cudaGetErrorString(e));
    return 0;
}

static inline unsigned int blocks_for(i64 n, int threads) { return (unsigned int)((n + threads - 1) / threads); }

// Number of SMs on the current device (cached per process; the library serves one GPU).
static int g_sm_count = 0;

// Programmatic dependent launch. The pressure-solve kernels are launched with programmatic stream
// serialisation (launch()), so a kernel's blocks may be scheduled while its predecessor in the stream
// is still running; each such kernel calls pdl_begin() before its first memory access. pdl_begin
// waits until the predecessor grid has completed and its writes are visible (griddepcontrol.wait:
// immediate when the kernel was launched without the attribute), then allows the next kernel of the
// stream to be scheduled. A grid completes only after every block has passed its own wait, so
// dependences on kernels further back in the stream hold as well. The waiting blocks are placed only
// after all blocks of the running grid have started, so they never take an SM a running grid needs.
__device__ __forceinline__ void pdl_begin() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

static bool g_use_pdl = true;  // clb_mg_set_option(1, ...) switches programmatic dependent launch off

// launch(grid, block, smem, stream)(kernel, args...): the kernel launch with programmatic stream
// serialisation (when enabled); the kernel must start with pdl_begin(). Errors are left for
// check_launch (cudaGetLastError).
struct Launch {
    dim3 grid, block;
    size_t smem;
    cudaStream_t stream;
    template <typename... P, typename... A>
    void operator()(void (*kernel)(P...), A&&... args) const {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = grid;
        cfg.blockDim = block;
        cfg.dynamicSmemBytes = smem;
        cfg.stream = stream;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attr[0].val.programmaticStreamSerializationAllowed = 1;
        cfg.attrs = attr;
        cfg.numAttrs = g_use_pdl ? 1 : 0;
        (void)cudaLaunchKernelEx(&cfg, kernel, static_cast<A&&>(args)...);
    }
};

static inline Launch launch(dim3 grid, dim3 block, size_t smem, cudaStream_t stream) {
    return Launch{grid, block, smem, stream};
}

}  // namespace clb

#define CLB_REQUIRE(cond, ...)                  \
    do {                                        \
        if (!(cond)) return clb::set_error(__VA_ARGS__); \
    } while (0)

#define CLB_LAUNCH_CHECK(what)                    \
    do {                                          \
        if (clb::check_launch(what)) return 1;    \
    } while (0)
