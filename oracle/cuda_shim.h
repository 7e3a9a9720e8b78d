/*
 * Test infrastructure (oracle only): a tiny host-side stand-in for the CUDA
 * built-ins used by the reference's CuPy RawKernel sources, so that those
 * kernel strings compile unchanged with g++ and run on CPU cores.
 *
 * A kernel call becomes a loop over (block, thread); `blockIdx`/`threadIdx`
 * are thread_local so an OpenMP loop over blocks is safe.  `atomicAdd` is a
 * plain add in serial mode (deterministic, used for golden vectors) and a
 * std::atomic_ref fetch_add when `g_ref_parallel` is set (CPU baseline).
 * Only the built-ins the live-path kernels use are provided:
 *   src/Grid.py:96-196, src/Particles.py:117-280,595-617,
 *   src/multigrid.py:13-274, src/MCC.py:7-83.
 * `__syncthreads` is a no-op, so kernels that rely on it across threads
 * (the norm kernel, src/multigrid.py:198-233) are restated by the driver
 * instead of being launched.
 */
#pragma once
#include <atomic>
#include <cmath>
#include <cstdint>

#define __global__
#define __device__
#define __forceinline__ inline

struct ref_dim3 {
    unsigned x, y, z;
};

extern thread_local ref_dim3 blockIdx;
extern thread_local ref_dim3 threadIdx;
extern thread_local ref_dim3 blockDim;
extern thread_local ref_dim3 gridDim;
extern int g_ref_parallel;

/* CUDA's overloads of min/max for the argument types the kernels mix
 * (e.g. max(0.0f, double) resolves to the double overload, as on the GPU). */
static inline double max(double a, double b) { return std::fmax(a, b); }
static inline double min(double a, double b) { return std::fmin(a, b); }
static inline float max(float a, float b) { return std::fmax(a, b); }
static inline float min(float a, float b) { return std::fmin(a, b); }
static inline int max(int a, int b) { return a > b ? a : b; }
static inline int min(int a, int b) { return a < b ? a : b; }

using std::isfinite;

static inline double atomicAdd(double* p, double v) {
    if (g_ref_parallel) return std::atomic_ref<double>(*p).fetch_add(v, std::memory_order_relaxed);
    double old = *p;
    *p = old + v;
    return old;
}
static inline int atomicAdd(int* p, int v) {
    if (g_ref_parallel) return std::atomic_ref<int>(*p).fetch_add(v, std::memory_order_relaxed);
    int old = *p;
    *p = old + v;
    return old;
}
static inline void __syncthreads() {}
