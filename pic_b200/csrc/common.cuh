// Shared device helpers and host error plumbing for libpicb200.so (sm_100a).
#pragma once

#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdint>
#include <cstdio>

#include "picb200.h"

namespace pic {

// ---- host-side status handling -------------------------------------------------

// Records a printf-style message for pic_last_error() and returns `code`.
int fail(int code, const char* fmt, ...);
void clear_error();

#define PIC_CUDA(call)                                                                              \
    do {                                                                                            \
        cudaError_t e_ = (call);                                                                    \
        if (e_ != cudaSuccess)                                                                      \
            return ::pic::fail(PIC_ERR_CUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), \
                               __FILE__, __LINE__);                                                 \
    } while (0)

#define PIC_LAUNCH_CHECK() PIC_CUDA(cudaGetLastError())

#define PIC_TRY(expr)               \
    do {                            \
        int st_ = (expr);           \
        if (st_ != PIC_OK) return st_; \
    } while (0)

inline cudaStream_t as_stream(void* s) { return static_cast<cudaStream_t>(s); }

inline int div_up(long a, long b) { return int((a + b - 1) / b); }

int num_sms();

// Raises a kernel's dynamic shared-memory limit to at least `bytes`.  The
// limit is one process-wide attribute of the kernel, so objects that need
// different sizes only ever raise it.
int raise_smem_limit(const void* kernel, size_t bytes);

// Velocity and position arrays of one species for the diagnostics kernels.
struct DiagSpecies {
    const float *vx, *vy, *vz, *x;
    int n;
};

// ---- internal electrodes --------------------------------------------------------
//
// Electrode edges are grid-line segments whose two end nodes are internal
// Dirichlet nodes: the vertical edge (X, j) is x = X, j < y < j + 1 (bit
// X * (ny - 1) + j of vb); the horizontal edge (i, Y) is y = Y, i < x < i + 1
// (bit Y * (nx - 1) + i of hb).  A particle whose straight drift (x0, y0) ->
// (x1, y1) (grid units, both inside the grid) crosses one is collected by the
// electrode.  A line is crossed when the drift ends on it or passes it, not
// when it starts on it; every crossing is intersected in FP32 with explicit
// rounding (the CPU oracle restates it operation for operation).
__device__ __forceinline__ bool edge_bit(const unsigned* b, long k) {
    return (__ldg(b + (k >> 5)) >> (k & 31)) & 1u;
}

__device__ inline bool hits_electrode(float x0, float y0, float x1, float y1, int nx, int ny,
                                      const unsigned* __restrict__ vb, const unsigned* __restrict__ hb) {
    const float ddx = __fsub_rn(x1, x0), ddy = __fsub_rn(y1, y0);
    if (ddx != 0.0f) {
        int a = ddx > 0.0f ? int(floorf(x0)) + 1 : int(ceilf(x1));
        int b = ddx > 0.0f ? int(floorf(x1)) : int(ceilf(x0)) - 1;
        a = max(a, 1);
        b = min(b, nx - 2);
        for (int X = a; X <= b; ++X) {
            const float t = __fdiv_rn(__fsub_rn(float(X), x0), ddx);
            const int j = int(floorf(__fmaf_rn(t, ddy, y0)));
            if (j >= 0 && j < ny - 1 && edge_bit(vb, long(X) * (ny - 1) + j)) return true;
        }
    }
    if (ddy != 0.0f) {
        int a = ddy > 0.0f ? int(floorf(y0)) + 1 : int(ceilf(y1));
        int b = ddy > 0.0f ? int(floorf(y1)) : int(ceilf(y0)) - 1;
        a = max(a, 1);
        b = min(b, ny - 2);
        for (int Y = a; Y <= b; ++Y) {
            const float t = __fdiv_rn(__fsub_rn(float(Y), y0), ddy);
            const int i = int(floorf(__fmaf_rn(t, ddx, x0)));
            if (i >= 0 && i < nx - 1 && edge_bit(hb, long(Y) * (nx - 1) + i)) return true;
        }
    }
    return false;
}

// ---- r-z node volumes -------------------------------------------------------------
//
// Volume of node row j of an r-z grid divided by dx*dy (so, in metres): the
// integral of 2 pi r times the row's linear weighting function over r.  With
// these volumes a uniformly loaded plasma deposits a uniform density:
// 2 pi r_j inside, pi dy / 3 on the axis, pi (r_top - dy/3) on the outer row.
__host__ __device__ inline double rz_row_volume(int j, int ny, double dy) {
    const double pi = 3.14159265358979323846;
    if (j == 0) return pi * dy / 3.0;
    if (j == ny - 1) return pi * (double(j) * dy - dy / 3.0);
    return 2.0 * pi * double(j) * dy;
}

// ---- r-z drift ---------------------------------------------------------------------
//
// One drift of an axisymmetric particle (x axial and y radial, grid units; vx
// axial, vy radial, vz azimuthal, m/s).  The particle moves on a straight line
// in 3D: in the plane normal to the axis it goes from (y, 0) to (y', t) =
// (y + vy dt/dy, vz dt/dy), its new radius is |(y', t)|, and (vy, vz) are
// turned by the angle of (y', t) into the new radial and azimuthal directions
// (Birdsall and Langdon, Plasma Physics via Computer Simulation, sec. 14-12).
// A path through the axis comes out on the other side with r >= 0.  Every
// operation is correctly rounded (IEEE square root and division), so the
// FP32 oracle reproduces it bit for bit.
__device__ __forceinline__ void drift_rz(float& x, float& y, float vx, float& vy, float& vz, float dtdx, float dtdy) {
    x = __fmaf_rn(vx, dtdx, x);
    const float yr = __fmaf_rn(vy, dtdy, y);
    const float yt = __fmul_rn(vz, dtdy);
    const float r = __fsqrt_rn(__fmaf_rn(yr, yr, __fmul_rn(yt, yt)));
    if (r > 0.0f) {
        const float c = __fdiv_rn(yr, r), s = __fdiv_rn(yt, r);
        const float vr = __fmaf_rn(c, vy, __fmul_rn(s, vz));
        const float vt = __fmaf_rn(c, vz, -__fmul_rn(s, vy));
        vy = vr;
        vz = vt;
    }
    y = r;
}

// ---- CIC weights (FP32, explicit rounding so the CPU oracle matches bit for bit) ----

struct Cic {
    int i0, j0, i1, j1;
    float w00, w10, w01, w11;
};

// Clamp to [0, n-1], floor, neighbour = min(i0+1, n-1): the rule of
// src/Grid.py:116-137 and src/Particles.py:140-163, in FP32 grid units.
__device__ __forceinline__ Cic cic_weights(float gx, float gy, int nx, int ny) {
    Cic c;
    const float cx = fminf(fmaxf(gx, 0.0f), float(nx - 1));
    const float cy = fminf(fmaxf(gy, 0.0f), float(ny - 1));
    c.i0 = int(floorf(cx));
    c.j0 = int(floorf(cy));
    c.i1 = min(c.i0 + 1, nx - 1);
    c.j1 = min(c.j0 + 1, ny - 1);
    const float wx = __fsub_rn(cx, float(c.i0));
    const float wy = __fsub_rn(cy, float(c.j0));
    const float ux = __fsub_rn(1.0f, wx);
    const float uy = __fsub_rn(1.0f, wy);
    c.w00 = __fmul_rn(ux, uy);
    c.w10 = __fmul_rn(wx, uy);
    c.w01 = __fmul_rn(ux, wy);
    c.w11 = __fmul_rn(wx, wy);
    return c;
}

// cic_weights for a position already in [0, nx-1] x [0, ny-1], where the
// clamp changes nothing: the same weights without it.
__device__ __forceinline__ Cic cic_weights_in_domain(float gx, float gy, int nx, int ny) {
    Cic c;
    c.i0 = int(floorf(gx));
    c.j0 = int(floorf(gy));
    c.i1 = min(c.i0 + 1, nx - 1);
    c.j1 = min(c.j0 + 1, ny - 1);
    const float wx = __fsub_rn(gx, float(c.i0));
    const float wy = __fsub_rn(gy, float(c.j0));
    const float ux = __fsub_rn(1.0f, wx);
    const float uy = __fsub_rn(1.0f, wy);
    c.w00 = __fmul_rn(ux, uy);
    c.w10 = __fmul_rn(wx, uy);
    c.w01 = __fmul_rn(ux, wy);
    c.w11 = __fmul_rn(wx, wy);
    return c;
}

// Interpolated field value: ((w00*a + w10*b) + w01*c) + w11*d with the first
// product rounded and the rest fused, in this order.
__device__ __forceinline__ float cic_interp(const Cic& c, float a, float b, float cc, float d) {
    float v = __fmul_rn(c.w00, a);
    v = __fmaf_rn(c.w10, b, v);
    v = __fmaf_rn(c.w01, cc, v);
    v = __fmaf_rn(c.w11, d, v);
    return v;
}

__device__ __forceinline__ bool is_live(float x) { return x == x; }

// ---- Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11) ----------------------------

__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint2 k) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        if (r) {
            k.x += 0x9E3779B9u;
            k.y += 0xBB67AE85u;
        }
        const uint32_t lo0 = 0xD2511F53u * c.x, hi0 = __umulhi(0xD2511F53u, c.x);
        const uint32_t lo1 = 0xCD9E8D57u * c.z, hi1 = __umulhi(0xCD9E8D57u, c.z);
        c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
    }
    return c;
}

// Uniforms in (0, 1]: double from all 32 bits, float from the top 24 bits.
__device__ __forceinline__ double u01_double(uint32_t x) { return (double(x) + 1.0) * (1.0 / 4294967296.0); }
__device__ __forceinline__ float u01_float(uint32_t x) {
    return __fadd_rn(__fmul_rn(float(x >> 8), 1.0f / 16777216.0f), 0.5f / 16777216.0f);
}

// ---- programmatic dependent launch -----------------------------------------------
//
// A kernel launched with launch_pdl may be scheduled while the kernel before
// it on the stream still runs (once every CTA of that kernel has called
// pdl_trigger, or exited).  pdl_wait blocks until that kernel has completed
// and its memory is visible; both are no-ops for a launch without the
// attribute.

__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

template <class... KArgs, class... Args>
static cudaError_t launch_pdl(void (*k)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                              Args... args) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, k, args...);
}

// ---- block reductions -----------------------------------------------------------

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

}  // namespace pic
