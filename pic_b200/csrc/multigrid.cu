// Geometric multigrid Poisson solver (replaces src/multigrid.py:277-455).
//
// Outer loop: FP64 iterative refinement on the fine grid
//     r = f - A phi   (FP64, 5-point operator on free nodes)
//     solve A e = r approximately with one V-cycle from e = 0
//     phi += e        (FP64)
// until ||r|| / ||f|| < tol or max_cycles.  The V-cycle runs in FP32
// (PIC_MG_MIXED) or FP64 (PIC_MG_FP64): red-black Gauss-Seidel smoothing,
// full-weighting restriction, bilinear prolongation, a dense FP64 solve on
// the coarsest level.  Dirichlet nodes (mask = 1, and the grid edges) carry a
// zero correction; a coarse node is Dirichlet when its injected fine node is.
//
// Kernels per V-cycle in the graph and host loops (7 launches for a 513^2
// grid):
//   down(l)     2*pre red/black half-sweeps on a 32x32 tile held in shared
//               memory with a halo wide enough for them, then the residual
//               and its full-weighting restriction to level l+1; on level 0
//               the right-hand side is the FP64 residual r
//   down2       the down phases of two levels (129^2 and 65^2 at 513^2) in
//               one launch, over halos wide enough that the coarser level's
//               tile equals what two launches give
//   direct      e = A^-1 g on the first level of at most 33^2 nodes (the
//               dense inverse of that level's operator on its free nodes,
//               formed at creation), one warp per row
//   up2         the up phases of the same two levels in one launch
//   up(l)       prolongation-add of level l+1 and 2*post half-sweeps
//   up_res      the finest up phase: phi += e, the FP64 residual updated on
//               the tile (r -= A e), its norm (deterministic last-block
//               reduction) and the loop decision
//   r0          once per solve, before the first cycle: r = f - A phi in
//               FP64, its norm and the first loop decision
// The single-CTA coarse kernel (every level of at most 33^2 nodes in shared
// memory, down to a dense solve) serves grids that small and the persistent
// and cluster modes.  The loop is a CUDA-graph conditional WHILE node whose
// condition up_res (r0 before the first cycle) sets, so a solve issues no
// host synchronisation.
#include <cooperative_groups.h>
#include <cuda/atomic>

#include <cmath>
#include <cstring>
#include <type_traits>
#include <vector>

#include "common.cuh"
#include "band_inverse.h"

namespace pic {

int grid_blocks(long n, int threads);

constexpr int kMgTile = 32;
constexpr int kMgThreads = 512;
constexpr int kMgMaxSweeps = 8;
constexpr int kMgMaxCoarseLevels = 8;
constexpr int kCoarseThreads = 1024;
constexpr long kCoarseMaxNodes32 = 33L * 33L;    // FP32 levels at or below this size run in the single-CTA kernel
constexpr long kCoarseMaxNodes64 = 33L * 33L;    // FP64 levels
constexpr int kMgMaxLevels = 16;
constexpr long kPersistCoarseMax = 33L * 33L;    // levels the persistent kernel's single block solves
constexpr long kHybridBandMax = 129L * 129L;     // PIC_MG_HYBRID: levels at or below this size run in the cluster
constexpr unsigned long long kBarrierPolls = 1ull << 24;  // a grid barrier gives up (error flag) after this

// One level of the hierarchy.  The correction has two arrays: the down
// phase writes e, and the up phase reads e (with its halo) and writes its
// result to eu, so that no kernel reads a neighbour tile's e while another
// CTA overwrites it.  ec is the correction the next finer level prolongs:
// eu on levels the up kernels smooth, e on the first level of a single-block
// coarse V-cycle (which writes e); the launch code sets it per launch mode.
template <class T>
struct LevelDev {
    int nx, ny;
    T cx, cy, inv_diag;
    const uint8_t* mask;  // 1 = Dirichlet
    T* e;
    T* eu;
    T* ec;
    T* g;
    // r-z geometry (row j = radius j*hy, row 0 the axis): per row
    // {wN, wS, 1/diag, D}, the weights of rows j+1 and j-1, the inverse
    // diagonal and the row's volume weight (j, 1/8 on the axis); null in
    // Cartesian geometry
    const T* rz;
};

// The residual norm and the loop decision: block partials, the counter of
// blocks finished, and the solve's state.
struct NormState {
    double* partial;   // [nblocks] r^2, then [nblocks] f^2
    unsigned* done;    // blocks finished
    double* norms;     // [||f||^2, ||r||^2]
    int* converged;
    int* cycles;       // V-cycles of the current solve
    long long* total;  // V-cycles since creation
};

// The finest up phase fused with the FP64 residual (k_mg_up_res).
struct ResArgs {
    double* r64;        // the residual of phi, FP64, kept between cycles
    const double* rz0;  // r-z: level-0 row coefficients in FP64, else null
    double cx, cy;
    NormState N;
    double tol2;
    int max_cycles;
    cudaGraphConditionalHandle cond;
    int use_cond;
};

// The levels as a launch mode uses them: up phases on the levels below
// `first_coarse` (their final correction is eu), the coarse V-cycle from it.
template <class T>
static std::vector<LevelDev<T>> with_corrections(const std::vector<LevelDev<T>>& lv, int first_coarse) {
    std::vector<LevelDev<T>> out = lv;
    for (size_t l = 0; l < out.size(); ++l) out[l].ec = int(l) < first_coarse ? out[l].eu : out[l].e;
    return out;
}

template <class T>
struct CoarseDesc {
    int nlev;
    LevelDev<T> lv[kMgMaxCoarseLevels];
    // shared memory, in bytes: the e arrays [0, e_bytes), then the g arrays, the
    // masks [m_off, ...) and, when they fit, the dense inverse (a_off) and its
    // node table (c_off); a_off < 0 reads those two from global memory
    int off_e[kMgMaxCoarseLevels], off_g[kMgMaxCoarseLevels], off_m[kMgMaxCoarseLevels];
    int e_bytes, m_off, a_off, c_off;
    // 16-byte sources of the one batch of loads that fills shared memory: the
    // mask image (edges and electrodes of every level), the finest level's g,
    // the inverse and the table; *_vec = 16-byte words of each
    const uint4* mimg;
    const uint4* g16;
    const uint4* ainv16;
    const uint4* cidx16;
    int m_vec, g_vec, a_vec, c_vec;
    const double* ainv;
    const int* cidx;
    int nf;
    T omega;
    int pre, post;
    double* phi0;  // set when the coarse kernel owns level 0: phi += e
};

// ---- shared-memory tile smoothing -------------------------------------------------
//
// Tile kernels are instantiated per sweep count S (1..kMgMaxSweeps), so the
// tile width W is a compile-time constant: index arithmetic becomes
// multiply-shift, and every global load of a phase is issued before the first
// one is used.

// Programmatic dependent launch: the V-cycle is a chain of small dependent
// kernels, launched with cudaLaunchAttributeProgrammaticStreamSerialization so
// that each one is scheduled while its predecessor runs.  pdl_wait blocks
// until the preceding grid has completed and its memory is visible (a no-op
// for a launch without the attribute); every kernel triggers its successor
// right after its own wait, so at most two grids of the chain are resident and
// the code of a kernel before its wait may read anything written two or more
// launches earlier (never what the kernel just before it writes).  The up
// kernels load their whole fine tile (mask, g, e of their level, phi) there,
// so only the coarse correction's load follows the wait.

template <int S>
struct DownGeom {
    static constexpr int H = 2 * S + 2, W = kMgTile + 2 * H;
};
// RES: the finest up phase fused with the residual, one more halo row so that
// e is final one node beyond the core.
template <int S, bool RES = false>
struct UpGeom {
    static constexpr int H = 2 * S + (RES ? 1 : 0), W = kMgTile + 2 * H, CW = W / 2 + 2;
};

// One red or black half-sweep over the nodes 1..W-2 of a W x W shared tile;
// `par` selects the nodes whose local (li + lj) parity equals it.
template <class T, int W, bool CYL>
__device__ __forceinline__ void tile_half_sweep(T* __restrict__ se, const T* __restrict__ sg,
                                                const uint8_t* __restrict__ sm, int par, T cx, T cy, T inv_diag,
                                                T omega, const T* __restrict__ srz) {
    constexpr int half = W / 2, N = half * W, IT = (N + kMgThreads - 1) / kMgThreads;
#pragma unroll
    for (int it = 0; it < IT; ++it) {
        const int q = it * kMgThreads + int(threadIdx.x);
        if (q >= N) break;
        const int lj = q / half;
        const int li = 2 * (q - lj * half) + ((par + lj) & 1);
        if (lj < 1 || lj > W - 2 || li < 1 || li > W - 2) continue;
        const int p = lj * W + li;
        if (sm[p]) continue;
        T upd;
        if constexpr (CYL) {
            const T* rc = srz + 4 * lj;
            const T s = cx * (se[p - 1] + se[p + 1]) + rc[0] * se[p + W] + rc[1] * se[p - W];
            upd = (s - sg[p]) * rc[2];
        } else {
            const T s = cx * (se[p - 1] + se[p + 1]) + cy * (se[p - W] + se[p + W]);
            upd = (s - sg[p]) * inv_diag;
        }
        const T old = se[p];
        se[p] = old + omega * (upd - old);
    }
}

// Loads level L over the W x W region at (ox, oy): mask (edges and outside
// the grid count as Dirichlet; in r-z geometry the axis row is free), g (from
// g64, the FP64 residual, when given), e (zero, or the stored correction on
// free nodes) and, in r-z geometry, the row coefficients of the W rows (zero
// outside the grid).
template <class T, int W, bool LOAD_E, bool CYL>
__device__ __forceinline__ void tile_load(const LevelDev<T>& L, int ox, int oy, T* __restrict__ se,
                                          T* __restrict__ sg, uint8_t* __restrict__ sm, T* __restrict__ srz,
                                          const double* __restrict__ g64 = nullptr) {
    constexpr int N = W * W, IT = (N + kMgThreads - 1) / kMgThreads;
    uint8_t mk[IT];
    T gv[IT], ev[IT];
#pragma unroll
    for (int it = 0; it < IT; ++it) {
        const int q = it * kMgThreads + int(threadIdx.x);
        const int i = ox + q % W, j = oy + q / W;
        const bool in = q < N && i >= 0 && j >= 0 && i < L.nx && j < L.ny;
        const long k = long(j) * L.nx + i;
        mk[it] = in ? L.mask[k] : uint8_t(1);
        gv[it] = in ? (g64 ? T(g64[k]) : L.g[k]) : T(0);
        ev[it] = (LOAD_E && in) ? L.e[k] : T(0);
    }
    if constexpr (CYL) {
        for (int q = threadIdx.x; q < 4 * W; q += kMgThreads) {
            const int j = oy + q / 4;
            srz[q] = (j >= 0 && j < L.ny) ? L.rz[4 * j + q % 4] : T(0);
        }
    }
#pragma unroll
    for (int it = 0; it < IT; ++it) {
        const int q = it * kMgThreads + int(threadIdx.x);
        if (q >= N) break;
        const int i = ox + q % W, j = oy + q / W;
        const bool fr = i > 0 && (CYL ? j >= 0 : j > 0) && i < L.nx - 1 && j < L.ny - 1 && !mk[it];
        sm[q] = fr ? 0 : 1;
        sg[q] = gv[it];
        se[q] = fr ? ev[it] : T(0);
    }
}

// g64 (level 0 of the graph and host loops): the right-hand side is the FP64
// residual, and the tile stores its FP32 copy of the core to F.g for the up
// phase of the same cycle.
template <class T, int S, bool CYL = false>
__device__ void down_tile(const LevelDev<T>& F, const LevelDev<T>& Cc, T omega, int tx, int ty,
                          unsigned char* smem, const double* __restrict__ g64 = nullptr) {
    constexpr int H = DownGeom<S>::H, W = DownGeom<S>::W, hx = kMgTile / 2;
    static_assert(hx * hx <= kMgThreads, "one coarse node per thread");
    T* se = reinterpret_cast<T*>(smem);
    T* sg = se + W * W;
    T* srz = sg + W * W;  // r-z row coefficients (4 W values), only with CYL
    uint8_t* sm = reinterpret_cast<uint8_t*>(srz + (CYL ? 4 * W : 0));
    const int x0 = tx * kMgTile, y0 = ty * kMgTile;
    const int ox = x0 - H, oy = y0 - H;
    const int tid = threadIdx.x;
    // the coarse node this thread restricts to, and its mask (loaded early)
    const int I = x0 / 2 + tid % hx, J = y0 / 2 + tid / hx;
    const bool own = tid < hx * hx && I < Cc.nx && J < Cc.ny;
    const long K = long(J) * Cc.nx + I;
    const bool cdir = own && (I == 0 || (!CYL && J == 0) || I == Cc.nx - 1 || J == Cc.ny - 1 || Cc.mask[K]);
    tile_load<T, W, false, CYL>(F, ox, oy, se, sg, sm, srz, g64);
    __syncthreads();
    // global red nodes have (i + j) even; locally (li + lj + ox + oy) even
    const int par0 = (ox + oy) & 1;
#pragma unroll 1
    for (int s = 0; s < S; ++s)
#pragma unroll
        for (int color = 0; color < 2; ++color) {
            tile_half_sweep<T, W, CYL>(se, sg, sm, color ^ par0, F.cx, F.cy, F.inv_diag, omega, srz);
            __syncthreads();
        }
#pragma unroll
    for (int q = tid; q < kMgTile * kMgTile; q += kMgThreads) {
        const int i = x0 + q % kMgTile, j = y0 + q / kMgTile;
        if (i >= F.nx || j >= F.ny) continue;
        const int lq = (H + q / kMgTile) * W + H + q % kMgTile;
        F.e[long(j) * F.nx + i] = se[lq];
        if (g64) F.g[long(j) * F.nx + i] = sg[lq];
    }
    // residual in place of g (each node reads only its own g)
    constexpr int IT = (W * W + kMgThreads - 1) / kMgThreads;
#pragma unroll
    for (int it = 0; it < IT; ++it) {
        const int q = it * kMgThreads + tid;
        if (q >= W * W) break;
        const int li = q % W, lj = q / W;
        if (li < 1 || lj < 1 || li > W - 2 || lj > W - 2 || sm[q]) continue;
        const T c = se[q];
        if constexpr (CYL) {
            // the residual weighted by the row's volume, for the volume-weighted restriction
            const T* rc = srz + 4 * lj;
            const T lap = F.cx * (se[q - 1] + se[q + 1] - T(2) * c) + rc[0] * (se[q + W] - c) + rc[1] * (se[q - W] - c);
            sg[q] = rc[3] * (sg[q] - lap);
        } else {
            const T lap = F.cx * (se[q - 1] + se[q + 1] - T(2) * c) + F.cy * (se[q - W] + se[q + W] - T(2) * c);
            sg[q] = sg[q] - lap;
        }
    }
    __syncthreads();
    // full weighting onto the coarse nodes injected from this tile
    if (own) {
        if (cdir) {
            Cc.g[K] = T(0);
        } else {
            const int p = (2 * J - oy) * W + (2 * I - ox);
            auto r = [&](int o) { return sm[p + o] ? T(0) : sg[p + o]; };
            T v = T(0.25) * r(0);
            v += T(0.125) * (r(-1) + r(1) + r(-W) + r(W));
            v += T(0.0625) * (r(-W - 1) + r(-W + 1) + r(W - 1) + r(W + 1));
            // r-z: divided by the stencil's weighted volume (2J; 5/16 on the
            // axis, where the row below the axis is absent)
            if constexpr (CYL) v *= J == 0 ? T(3.2) : T(0.5) / T(J);
            Cc.g[K] = v;
        }
    }
    __syncthreads();  // the caller may reuse the shared tile
}

template <class T, int S, bool CYL>
__global__ void __launch_bounds__(kMgThreads) k_mg_down(LevelDev<T> F, LevelDev<T> Cc, T omega,
                                                        const double* __restrict__ g64) {
    extern __shared__ __align__(16) unsigned char smem[];
    pdl_wait();
    pdl_trigger();
    down_tile<T, S, CYL>(F, Cc, omega, blockIdx.x, blockIdx.y, smem, g64);
}

// RES (level 0 only): also r -= A e in FP64 on the core's free nodes (R->r64,
// the residual of phi before the cycle, becomes the residual after it);
// returns the tile's sum of r^2 (0 without RES).
template <class T, int S, bool CYL = false, bool PDL = false, bool RES = false>
__device__ double up_tile(const LevelDev<T>& F, const LevelDev<T>& Cc, T omega, double* __restrict__ phi, int tx,
                          int ty, unsigned char* smem, const ResArgs* R = nullptr) {
    constexpr int H = UpGeom<S, RES>::H, W = UpGeom<S, RES>::W, CW = UpGeom<S, RES>::CW;
    constexpr int CIT = (CW * CW + kMgThreads - 1) / kMgThreads;
    constexpr int OIT = (kMgTile * kMgTile + kMgThreads - 1) / kMgThreads;
    T* se = reinterpret_cast<T*>(smem);
    T* sg = se + W * W;
    T* sc = sg + W * W;
    T* srz = sc + CW * CW;  // r-z row coefficients (4 W values), only with CYL
    uint8_t* sm = reinterpret_cast<uint8_t*>(srz + (CYL ? 4 * W : 0));
    const int x0 = tx * kMgTile, y0 = ty * kMgTile;
    const int ox = x0 - H, oy = y0 - H;
    const int cox = ox >> 1, coy = oy >> 1;  // floor for negative origins
    const int tid = threadIdx.x;
    double pv[OIT], rv[RES ? OIT : 1];
#pragma unroll
    for (int it = 0; it < OIT; ++it) {
        const int q = it * kMgThreads + tid;
        const int i = x0 + q % kMgTile, j = y0 + q / kMgTile;
        const bool in = q < kMgTile * kMgTile && i < F.nx && j < F.ny;
        pv[it] = (phi && in) ? phi[long(j) * F.nx + i] : 0.0;
        if constexpr (RES) rv[it] = in ? R->r64[long(j) * F.nx + i] : 0.0;
    }
    tile_load<T, W, true, CYL>(F, ox, oy, se, sg, sm, srz);
    if constexpr (PDL) {
        pdl_wait();
        pdl_trigger();
    }
    T cv[CIT];
#pragma unroll
    for (int it = 0; it < CIT; ++it) {
        const int q = it * kMgThreads + tid;
        const int I = cox + q % CW, J = coy + q / CW;
        const bool in = q < CW * CW && I >= 0 && J >= 0 && I < Cc.nx && J < Cc.ny;
        cv[it] = in ? Cc.ec[long(J) * Cc.nx + I] : T(0);
    }
#pragma unroll
    for (int it = 0; it < CIT; ++it) {
        const int q = it * kMgThreads + tid;
        if (q < CW * CW) sc[q] = cv[it];
    }
    __syncthreads();
    // bilinear prolongation of the coarse correction, added on free nodes
    constexpr int IT = (W * W + kMgThreads - 1) / kMgThreads;
#pragma unroll
    for (int it = 0; it < IT; ++it) {
        const int q = it * kMgThreads + tid;
        if (q >= W * W) break;
        if (sm[q]) continue;
        const int i = ox + q % W, j = oy + q / W;
        const int c = ((j >> 1) - coy) * CW + ((i >> 1) - cox);
        T v;
        if (!(i & 1) && !(j & 1)) v = sc[c];
        else if ((i & 1) && !(j & 1)) v = T(0.5) * (sc[c] + sc[c + 1]);
        else if (!(i & 1) && (j & 1)) v = T(0.5) * (sc[c] + sc[c + CW]);
        else v = T(0.25) * (sc[c] + sc[c + 1] + sc[c + CW] + sc[c + CW + 1]);
        se[q] += v;
    }
    __syncthreads();
    const int par0 = (ox + oy) & 1;
#pragma unroll 1
    for (int s = 0; s < S; ++s)
#pragma unroll
        for (int color = 0; color < 2; ++color) {
            tile_half_sweep<T, W, CYL>(se, sg, sm, color ^ par0, F.cx, F.cy, F.inv_diag, omega, srz);
            __syncthreads();
        }
    double r2 = 0.0;
#pragma unroll
    for (int it = 0; it < OIT; ++it) {
        const int q = it * kMgThreads + tid;
        const int i = x0 + q % kMgTile, j = y0 + q / kMgTile;
        if (q >= kMgTile * kMgTile || i >= F.nx || j >= F.ny) continue;
        const long k = long(j) * F.nx + i;
        const int lq = (H + q / kMgTile) * W + H + q % kMgTile;
        const T v = se[lq];
        if (phi) phi[k] = pv[it] + double(v);
        else F.ec[k] = v;
        if constexpr (RES) {
            if (!sm[lq]) {
                // the change of the FP64 residual, f - A(phi + e) = r - A e, in
                // the association of k_mg_r0's Laplacian
                const double c = double(v), w = double(se[lq - 1]), e = double(se[lq + 1]);
                const double sv = double(se[lq - W]), nv = double(se[lq + W]);
                double lap;
                if constexpr (CYL)
                    lap = R->cx * ((w - c) + (e - c)) + R->rz0[4 * j] * (nv - c) + R->rz0[4 * j + 1] * (sv - c);
                else
                    lap = R->cx * ((w - c) + (e - c)) + R->cy * ((sv - c) + (nv - c));
                const double r = rv[it] - lap;
                R->r64[k] = r;
                r2 += r * r;
            }
        }
    }
    __syncthreads();  // the caller may reuse the shared tile
    return r2;
}

template <class T, int S, bool CYL>
__global__ void __launch_bounds__(kMgThreads) k_mg_up(LevelDev<T> F, LevelDev<T> Cc, T omega,
                                                      double* __restrict__ phi) {
    extern __shared__ __align__(16) unsigned char smem[];
    up_tile<T, S, CYL, true>(F, Cc, omega, phi, blockIdx.x, blockIdx.y, smem);
}

// ---- two levels in one launch --------------------------------------------------
//
// The down phases of a fine level F and the next level C in one launch, and
// the up phases of C and F in another (Cartesian levels above the direct
// solve).  A CTA owns a 32 x 32 tile of F, that is a 16 x 16 tile of C, and
// works both levels over halos wide enough that its C tile comes out exactly
// as the separate launches give it: F is smoothed over a halo of HF nodes so
// that F's residual is final where C's restriction over C's own smoothing halo
// reads it.  The redundant halo work runs on SMs that the separate launches of
// these small levels (25 and 9 CTAs at 513^2) leave idle.

template <int S>
struct Down2Geom {
    static constexpr int HC = 2 * S + 2, WC = kMgTile / 2 + 2 * HC;  // C: as DownGeom
    // F residual on 2HC + 1 nodes around the tile, e final one node further
    static constexpr int HF = 2 * HC + 2 + 2 * S, WF = kMgTile + 2 * HF;
};
template <int S>
struct Up2Geom {
    static constexpr int HF = 2 * S, WF = kMgTile + 2 * HF, CWF = WF / 2 + 2;  // F: as UpGeom
    // C final on F's prolongation window, smoothed over 2S more
    static constexpr int WC = CWF + 4 * S, CWC = WC / 2 + 2;
};

// Full-weighting restriction of the residual held in `r` (a W x W tile at
// (ox, oy) of the fine level, masked by `sm`) to coarse node (I, J).
template <class T, int W>
__device__ __forceinline__ T restrict_fw(const T* r, const uint8_t* sm, int I, int J, int ox, int oy) {
    const int p = (2 * J - oy) * W + (2 * I - ox);
    auto rv = [&](int o) { return sm[p + o] ? T(0) : r[p + o]; };
    T v = T(0.25) * rv(0);
    v += T(0.125) * (rv(-1) + rv(1) + rv(-W) + rv(W));
    v += T(0.0625) * (rv(-W - 1) + rv(-W + 1) + rv(W - 1) + rv(W + 1));
    return v;
}

// The residual g - A e in place of g on the interior of a W x W tile (each
// node reads only its own g).
template <class T, int W>
__device__ __forceinline__ void tile_residual(const T* se, T* sg, const uint8_t* sm, T cx, T cy) {
    constexpr int IT = (W * W + kMgThreads - 1) / kMgThreads;
#pragma unroll
    for (int it = 0; it < IT; ++it) {
        const int q = it * kMgThreads + int(threadIdx.x);
        if (q >= W * W) break;
        const int li = q % W, lj = q / W;
        if (li < 1 || lj < 1 || li > W - 2 || lj > W - 2 || sm[q]) continue;
        const T c = se[q];
        sg[q] = sg[q] - (cx * (se[q - 1] + se[q + 1] - T(2) * c) + cy * (se[q - W] + se[q + W] - T(2) * c));
    }
}

template <class T, int S>
__device__ void down2_tile(const LevelDev<T>& F, const LevelDev<T>& C, const LevelDev<T>& C2, T omega, int tx, int ty,
                           unsigned char* smem) {
    using G = Down2Geom<S>;
    constexpr int WF = G::WF, WC = G::WC, HF = G::HF, HC = G::HC;
    T* seF = reinterpret_cast<T*>(smem);
    T* sgF = seF + WF * WF;
    T* seC = sgF + WF * WF;
    T* sgC = seC + WC * WC;
    uint8_t* smF = reinterpret_cast<uint8_t*>(sgC + WC * WC);
    uint8_t* smC = smF + WF * WF;
    const int tid = threadIdx.x;
    const int x0 = tx * kMgTile, y0 = ty * kMgTile, ox = x0 - HF, oy = y0 - HF;
    const int cx0 = x0 / 2, cy0 = y0 / 2, cox = cx0 - HC, coy = cy0 - HC;
    // C's mask over its region (edges and outside the grid Dirichlet)
    constexpr int CIT = (WC * WC + kMgThreads - 1) / kMgThreads;
    uint8_t cm[CIT];
#pragma unroll
    for (int it = 0; it < CIT; ++it) {
        const int q = it * kMgThreads + tid;
        const int I = cox + q % WC, J = coy + q / WC;
        const bool in = q < WC * WC && I > 0 && J > 0 && I < C.nx - 1 && J < C.ny - 1;
        cm[it] = in ? C.mask[long(J) * C.nx + I] : uint8_t(1);
    }
    tile_load<T, WF, false, false>(F, ox, oy, seF, sgF, smF, nullptr);
    __syncthreads();
    const int parF = (ox + oy) & 1;
#pragma unroll 1
    for (int s = 0; s < S; ++s)
#pragma unroll
        for (int color = 0; color < 2; ++color) {
            tile_half_sweep<T, WF, false>(seF, sgF, smF, color ^ parF, F.cx, F.cy, F.inv_diag, omega, nullptr);
            __syncthreads();
        }
    for (int q = tid; q < kMgTile * kMgTile; q += kMgThreads) {
        const int i = x0 + q % kMgTile, j = y0 + q / kMgTile;
        if (i < F.nx && j < F.ny) F.e[long(j) * F.nx + i] = seF[(HF + q / kMgTile) * WF + HF + q % kMgTile];
    }
    tile_residual<T, WF>(seF, sgF, smF, F.cx, F.cy);
    __syncthreads();
    // C over its region: g restricted from F, e from zero; C's own tile of g
    // is kept for C's up phase
#pragma unroll
    for (int it = 0; it < CIT; ++it) {
        const int q = it * kMgThreads + tid;
        if (q >= WC * WC) break;
        const int LI = q % WC, LJ = q / WC, I = cox + LI, J = coy + LJ;
        const T g = cm[it] ? T(0) : restrict_fw<T, WF>(sgF, smF, I, J, ox, oy);
        smC[q] = cm[it];
        sgC[q] = g;
        seC[q] = T(0);
        if (LI >= HC && LJ >= HC && LI < HC + kMgTile / 2 && LJ < HC + kMgTile / 2 && I < C.nx && J < C.ny)
            C.g[long(J) * C.nx + I] = g;
    }
    __syncthreads();
    const int parC = (cox + coy) & 1;
#pragma unroll 1
    for (int s = 0; s < S; ++s)
#pragma unroll
        for (int color = 0; color < 2; ++color) {
            tile_half_sweep<T, WC, false>(seC, sgC, smC, color ^ parC, C.cx, C.cy, C.inv_diag, omega, nullptr);
            __syncthreads();
        }
    constexpr int hc = kMgTile / 2;
    for (int q = tid; q < hc * hc; q += kMgThreads) {
        const int I = cx0 + q % hc, J = cy0 + q / hc;
        if (I < C.nx && J < C.ny) C.e[long(J) * C.nx + I] = seC[(HC + q / hc) * WC + HC + q % hc];
    }
    tile_residual<T, WC>(seC, sgC, smC, C.cx, C.cy);
    __syncthreads();
    // C's residual restricted to the C2 nodes of this tile
    constexpr int h2 = kMgTile / 4;
    if (tid < h2 * h2) {
        const int I = cx0 / 2 + tid % h2, J = cy0 / 2 + tid / h2;
        if (I < C2.nx && J < C2.ny) {
            const long K = long(J) * C2.nx + I;
            const bool dir = I == 0 || J == 0 || I == C2.nx - 1 || J == C2.ny - 1 || C2.mask[K];
            C2.g[K] = dir ? T(0) : restrict_fw<T, WC>(sgC, smC, I, J, cox, coy);
        }
    }
}

template <class T, int S>
__global__ void __launch_bounds__(kMgThreads) k_mg_down2(LevelDev<T> F, LevelDev<T> C, LevelDev<T> C2, T omega) {
    extern __shared__ __align__(16) unsigned char smem[];
    pdl_wait();
    pdl_trigger();
    down2_tile<T, S>(F, C, C2, omega, blockIdx.x, blockIdx.y, smem);
}

// Bilinear prolongation of the coarse values `sc` (a CW-wide window at
// (cox, coy) of the coarse level) added onto the free nodes of a W x W tile
// at (ox, oy).
template <class T, int W, int CW>
__device__ __forceinline__ void tile_prolong(T* se, const uint8_t* sm, const T* sc, int ox, int oy, int cox, int coy) {
    constexpr int IT = (W * W + kMgThreads - 1) / kMgThreads;
#pragma unroll
    for (int it = 0; it < IT; ++it) {
        const int q = it * kMgThreads + int(threadIdx.x);
        if (q >= W * W) break;
        if (sm[q]) continue;
        const int i = ox + q % W, j = oy + q / W;
        const int c = ((j >> 1) - coy) * CW + ((i >> 1) - cox);
        T v;
        if (!(i & 1) && !(j & 1)) v = sc[c];
        else if ((i & 1) && !(j & 1)) v = T(0.5) * (sc[c] + sc[c + 1]);
        else if (!(i & 1) && (j & 1)) v = T(0.5) * (sc[c] + sc[c + CW]);
        else v = T(0.25) * (sc[c] + sc[c + 1] + sc[c + CW] + sc[c + CW + 1]);
        se[q] += v;
    }
}

template <class T, int S>
__device__ void up2_tile(const LevelDev<T>& F, const LevelDev<T>& C, const LevelDev<T>& C2, T omega, int tx, int ty,
                         unsigned char* smem) {
    using G = Up2Geom<S>;
    constexpr int WF = G::WF, HF = G::HF, WC = G::WC, CWC = G::CWC;
    T* seF = reinterpret_cast<T*>(smem);
    T* sgF = seF + WF * WF;
    T* seC = sgF + WF * WF;
    T* sgC = seC + WC * WC;
    T* sc2 = sgC + WC * WC;
    uint8_t* smF = reinterpret_cast<uint8_t*>(sc2 + CWC * CWC);
    uint8_t* smC = smF + WF * WF;
    const int tid = threadIdx.x;
    const int x0 = tx * kMgTile, y0 = ty * kMgTile, ox = x0 - HF, oy = y0 - HF;
    const int fcx = ox >> 1, fcy = oy >> 1;                    // F's prolongation window on C
    const int cox = fcx - 2 * S, coy = fcy - 2 * S;            // C's region
    const int c2x = cox >> 1, c2y = coy >> 1;                  // C's prolongation window on C2
    // every tile load is issued before the wait: F and C were written by the
    // down phase two launches back; only C2's correction follows the wait
    tile_load<T, WF, true, false>(F, ox, oy, seF, sgF, smF, nullptr);
    tile_load<T, WC, true, false>(C, cox, coy, seC, sgC, smC, nullptr);
    pdl_wait();
    pdl_trigger();
    for (int q = tid; q < CWC * CWC; q += kMgThreads) {
        const int I = c2x + q % CWC, J = c2y + q / CWC;
        sc2[q] = (I >= 0 && J >= 0 && I < C2.nx && J < C2.ny) ? C2.ec[long(J) * C2.nx + I] : T(0);
    }
    __syncthreads();
    tile_prolong<T, WC, CWC>(seC, smC, sc2, cox, coy, c2x, c2y);
    __syncthreads();
    const int parC = (cox + coy) & 1;
#pragma unroll 1
    for (int s = 0; s < S; ++s)
#pragma unroll
        for (int color = 0; color < 2; ++color) {
            tile_half_sweep<T, WC, false>(seC, sgC, smC, color ^ parC, C.cx, C.cy, C.inv_diag, omega, nullptr);
            __syncthreads();
        }
    // F's prolongation window lies 2S inside C's region
    tile_prolong<T, WF, WC>(seF, smF, seC, ox, oy, cox, coy);
    __syncthreads();
    const int parF = (ox + oy) & 1;
#pragma unroll 1
    for (int s = 0; s < S; ++s)
#pragma unroll
        for (int color = 0; color < 2; ++color) {
            tile_half_sweep<T, WF, false>(seF, sgF, smF, color ^ parF, F.cx, F.cy, F.inv_diag, omega, nullptr);
            __syncthreads();
        }
    for (int q = tid; q < kMgTile * kMgTile; q += kMgThreads) {
        const int i = x0 + q % kMgTile, j = y0 + q / kMgTile;
        if (i < F.nx && j < F.ny) F.ec[long(j) * F.nx + i] = seF[(HF + q / kMgTile) * WF + HF + q % kMgTile];
    }
}

template <class T, int S>
__global__ void __launch_bounds__(kMgThreads) k_mg_up2(LevelDev<T> F, LevelDev<T> C, LevelDev<T> C2, T omega) {
    extern __shared__ __align__(16) unsigned char smem[];
    up2_tile<T, S>(F, C, C2, omega, blockIdx.x, blockIdx.y, smem);
}

// Sums (a, b) over the grid: block partials into N.partial; the last block to
// finish adds them in a fixed order (the same decision on every run) and
// takes the loop decision: initial (first residual of a solve) records
// ||f||^2 = b and zeroes the cycle count, else counts a V-cycle; converged
// when ||r||^2 = a < tol2 ||f||^2; the WHILE node's condition (use_cond) is
// to go on while neither converged nor at max_cycles.
__device__ void norm_reduce_decide(double a, double b, const NormState& N, double tol2, int max_cycles, int initial,
                                   cudaGraphConditionalHandle cond, int use_cond) {
    __shared__ double ws[2][32];
    __shared__ bool last;
    const int t = threadIdx.y * blockDim.x + threadIdx.x, nt = blockDim.x * blockDim.y, nw = nt >> 5;
    const int lane = t & 31, w = t >> 5;
    a = warp_sum(a);
    b = warp_sum(b);
    if (lane == 0) {
        ws[0][w] = a;
        ws[1][w] = b;
    }
    __syncthreads();
    const int nb = gridDim.x * gridDim.y, bid = blockIdx.y * gridDim.x + blockIdx.x;
    if (w == 0) {
        // the block's sums: a warp reduction of the warps' sums (lane 0's value)
        double sa = lane < nw ? ws[0][lane] : 0.0, sb = lane < nw ? ws[1][lane] : 0.0;
        sa = warp_sum(sa);
        sb = warp_sum(sb);
        if (lane == 0) {
            N.partial[bid] = sa;
            N.partial[nb + bid] = sb;
            cuda::atomic_ref<unsigned, cuda::thread_scope_device> done(*N.done);
            last = done.fetch_add(1u, cuda::memory_order_acq_rel) == unsigned(nb - 1);
        }
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    // the solve's state and every block partial, loaded together
    int cyc = 0;
    long long tot = 0;
    double ref0 = 0.0;
    if (t == 0) {
        cyc = *reinterpret_cast<volatile int*>(N.cycles);
        tot = *reinterpret_cast<volatile long long*>(N.total);
        ref0 = *reinterpret_cast<volatile double*>(N.norms);
    }
    const volatile double* P = N.partial;
    double sa = 0.0, sb = 0.0;
    for (int q = t; q < nb; q += nt) {
        sa += P[q];
        sb += P[nb + q];
    }
    sa = warp_sum(sa);
    sb = warp_sum(sb);
    __syncthreads();
    if (lane == 0) {
        ws[0][w] = sa;
        ws[1][w] = sb;
    }
    __syncthreads();
    if (w == 0) {
        double r2 = lane < nw ? ws[0][lane] : 0.0, f2 = lane < nw ? ws[1][lane] : 0.0;
        r2 = warp_sum(r2);
        f2 = warp_sum(f2);
        if (lane == 0) {
            if (initial) {
                ref0 = f2;
                N.norms[0] = f2;
                cyc = 0;
            } else {
                cyc += 1;
                *N.total = tot + 1;
            }
            *N.cycles = cyc;
            N.norms[1] = r2;
            const int conv = r2 < tol2 * (ref0 > 0.0 ? ref0 : 1.0);
            *N.converged = conv;
            const int cont = !conv && cyc < max_cycles;
            if (use_cond) cudaGraphSetConditional(cond, cont ? 1u : 0u);
            *N.done = 0u;
        }
    }
}

// The finest up phase of a graph- or host-loop V-cycle fused with the FP64
// residual and the loop decision of k_mg_r0: phi += e, r -= A e on the core,
// then the norm of r.
template <class T, int S, bool CYL>
__global__ void __launch_bounds__(kMgThreads) k_mg_up_res(LevelDev<T> F, LevelDev<T> Cc, T omega,
                                                          double* __restrict__ phi, ResArgs R) {
    extern __shared__ __align__(16) unsigned char smem[];
    const double r2 = up_tile<T, S, CYL, true, true>(F, Cc, omega, phi, blockIdx.x, blockIdx.y, smem, &R);
    norm_reduce_decide(r2, 0.0, R.N, R.tol2, R.max_cycles, 0, R.cond, R.use_cond);
}

// Runtime sweep counts (the persistent kernel) dispatched to the instances.
template <class T>
__device__ void down_tile_n(int pre, const LevelDev<T>& F, const LevelDev<T>& Cc, T omega, int tx, int ty,
                            unsigned char* smem) {
    switch (pre) {
        case 1: down_tile<T, 1>(F, Cc, omega, tx, ty, smem); break;
        case 2: down_tile<T, 2>(F, Cc, omega, tx, ty, smem); break;
        case 3: down_tile<T, 3>(F, Cc, omega, tx, ty, smem); break;
        case 4: down_tile<T, 4>(F, Cc, omega, tx, ty, smem); break;
        case 5: down_tile<T, 5>(F, Cc, omega, tx, ty, smem); break;
        case 6: down_tile<T, 6>(F, Cc, omega, tx, ty, smem); break;
        case 7: down_tile<T, 7>(F, Cc, omega, tx, ty, smem); break;
        default: down_tile<T, 8>(F, Cc, omega, tx, ty, smem); break;
    }
}

template <class T>
__device__ void up_tile_n(int post, const LevelDev<T>& F, const LevelDev<T>& Cc, T omega, double* phi, int tx,
                          int ty, unsigned char* smem) {
    switch (post) {
        case 1: up_tile<T, 1>(F, Cc, omega, phi, tx, ty, smem); break;
        case 2: up_tile<T, 2>(F, Cc, omega, phi, tx, ty, smem); break;
        case 3: up_tile<T, 3>(F, Cc, omega, phi, tx, ty, smem); break;
        case 4: up_tile<T, 4>(F, Cc, omega, phi, tx, ty, smem); break;
        case 5: up_tile<T, 5>(F, Cc, omega, phi, tx, ty, smem); break;
        case 6: up_tile<T, 6>(F, Cc, omega, phi, tx, ty, smem); break;
        case 7: up_tile<T, 7>(F, Cc, omega, phi, tx, ty, smem); break;
        default: up_tile<T, 8>(F, Cc, omega, phi, tx, ty, smem); break;
    }
}

template <class T>
using DownKernel = void (*)(LevelDev<T>, LevelDev<T>, T, const double*);
template <class T>
using UpKernel = void (*)(LevelDev<T>, LevelDev<T>, T, double*);
template <class T>
using UpResKernel = void (*)(LevelDev<T>, LevelDev<T>, T, double*, ResArgs);

template <class T, bool CYL>
static DownKernel<T> down_kernel(int s) {
    static const DownKernel<T> k[kMgMaxSweeps + 1] = {
        nullptr,                 k_mg_down<T, 1, CYL>, k_mg_down<T, 2, CYL>, k_mg_down<T, 3, CYL>,
        k_mg_down<T, 4, CYL>,    k_mg_down<T, 5, CYL>, k_mg_down<T, 6, CYL>, k_mg_down<T, 7, CYL>,
        k_mg_down<T, 8, CYL>};
    return k[s];
}

template <class T, bool CYL>
static UpKernel<T> up_kernel(int s) {
    static const UpKernel<T> k[kMgMaxSweeps + 1] = {
        nullptr,              k_mg_up<T, 1, CYL>, k_mg_up<T, 2, CYL>, k_mg_up<T, 3, CYL>, k_mg_up<T, 4, CYL>,
        k_mg_up<T, 5, CYL>,   k_mg_up<T, 6, CYL>, k_mg_up<T, 7, CYL>, k_mg_up<T, 8, CYL>};
    return k[s];
}

template <class T, bool CYL>
static UpResKernel<T> up_res_kernel(int s) {
    static const UpResKernel<T> k[kMgMaxSweeps + 1] = {
        nullptr,                  k_mg_up_res<T, 1, CYL>, k_mg_up_res<T, 2, CYL>, k_mg_up_res<T, 3, CYL>,
        k_mg_up_res<T, 4, CYL>,   k_mg_up_res<T, 5, CYL>, k_mg_up_res<T, 6, CYL>, k_mg_up_res<T, 7, CYL>,
        k_mg_up_res<T, 8, CYL>};
    return k[s];
}

template <class T>
using Fused2Kernel = void (*)(LevelDev<T>, LevelDev<T>, LevelDev<T>, T);

template <class T>
static Fused2Kernel<T> down2_kernel(int s) {
    static const Fused2Kernel<T> k[kMgMaxSweeps + 1] = {
        nullptr,           k_mg_down2<T, 1>, k_mg_down2<T, 2>, k_mg_down2<T, 3>, k_mg_down2<T, 4>,
        k_mg_down2<T, 5>,  k_mg_down2<T, 6>, k_mg_down2<T, 7>, k_mg_down2<T, 8>};
    return k[s];
}

template <class T>
static Fused2Kernel<T> up2_kernel(int s) {
    static const Fused2Kernel<T> k[kMgMaxSweeps + 1] = {
        nullptr,         k_mg_up2<T, 1>, k_mg_up2<T, 2>, k_mg_up2<T, 3>, k_mg_up2<T, 4>,
        k_mg_up2<T, 5>,  k_mg_up2<T, 6>, k_mg_up2<T, 7>, k_mg_up2<T, 8>};
    return k[s];
}

template <class T>
static size_t down2_smem(int s) {
    const size_t HC = 2 * s + 2, WC = kMgTile / 2 + 2 * HC, HF = 2 * HC + 2 + 2 * s, WF = kMgTile + 2 * HF;
    return (WF * WF + WC * WC) * (2 * sizeof(T) + 1);
}

template <class T>
static size_t up2_smem(int s) {
    const size_t WF = kMgTile + 4 * s, CWF = WF / 2 + 2, WC = CWF + 4 * s, CWC = WC / 2 + 2;
    return (WF * WF + WC * WC) * (2 * sizeof(T) + 1) + CWC * CWC * sizeof(T);
}

template <class T>
static size_t down_smem(int s, bool cyl = false) {
    const size_t W = kMgTile + 2 * (2 * s + 2);
    return W * W * (2 * sizeof(T) + 1) + (cyl ? 4 * W * sizeof(T) : 0);
}

template <class T>
static size_t up_smem(int s, bool cyl = false, bool res = false) {
    const size_t W = kMgTile + 2 * (2 * s + (res ? 1 : 0)), CW = W / 2 + 2;
    return W * W * (2 * sizeof(T) + 1) + CW * CW * sizeof(T) + (cyl ? 4 * W * sizeof(T) : 0);
}

// ---- single-CTA V-cycle of the coarse levels --------------------------------------

// q / d for 0 <= q < 2^22 from a float reciprocal of d: (q + 1/2) / d lies at
// least 1/(2d) from an integer and the two float roundings move it by less.
__device__ __forceinline__ int div_small(int q, float inv_d) { return int((float(q) + 0.5f) * inv_d); }

template <class T, bool CYL>
__device__ void level_sweeps(T* se, const T* sg, const uint8_t* sm, const LevelDev<T>& L, T omega, int sweeps) {
    const int nx = L.nx, ny = L.ny;
    const int hx = (nx + 1) / 2;
    const float inv_hx = 1.0f / float(hx);
    for (int s = 0; s < sweeps; ++s)
        for (int color = 0; color < 2; ++color) {
            for (int q = threadIdx.x; q < hx * ny; q += blockDim.x) {
                const int j = div_small(q, inv_hx);
                const int i = 2 * (q - j * hx) + ((color + j) & 1);
                if (i >= nx) continue;
                const int p = j * nx + i;
                if (sm[p]) continue;
                T upd;
                if constexpr (CYL) {
                    // no row below the axis (its weight is zero)
                    const T s = j > 0 ? se[p - nx] : T(0);
                    const T* rc = L.rz + 4 * j;
                    upd = (L.cx * (se[p - 1] + se[p + 1]) + __ldg(rc) * se[p + nx] + __ldg(rc + 1) * s - sg[p]) *
                          __ldg(rc + 2);
                } else {
                    const T sum = L.cx * (se[p - 1] + se[p + 1]) + L.cy * (se[p - nx] + se[p + nx]);
                    upd = (sum - sg[p]) * L.inv_diag;
                }
                const T old = se[p];
                se[p] = old + omega * (upd - old);
            }
            __syncthreads();
        }
}

template <class T, bool CYL = false>
__device__ void coarse_vcycle(const CoarseDesc<T>& D, unsigned char* smem) {
    // level pointers into shared memory, from the descriptor's offsets (no
    // per-thread pointer arrays: they would live in local memory)
    auto E = [&](int l) { return reinterpret_cast<T*>(smem + D.off_e[l]); };
    auto Gs = [&](int l) { return reinterpret_cast<T*>(smem + D.off_g[l]); };
    auto M = [&](int l) { return smem + D.off_m[l]; };
    {
        uint4* s4 = reinterpret_cast<uint4*>(smem);
        const uint4 z = make_uint4(0u, 0u, 0u, 0u);
        for (int q = threadIdx.x; q < D.e_bytes / 16; q += blockDim.x) s4[q] = z;
        // every global read of the set in one batch: each thread issues its
        // loads before storing any of them
        const int n1 = D.m_vec, n2 = n1 + D.g_vec, n3 = n2 + D.a_vec, n4 = n3 + D.c_vec;
        for (int base = 0; base < n4; base += 4 * int(blockDim.x)) {
            uint4 v[4];
            int dst[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int q = base + u * int(blockDim.x) + int(threadIdx.x);
                dst[u] = -1;
                v[u] = z;
                if (q < n1) {
                    v[u] = __ldg(D.mimg + q);
                    dst[u] = D.m_off / 16 + q;
                } else if (q < n2) {
                    v[u] = D.g16[q - n1];
                    dst[u] = D.off_g[0] / 16 + (q - n1);
                } else if (q < n3) {
                    v[u] = __ldg(D.ainv16 + (q - n2));
                    dst[u] = D.a_off / 16 + (q - n2);
                } else if (q < n4) {
                    v[u] = __ldg(D.cidx16 + (q - n3));
                    dst[u] = D.c_off / 16 + (q - n3);
                }
            }
#pragma unroll
            for (int u = 0; u < 4; ++u)
                if (dst[u] >= 0) s4[dst[u]] = v[u];
        }
    }
    __syncthreads();
    const int last = D.nlev - 1;
    for (int l = 0; l < last; ++l) {
        const LevelDev<T>& L = D.lv[l];
        const LevelDev<T>& C = D.lv[l + 1];
        level_sweeps<T, CYL>(E(l), Gs(l), M(l), L, D.omega, D.pre);
        // restriction of the residual, evaluated on the fly: g of this level
        // must survive for the post-smoothing on the way back up
        const T* e = E(l);
        const T* g = Gs(l);
        const uint8_t* mk = M(l);
        const int nx = L.nx;
        const float inv_cnx = 1.0f / float(C.nx);
        for (int Q = threadIdx.x; Q < C.nx * C.ny; Q += blockDim.x) {
            if (M(l + 1)[Q]) {
                Gs(l + 1)[Q] = T(0);
                continue;
            }
            const int J = div_small(Q, inv_cnx), I = Q - J * C.nx;
            const int p = 2 * J * nx + 2 * I;
            if constexpr (CYL) {
                // volume-weighted full weighting; the axis row has no row below
                auto rrow = [&](int jf, int q) {
                    if (mk[q]) return T(0);
                    const T c = e[q];
                    const T* rc = L.rz + 4 * jf;
                    const T s = jf > 0 ? e[q - nx] : T(0);
                    const T lap = L.cx * (e[q - 1] + e[q + 1] - T(2) * c) + __ldg(rc) * (e[q + nx] - c) +
                                  __ldg(rc + 1) * (s - c);
                    return __ldg(rc + 3) * (g[q] - lap);
                };
                auto line = [&](int jf, int q) {
                    return T(0.5) * rrow(jf, q) + T(0.25) * (rrow(jf, q - 1) + rrow(jf, q + 1));
                };
                T v = T(0.5) * line(2 * J, p) + T(0.25) * line(2 * J + 1, p + nx);
                if (J > 0) v += T(0.25) * line(2 * J - 1, p - nx);
                Gs(l + 1)[Q] = v * (J == 0 ? T(3.2) : T(0.5) / T(J));
            } else {
                auto rr = [&](int o) {
                    const int q = p + o;
                    if (mk[q]) return T(0);
                    const T c = e[q];
                    return g[q] - (L.cx * (e[q - 1] + e[q + 1] - T(2) * c) + L.cy * (e[q - nx] + e[q + nx] - T(2) * c));
                };
                T v = T(0.25) * rr(0);
                v += T(0.125) * (rr(-1) + rr(1) + rr(-nx) + rr(nx));
                v += T(0.0625) * (rr(-nx - 1) + rr(-nx + 1) + rr(nx - 1) + rr(nx + 1));
                Gs(l + 1)[Q] = v;
            }
        }
        __syncthreads();
    }
    // dense direct solve on the coarsest level: one warp per row, lanes
    // striding over the row of the inverse (in shared memory when it fits)
    {
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
        const double* ainv = D.a_off >= 0 ? reinterpret_cast<const double*>(smem + D.a_off) : D.ainv;
        const int* cidx = D.a_off >= 0 ? reinterpret_cast<const int*>(smem + D.c_off) : D.cidx;
        for (int a = warp; a < D.nf; a += nw) {
            const double* row = ainv + long(a) * D.nf;
            double s = 0.0;
            for (int b = lane; b < D.nf; b += 32) s += row[b] * double(Gs(last)[cidx[b]]);
            s = warp_sum(s);
            if (lane == 0) E(last)[cidx[a]] = T(s);
        }
    }
    __syncthreads();
    for (int l = last - 1; l >= 0; --l) {
        const LevelDev<T>& L = D.lv[l];
        const LevelDev<T>& C = D.lv[l + 1];
        const float inv_nx = 1.0f / float(L.nx);
        for (int q = threadIdx.x; q < L.nx * L.ny; q += blockDim.x) {
            if (M(l)[q]) continue;
            const int j = div_small(q, inv_nx), i = q - j * L.nx;
            const int K = (j >> 1) * C.nx + (i >> 1);
            const T* ec = E(l + 1);
            T v;
            if (!(i & 1) && !(j & 1)) v = ec[K];
            else if ((i & 1) && !(j & 1)) v = T(0.5) * (ec[K] + ec[K + 1]);
            else if (!(i & 1) && (j & 1)) v = T(0.5) * (ec[K] + ec[K + C.nx]);
            else v = T(0.25) * (ec[K] + ec[K + 1] + ec[K + C.nx] + ec[K + C.nx + 1]);
            E(l)[q] += v;
        }
        __syncthreads();
        level_sweeps<T, CYL>(E(l), Gs(l), M(l), L, D.omega, D.post);
    }
    const LevelDev<T>& L0 = D.lv[0];
    for (int q = threadIdx.x; q < L0.nx * L0.ny; q += blockDim.x) {
        if (D.phi0) D.phi0[q] += double(E(0)[q]);
        else L0.e[q] = E(0)[q];
    }
    __syncthreads();
}

template <class T, bool CYL>
__global__ void __launch_bounds__(kCoarseThreads) k_mg_coarse(CoarseDesc<T> D) {
    extern __shared__ __align__(16) unsigned char smem[];
    pdl_wait();
    pdl_trigger();
    coarse_vcycle<T, CYL>(D, smem);
}

// ---- direct solve of the first coarse level ----------------------------------------
//
// The coarse end of a graph- or host-loop V-cycle: e = A^-1 g on the first
// level of at most 33^2 nodes, A^-1 the inverse of that level's operator on its
// free nodes (band LU at creation), instead of a V-cycle of the levels below
// in one CTA.  One warp per row of the inverse, kDirectRows rows per CTA;
// a warp's row never changes, so it is loaded before the wait, and only the
// gather of g follows it.

constexpr int kDirectMaxFree = 1120;              // free nodes of the level
constexpr int kDirectCols = kDirectMaxFree / 32;  // entries of a row per lane
constexpr int kDirectRows = 8;                    // rows (warps) per CTA
constexpr int kDirectGather = (kDirectMaxFree + kDirectRows * 32 - 1) / (kDirectRows * 32);

template <class T>
struct DirectDesc {
    const void* ainv;  // [n][n], row-major, FP64 (a64) or in the V-cycle's precision
    const int* idx;   // the free node of each row
    const int* zidx;  // the level's other nodes (their e is 0)
    const T* g;       // right-hand side (every node of the level)
    T* e;             // solution (every node of the level)
    int n, nz;
};

// MT: the precision of the inverse and of the products (double: the solve
// in FP64 whatever the V-cycle's precision).
template <class T, class MT>
__global__ void __launch_bounds__(kDirectRows * 32) k_mg_direct(DirectDesc<T> D) {
    __shared__ MT gs[kDirectMaxFree];
    const int lane = threadIdx.x & 31, row = blockIdx.x * kDirectRows + int(threadIdx.x >> 5);
    const MT* __restrict__ ainv = static_cast<const MT*>(D.ainv);
    MT a[kDirectCols];
#pragma unroll
    for (int u = 0; u < kDirectCols; ++u) {
        const int c = lane + 32 * u;
        a[u] = (row < D.n && c < D.n) ? __ldg(ainv + long(row) * D.n + c) : MT(0);
    }
    int gi[kDirectGather];
#pragma unroll
    for (int u = 0; u < kDirectGather; ++u) {
        const int k = int(threadIdx.x) + u * kDirectRows * 32;
        gi[u] = k < D.n ? __ldg(D.idx + k) : -1;
    }
    const int out = row < D.n ? __ldg(D.idx + row) : -1;
    pdl_wait();
    pdl_trigger();
#pragma unroll
    for (int u = 0; u < kDirectGather; ++u)
        if (gi[u] >= 0) gs[threadIdx.x + u * kDirectRows * 32] = MT(D.g[gi[u]]);
    if (blockIdx.x == 0)
        for (int k = threadIdx.x; k < D.nz; k += blockDim.x) D.e[D.zidx[k]] = T(0);
    __syncthreads();
    MT s = MT(0);
#pragma unroll
    for (int u = 0; u < kDirectCols; ++u) {
        const int c = lane + 32 * u;
        if (c < D.n) s += a[u] * gs[c];
    }
    const double t = warp_sum(double(s));
    if (lane == 0 && out >= 0) D.e[out] = T(t);
}

// ---- FP64 residual, norms and the loop decision -----------------------------------


constexpr int kR0Rows = 4;  // rows per thread of the residual kernel

// rz0: in r-z geometry the level-0 row coefficients in FP64 ({wN, wS, 1/diag,
// D} per row, as LevelDev::rz), else null.  The residual goes to g0 (the
// V-cycle's precision) and, when given, to r64 in FP64.
template <class T, bool CYL>
__global__ void __launch_bounds__(256) k_mg_r0(const double* __restrict__ phi, const double* __restrict__ f,
                                               const uint8_t* __restrict__ mask, int nx, int ny, double cx, double cy,
                                               T* __restrict__ g0, NormState N, double tol2, int max_cycles,
                                               int initial, cudaGraphConditionalHandle cond, int use_cond,
                                               const double* __restrict__ rz0, double* __restrict__ r64) {
    // a 32 x 8 block covers 32 x 32 nodes, four rows per thread, every load
    // of a thread issued before the first is used
    pdl_wait();
    pdl_trigger();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double r = 0.0, fv = 0.0;
    double pc[kR0Rows], pw[kR0Rows], pe[kR0Rows], ps[kR0Rows], pn[kR0Rows], pf[kR0Rows];
    bool use[kR0Rows];
#pragma unroll
    for (int u = 0; u < kR0Rows; ++u) {
        const int j = blockIdx.y * (blockDim.y * kR0Rows) + threadIdx.y + u * blockDim.y;
        const long k = long(j) * nx + i;
        const bool inner = i > 0 && (CYL ? j >= 0 : j > 0) && i < nx - 1 && j < ny - 1;
        use[u] = inner && !mask[k];
        pc[u] = inner ? phi[k] : 0.0;
        pw[u] = inner ? phi[k - 1] : 0.0;
        pe[u] = inner ? phi[k + 1] : 0.0;
        ps[u] = (inner && j > 0) ? phi[k - nx] : 0.0;
        pn[u] = inner ? phi[k + nx] : 0.0;
        pf[u] = inner ? f[k] : 0.0;
    }
#pragma unroll
    for (int u = 0; u < kR0Rows; ++u) {
        const int j = blockIdx.y * (blockDim.y * kR0Rows) + threadIdx.y + u * blockDim.y;
        if (i >= nx || j >= ny) continue;
        double ru = 0.0;
        if (use[u]) {
            const double c = pc[u];
            double lap;
            if constexpr (CYL)
                lap = cx * ((pw[u] - c) + (pe[u] - c)) + rz0[4 * j] * (pn[u] - c) + rz0[4 * j + 1] * (ps[u] - c);
            else
                lap = cx * ((pw[u] - c) + (pe[u] - c)) + cy * ((ps[u] - c) + (pn[u] - c));
            ru = pf[u] - lap;
            fv += pf[u] * pf[u];
        }
        r += ru * ru;
        g0[long(j) * nx + i] = T(ru);
        if (r64) r64[long(j) * nx + i] = ru;
    }
    norm_reduce_decide(r, fv, N, tol2, max_cycles, initial, cond, use_cond);
}

// ---- persistent cooperative solve -------------------------------------------------

struct GridBar {
    unsigned count;
    unsigned gen;
};

// Grid-wide barrier of a cooperative launch; false (and *error set) if it
// did not complete within `polls` polls (kBarrierPolls unless the solver's
// wait limit was changed).  On a timeout the block also records, in
// error[1..5], the barrier's sequence number, its block index and the counter
// state it saw.
__device__ __forceinline__ bool grid_barrier(GridBar* b, int* error, int seq, unsigned long long polls) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        cuda::atomic_ref<unsigned, cuda::thread_scope_device> gen(b->gen), cnt(b->count);
        const unsigned g = gen.load(cuda::memory_order_acquire);
        const unsigned nb = gridDim.x * gridDim.y;
        int ok = 1;
        __threadfence();
        if (cnt.fetch_add(1u, cuda::memory_order_acq_rel) == nb - 1u) {
            cnt.store(0u, cuda::memory_order_relaxed);
            gen.fetch_add(1u, cuda::memory_order_release);
        } else {
            unsigned long long k = 0;
            while (gen.load(cuda::memory_order_acquire) == g) {
                if (++k > polls) {
                    ok = 0;
                    if (atomicExch(error, 1) == 0) {
                        error[1] = seq;
                        error[2] = int(blockIdx.x);
                        error[3] = int(cnt.load(cuda::memory_order_relaxed));
                        error[4] = int(gen.load(cuda::memory_order_relaxed));
                        error[5] = int(g);
                    }
                    break;
                }
            }
        }
        __threadfence();
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

template <class T>
struct SolveDesc {
    int L, Lp;  // levels; first level handled by the single-block coarse phase
    LevelDev<T> lv[kMgMaxLevels];
    CoarseDesc<T> coarse;  // levels Lp..L-1
    const double* f;
    double* phi;
    int nx, ny;
    double cx, cy;
    NormState N;
    double tol2;
    int max_cycles;
    T omega;
    int pre, post;
    GridBar* bar;
    int* error;
    unsigned long long polls;  // grid-barrier wait limit
};

// FP64 residual of phi on level 0 (written to g0 as the next V-cycle's
// right-hand side) and its norm, identical in every block: the block partials
// are summed after a grid barrier in a fixed order.
template <class T>
__device__ bool r0_phase(const SolveDesc<T>& S, double& r2, double& f2, int& seq) {
    const int tnx = (S.nx + kMgTile - 1) / kMgTile, tny = (S.ny + kMgTile - 1) / kMgTile;
    const double* __restrict__ phi = S.phi;
    const uint8_t* __restrict__ mask = S.lv[0].mask;
    const int nx = S.nx, ny = S.ny;
    double a = 0.0, b = 0.0;
    for (int t = blockIdx.x; t < tnx * tny; t += gridDim.x) {
        const int x0 = (t % tnx) * kMgTile, y0 = (t / tnx) * kMgTile;
        for (int q = threadIdx.x; q < kMgTile * kMgTile; q += blockDim.x) {
            const int i = x0 + q % kMgTile, j = y0 + q / kMgTile;
            if (i >= nx || j >= ny) continue;
            const long k = long(j) * nx + i;
            double r = 0.0;
            if (i > 0 && j > 0 && i < nx - 1 && j < ny - 1 && !mask[k]) {
                const double c = phi[k];
                const double lap = S.cx * ((phi[k - 1] - c) + (phi[k + 1] - c)) +
                                   S.cy * ((phi[k - nx] - c) + (phi[k + nx] - c));
                const double fv = S.f[k];
                r = fv - lap;
                b += fv * fv;
            }
            S.lv[0].g[k] = T(r);
            a += r * r;
        }
    }
    __shared__ double ws[2][kMgThreads / 32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    a = warp_sum(a);
    b = warp_sum(b);
    if (lane == 0) {
        ws[0][w] = a;
        ws[1][w] = b;
    }
    __syncthreads();
    const int nb = gridDim.x;
    if (threadIdx.x == 0) {
        double sa = 0.0, sb = 0.0;
        for (int q = 0; q < nw; ++q) {
            sa += ws[0][q];
            sb += ws[1][q];
        }
        S.N.partial[blockIdx.x] = sa;
        S.N.partial[nb + blockIdx.x] = sb;
    }
    if (!grid_barrier(S.bar, S.error, seq++, S.polls)) return false;
    const volatile double* P = S.N.partial;
    double sa = 0.0, sb = 0.0;
    for (int q = threadIdx.x; q < nb; q += blockDim.x) {
        sa += P[q];
        sb += P[nb + q];
    }
    sa = warp_sum(sa);
    sb = warp_sum(sb);
    __syncthreads();
    if (lane == 0) {
        ws[0][w] = sa;
        ws[1][w] = sb;
    }
    __syncthreads();
    r2 = 0.0;
    f2 = 0.0;
    for (int q = 0; q < nw; ++q) {
        r2 += ws[0][q];
        f2 += ws[1][q];
    }
    __syncthreads();
    return true;
}

// The whole solve in one cooperative launch: residual, then V-cycles until
// converged or max_cycles, each phase separated by a grid barrier.
template <class T>
__global__ void __launch_bounds__(kMgThreads) k_mg_solve(SolveDesc<T> S) {
    extern __shared__ __align__(16) unsigned char smem[];
    double r2 = 0.0, f2 = 0.0, dummy = 0.0;
    int seq = 0;
    if (!r0_phase(S, r2, f2, seq)) return;
    const double ref = f2 > 0.0 ? f2 : 1.0;
    int cycles = 0;
    bool conv = r2 < S.tol2 * ref;
    while (!conv && cycles < S.max_cycles) {
        for (int l = 0; l < S.Lp; ++l) {
            const int tnx = (S.lv[l].nx + kMgTile - 1) / kMgTile, tny = (S.lv[l].ny + kMgTile - 1) / kMgTile;
            for (int t = blockIdx.x; t < tnx * tny; t += gridDim.x)
                down_tile_n(S.pre, S.lv[l], S.lv[l + 1], S.omega, t % tnx, t / tnx, smem);
            if (!grid_barrier(S.bar, S.error, seq++, S.polls)) return;
        }
        if (blockIdx.x == 0) coarse_vcycle(S.coarse, smem);
        if (!grid_barrier(S.bar, S.error, seq++, S.polls)) return;
        for (int l = S.Lp - 1; l >= 0; --l) {
            const int tnx = (S.lv[l].nx + kMgTile - 1) / kMgTile, tny = (S.lv[l].ny + kMgTile - 1) / kMgTile;
            for (int t = blockIdx.x; t < tnx * tny; t += gridDim.x)
                up_tile_n(S.post, S.lv[l], S.lv[l + 1], S.omega, l == 0 ? S.phi : nullptr, t % tnx, t / tnx, smem);
            if (!grid_barrier(S.bar, S.error, seq++, S.polls)) return;
        }
        if (!r0_phase(S, r2, dummy, seq)) return;
        ++cycles;
        conv = r2 < S.tol2 * ref;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        S.N.norms[0] = f2;
        S.N.norms[1] = r2;
        *S.N.cycles = cycles;
        *S.N.converged = conv ? 1 : 0;
        *S.N.total += cycles;
    }
}

// ---- cluster-resident solve ---------------------------------------------------------
//
// The whole solve in one launch of a single thread-block cluster (16 CTAs of
// 1024 threads where the device allows, else 8): every level of more than
// 33^2 nodes is cut into row bands, one per CTA; a phase loads the CTA's band
// with its halo rows into shared memory, works there and writes the band
// back; the cluster barrier (a hardware barrier, no polling) separates the
// phases.  CTA 0 alone runs the levels of at most 33^2 nodes.  The FP64
// residual norm is summed over the CTAs through distributed shared memory,
// in rank order, so every CTA takes the same loop decision.

constexpr int kClusterThreads = 1024;
constexpr int kBandBatch = 4;  // global loads a thread issues before the first is used

struct ClusterDesc {
    int L, Lb;  // levels; [0, Lb) in bands over the cluster, [Lb, L) in CTA 0
    int Lt;     // tail: one V-cycle of levels [Lt, L), no residual and no loop (PIC_MG_HYBRID)
    int tail;
    LevelDev<float> lv[kMgMaxLevels];
    CoarseDesc<float> coarse;
    const double* f;
    double* phi;
    int nx, ny;
    double cx, cy;
    NormState N;
    double tol2;
    int max_cycles;
    float omega;
    int pre, post;
};

// Rows [a, b) of an n-row level that CTA r of `parts` owns.
__device__ __host__ __forceinline__ void band_rows(int n, int parts, int r, int& a, int& b) {
    const int per = (n + parts - 1) / parts;
    a = n < r * per ? n : r * per;
    b = n < a + per ? n : a + per;
}

// Loads rows [j0, j0 + R) of level L (full width) into the shared band:
// mask (edges, electrodes and rows outside the grid are Dirichlet), g, and e
// (zero, or the stored correction on free nodes).
__device__ void band_load(const LevelDev<float>& L, int j0, int R, float* __restrict__ se, float* __restrict__ sg,
                          uint8_t* __restrict__ sm, bool load_e) {
    const int nx = L.nx, N = R * nx, T = blockDim.x;
    const float inv = 1.0f / float(nx);
    for (int base = 0; base < N; base += kBandBatch * T) {
        uint8_t m[kBandBatch];
        float g[kBandBatch], e[kBandBatch];
#pragma unroll
        for (int u = 0; u < kBandBatch; ++u) {
            const int q = base + u * T + int(threadIdx.x);
            const int lr = div_small(q, inv), i = q - lr * nx, j = j0 + lr;
            const bool in = q < N && j >= 0 && j < L.ny;
            const long k = long(j) * nx + i;
            m[u] = in ? L.mask[k] : uint8_t(1);
            g[u] = in ? L.g[k] : 0.0f;
            e[u] = (load_e && in) ? L.e[k] : 0.0f;
        }
#pragma unroll
        for (int u = 0; u < kBandBatch; ++u) {
            const int q = base + u * T + int(threadIdx.x);
            if (q >= N) break;
            const int lr = div_small(q, inv), i = q - lr * nx, j = j0 + lr;
            const bool fr = i > 0 && j > 0 && i < nx - 1 && j < L.ny - 1 && !m[u];
            sm[q] = fr ? 0 : 1;
            sg[q] = g[u];
            se[q] = fr ? e[u] : 0.0f;
        }
    }
}

// One red (color 0: (i + j) even) or black half-sweep over the band's rows
// 1 .. R-2 (j0: global row of band row 0).
__device__ void band_half_sweep(float* __restrict__ se, const float* __restrict__ sg, const uint8_t* __restrict__ sm,
                                const LevelDev<float>& L, int j0, int R, int color, float omega) {
    const int nx = L.nx, hx = (nx + 1) / 2, T = blockDim.x;
    const float inv = 1.0f / float(hx);
    for (int q = threadIdx.x; q < R * hx; q += T) {
        const int lr = div_small(q, inv);
        const int i = 2 * (q - lr * hx) + ((color + j0 + lr) & 1);
        if (lr < 1 || lr > R - 2 || i >= nx) continue;
        const int p = lr * nx + i;
        if (sm[p]) continue;
        const float s = L.cx * (se[p - 1] + se[p + 1]) + L.cy * (se[p - nx] + se[p + nx]);
        const float upd = (s - sg[p]) * L.inv_diag;
        const float old = se[p];
        se[p] = old + omega * (upd - old);
    }
}

__device__ void band_sweeps(float* se, const float* sg, const uint8_t* sm, const LevelDev<float>& L, int j0, int R,
                            int sweeps, float omega) {
    for (int s = 0; s < sweeps; ++s)
        for (int color = 0; color < 2; ++color) {
            band_half_sweep(se, sg, sm, L, j0, R, color, omega);
            __syncthreads();
        }
}

// Pre-smoothing of level F on this CTA's band, the residual, and its
// full-weighting restriction onto the coarse rows J with 2J in the band.
__device__ void band_down(const LevelDev<float>& F, const LevelDev<float>& Cc, float omega, int pre, int rank,
                          int parts, unsigned char* smem) {
    int fa, fb;
    band_rows(F.ny, parts, rank, fa, fb);
    const int H = 2 * pre + 2, j0 = fa - H, R = (fb - fa) + 2 * H, nx = F.nx, T = blockDim.x;
    float* se = reinterpret_cast<float*>(smem);
    float* sg = se + R * nx;
    uint8_t* sm = reinterpret_cast<uint8_t*>(sg + R * nx);
    if (fa < fb) {
        band_load(F, j0, R, se, sg, sm, false);
        __syncthreads();
        band_sweeps(se, sg, sm, F, j0, R, pre, omega);
        // the smoothed correction of the band's own rows
        for (int q = threadIdx.x; q < (fb - fa) * nx; q += T) F.e[long(fa) * nx + q] = se[H * nx + q];
        // residual in place of g (each node reads only its own g)
        const float inv = 1.0f / float(nx);
        for (int q = threadIdx.x; q < R * nx; q += T) {
            const int lr = div_small(q, inv);
            if (lr < 1 || lr > R - 2 || sm[q]) continue;
            const float c = se[q];
            const float lap = F.cx * (se[q - 1] + se[q + 1] - 2.0f * c) + F.cy * (se[q - nx] + se[q + nx] - 2.0f * c);
            sg[q] = sg[q] - lap;
        }
        __syncthreads();
        const int Ja = (fa + 1) / 2, Jb = min(Cc.ny, (fb + 1) / 2);
        const int cnx = Cc.nx;
        const float cinv = 1.0f / float(cnx);
        for (int q = threadIdx.x; q < (Jb - Ja) * cnx; q += T) {
            const int dJ = div_small(q, cinv), I = q - dJ * cnx, J = Ja + dJ;
            const long K = long(J) * cnx + I;
            if (I == 0 || J == 0 || I == cnx - 1 || J == Cc.ny - 1 || Cc.mask[K]) {
                Cc.g[K] = 0.0f;
                continue;
            }
            const int p = (2 * J - j0) * nx + 2 * I;
            auto r = [&](int o) { return sm[p + o] ? 0.0f : sg[p + o]; };
            float v = 0.25f * r(0);
            v += 0.125f * (r(-1) + r(1) + r(-nx) + r(nx));
            v += 0.0625f * (r(-nx - 1) + r(-nx + 1) + r(nx - 1) + r(nx + 1));
            Cc.g[K] = v;
        }
    }
    __syncthreads();
}

// Prolongation-add of the coarse correction and post-smoothing on this CTA's
// band of level F; on level 0 (phi given) phi += e instead of storing e.
__device__ void band_up(const LevelDev<float>& F, const LevelDev<float>& Cc, float omega, int post, double* phi,
                        int rank, int parts, unsigned char* smem) {
    int fa, fb;
    band_rows(F.ny, parts, rank, fa, fb);
    const int H = 2 * post, j0 = fa - H, R = (fb - fa) + 2 * H, nx = F.nx, T = blockDim.x;
    const int cj0 = j0 >> 1, CR = ((j0 + R - 1) >> 1) + 2 - cj0, cnx = Cc.nx;
    float* se = reinterpret_cast<float*>(smem);
    float* sg = se + R * nx;
    float* sc = sg + R * nx;
    uint8_t* sm = reinterpret_cast<uint8_t*>(sc + CR * cnx);
    if (fa < fb) {
        // the coarse rows the band's prolongation reads
        const float cinv = 1.0f / float(cnx);
        for (int base = 0; base < CR * cnx; base += kBandBatch * T) {
            float v[kBandBatch];
#pragma unroll
            for (int u = 0; u < kBandBatch; ++u) {
                const int q = base + u * T + int(threadIdx.x);
                const int dJ = div_small(q, cinv), I = q - dJ * cnx, J = cj0 + dJ;
                const bool in = q < CR * cnx && J >= 0 && J < Cc.ny;
                v[u] = in ? Cc.ec[long(J) * cnx + I] : 0.0f;
            }
#pragma unroll
            for (int u = 0; u < kBandBatch; ++u) {
                const int q = base + u * T + int(threadIdx.x);
                if (q < CR * cnx) sc[q] = v[u];
            }
        }
        band_load(F, j0, R, se, sg, sm, true);
        __syncthreads();
        const float inv = 1.0f / float(nx);
        for (int q = threadIdx.x; q < R * nx; q += T) {
            if (sm[q]) continue;
            const int lr = div_small(q, inv), i = q - lr * nx, j = j0 + lr;
            const int c = ((j >> 1) - cj0) * cnx + (i >> 1);
            float v;
            if (!(i & 1) && !(j & 1)) v = sc[c];
            else if ((i & 1) && !(j & 1)) v = 0.5f * (sc[c] + sc[c + 1]);
            else if (!(i & 1) && (j & 1)) v = 0.5f * (sc[c] + sc[c + cnx]);
            else v = 0.25f * (sc[c] + sc[c + 1] + sc[c + cnx] + sc[c + cnx + 1]);
            se[q] += v;
        }
        __syncthreads();
        band_sweeps(se, sg, sm, F, j0, R, post, omega);
        const int N = (fb - fa) * nx;
        if (phi) {
            for (int base = 0; base < N; base += kBandBatch * T) {
                double pv[kBandBatch];
#pragma unroll
                for (int u = 0; u < kBandBatch; ++u) {
                    const int q = base + u * T + int(threadIdx.x);
                    pv[u] = q < N ? phi[long(fa) * nx + q] : 0.0;
                }
#pragma unroll
                for (int u = 0; u < kBandBatch; ++u) {
                    const int q = base + u * T + int(threadIdx.x);
                    if (q < N) phi[long(fa) * nx + q] = pv[u] + double(se[H * nx + q]);
                }
            }
        } else {
            for (int q = threadIdx.x; q < N; q += T) F.ec[long(fa) * nx + q] = se[H * nx + q];
        }
    }
    __syncthreads();
}

// FP64 residual of phi on this CTA's rows of level 0 (written to g0 as the
// next V-cycle's right-hand side) and the norms summed over the cluster in
// rank order.
__device__ void cluster_r0(const ClusterDesc& S, int rank, int parts, double* s_part, double& r2, double& f2) {
    namespace cg = cooperative_groups;
    int fa, fb;
    band_rows(S.ny, parts, rank, fa, fb);
    const int nx = S.nx, ny = S.ny, T = blockDim.x;
    const double* __restrict__ phi = S.phi;
    const uint8_t* __restrict__ mask = S.lv[0].mask;
    double a = 0.0, b = 0.0;
    const int N = (fb - fa) * nx;
    const float inv = 1.0f / float(nx);
    for (int base = 0; base < N; base += 4 * T) {
        double rv[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int q = base + u * T + int(threadIdx.x);
            rv[u] = 0.0;
            if (q >= N) continue;
            const long k = long(fa) * nx + q;
            const int lr = div_small(q, inv), i = q - lr * nx, j = fa + lr;
            if (i > 0 && j > 0 && i < nx - 1 && j < ny - 1 && !mask[k]) {
                const double c = phi[k];
                const double lap =
                    S.cx * ((phi[k - 1] - c) + (phi[k + 1] - c)) + S.cy * ((phi[k - nx] - c) + (phi[k + nx] - c));
                const double fv = S.f[k];
                rv[u] = fv - lap;
                b += fv * fv;
            }
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int q = base + u * T + int(threadIdx.x);
            if (q < N) S.lv[0].g[long(fa) * nx + q] = float(rv[u]);
            a += rv[u] * rv[u];
        }
    }
    __shared__ double ws[2][kClusterThreads / 32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    a = warp_sum(a);
    b = warp_sum(b);
    if (lane == 0) {
        ws[0][w] = a;
        ws[1][w] = b;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double sa = 0.0, sb = 0.0;
        for (int q = 0; q < nw; ++q) {
            sa += ws[0][q];
            sb += ws[1][q];
        }
        s_part[0] = sa;
        s_part[1] = sb;
    }
    cg::cluster_group cl = cg::this_cluster();
    cl.sync();
    double sa = 0.0, sb = 0.0;
    for (int r = 0; r < parts; ++r) {
        const double* p = cl.map_shared_rank(s_part, r);
        sa += p[0];
        sb += p[1];
    }
    r2 = sa;
    f2 = sb;
}

__global__ void __launch_bounds__(kClusterThreads, 1) k_mg_cluster(ClusterDesc S) {
    namespace cg = cooperative_groups;
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ double s_part[2];
    cg::cluster_group cl = cg::this_cluster();
    const int rank = int(cl.block_rank()), parts = int(cl.num_blocks());
    if (S.tail) {
        // the coarse end of a V-cycle whose finer levels run in tile kernels:
        // g of level Lt in, the correction of level Lt (its ec) out
        for (int l = S.Lt; l < S.Lb; ++l) {
            band_down(S.lv[l], S.lv[l + 1], S.omega, S.pre, rank, parts, smem);
            cl.sync();
        }
        if (rank == 0) coarse_vcycle(S.coarse, smem);
        cl.sync();
        for (int l = S.Lb - 1; l >= S.Lt; --l) {
            band_up(S.lv[l], S.lv[l + 1], S.omega, S.post, nullptr, rank, parts, smem);
            cl.sync();
        }
        return;
    }
    double r2 = 0.0, f2 = 0.0, dummy = 0.0;
    cluster_r0(S, rank, parts, s_part, r2, f2);
    const double ref = f2 > 0.0 ? f2 : 1.0;
    int cycles = 0;
    bool conv = r2 < S.tol2 * ref;
    while (!conv && cycles < S.max_cycles) {
        for (int l = 0; l < S.Lb; ++l) {
            band_down(S.lv[l], S.lv[l + 1], S.omega, S.pre, rank, parts, smem);
            cl.sync();
        }
        if (rank == 0) coarse_vcycle(S.coarse, smem);
        cl.sync();
        for (int l = S.Lb - 1; l >= 0; --l) {
            band_up(S.lv[l], S.lv[l + 1], S.omega, S.post, l == 0 ? S.phi : nullptr, rank, parts, smem);
            cl.sync();
        }
        cluster_r0(S, rank, parts, s_part, r2, dummy);
        ++cycles;
        conv = r2 < S.tol2 * ref;
    }
    if (rank == 0 && threadIdx.x == 0) {
        S.N.norms[0] = f2;
        S.N.norms[1] = r2;
        *S.N.cycles = cycles;
        *S.N.converged = conv ? 1 : 0;
        *S.N.total += cycles;
    }
    // no CTA may exit while another can still read its shared memory
    cl.sync();
}

// ---- host object ---------------------------------------------------------------

// Shared-memory layout of a set of coarse levels (see CoarseDesc).
struct CoarseLayout {
    int first = 0;
    int off_e[kMgMaxCoarseLevels]{}, off_g[kMgMaxCoarseLevels]{}, off_m[kMgMaxCoarseLevels]{};
    int e_bytes = 0, m_off = 0, a_off = -1, c_off = -1;
    int m_vec = 0, g_vec = 0, a_vec = 0, c_vec = 0;
    size_t smem = 0;
    uint4* mimg = nullptr;
};

struct DstPlan;
int dst_create(int nx, int ny, double dx, double dy, DstPlan** out);
void dst_destroy(DstPlan* P);
int dst_launch(DstPlan* P, double* phi, const double* f, cudaStream_t st);

struct MgImpl {
    int precision = PIC_MG_MIXED;
    int nx = 0, ny = 0, L = 0, Lc = 0;
    double dx = 0, dy = 0;
    bool rz = false;          // r-z geometry (PIC_GEOM_RZ)
    double* rz0 = nullptr;    // level-0 row coefficients in FP64 (r-z)
    DstPlan* dst = nullptr;   // PIC_MG_DST: the sine-transform solve
    bool hybrid = false;      // PIC_MG_HYBRID: levels [Lt, L) in one cluster launch per cycle
    int Lt = 0;
    pic_mg_options o{};
    std::vector<LevelDev<float>> lf;
    std::vector<LevelDev<double>> ld;
    std::vector<void*> allocs;
    double* ainv = nullptr;
    int* cidx = nullptr;
    int nfree_c = 0;
    // direct solve of level Lc (graph and host loops; else the coarse kernel)
    bool direct = false;
    void* dinv = nullptr;  // [dn][dn], FP64 unless a mixed V-cycle asked for FP32 (pic_mg_options.coarse_fp32)
    bool dinv64 = true;
    int* didx = nullptr;   // dn free nodes, then dnz others
    int dn = 0, dnz = 0;
    double* r64 = nullptr;  // FP64 residual of phi between the cycles of a graph- or host-loop solve
    bool fuse2 = false;     // levels Lc-2 and Lc-1 in one down and one up launch (k_mg_down2, k_mg_up2)
    NormState N{};
    dim3 blk0{32, 8}, grd0;
    CoarseLayout cl[2];  // the coarse kernel's levels (from Lc) and the persistent/cluster ones (from Lp)
    long long launches = 0;  // kernels executed by solves
    int body_launches = 0;   // kernels per V-cycle (graph and host loops)
    // persistent cooperative solve
    int Lp = 0;
    size_t solve_smem = 0;
    int solve_grid = 0;
    // cluster-resident solve
    bool cluster_ok = false;
    int cluster_size = 0;
    size_t cluster_smem = 0;
    GridBar* bar = nullptr;
    int* error = nullptr;
    unsigned long long wait_polls = kBarrierPolls;  // grid-barrier wait limit of the persistent solve
    cudaStream_t side = nullptr;
    cudaStream_t cap = nullptr;
    // cached solve graph
    cudaGraphExec_t exec = nullptr;
    double* g_phi = nullptr;
    const double* g_f = nullptr;
    double g_tol = 0;
    int g_max = -1;
    int g_min = -1;
};

}  // namespace pic

struct pic_mg {
    pic::MgImpl m;
};

namespace pic {

// Row coefficients of the r-z operator on a level with spacings hx (axial)
// and hy (radial), row j at radius j*hy:
//   (1/r) d/dr (r dphi/dr) ~ [(1 + 1/2j) phi_{j+1} + (1 - 1/2j) phi_{j-1} - 2 phi_j] / hy^2,
// and on the axis, by symmetry, 2 d2phi/dr2 ~ 4 (phi_1 - phi_0) / hy^2.
// Per row {wN, wS, 1/diag, D}; D is the row's volume weight (2 pi r dr per
// 2 pi hy^2: j, and 1/8 for the axis control volume of radius hy/2).
static std::vector<double> rz_rows(int ny, double hx, double hy) {
    const double cx = 1.0 / (hx * hx), cy = 1.0 / (hy * hy);
    std::vector<double> r(size_t(4) * ny);
    for (int j = 0; j < ny; ++j) {
        const double wn = j == 0 ? 4.0 * cy : cy * (1.0 + 0.5 / j);
        const double ws = j == 0 ? 0.0 : cy * (1.0 - 0.5 / j);
        r[4 * j] = wn;
        r[4 * j + 1] = ws;
        r[4 * j + 2] = 1.0 / (2.0 * cx + wn + ws);
        r[4 * j + 3] = j == 0 ? 0.125 : double(j);
    }
    return r;
}

template <class T>
static int alloc_levels(MgImpl& M, std::vector<LevelDev<T>>& lv, const std::vector<std::vector<uint8_t>>& masks,
                        const std::vector<int>& nxs, const std::vector<int>& nys) {
    for (int l = 0; l < M.L; ++l) {
        LevelDev<T> v{};
        v.nx = nxs[l];
        v.ny = nys[l];
        const double hx = M.dx * double(1 << l), hy = M.dy * double(1 << l);
        const double cx = 1.0 / (hx * hx), cy = 1.0 / (hy * hy);
        v.cx = T(cx);
        v.cy = T(cy);
        v.inv_diag = T(1.0 / (2.0 * (cx + cy)));
        const size_t G = size_t(v.nx) * v.ny;
        uint8_t* mk = nullptr;
        PIC_CUDA(cudaMalloc(&mk, G));
        M.allocs.push_back(mk);
        PIC_CUDA(cudaMemcpy(mk, masks[l].data(), G, cudaMemcpyHostToDevice));
        v.mask = mk;
        // padded to 16 bytes: the coarse kernel reads g in 16-byte words
        const size_t bytes = (G * sizeof(T) + 15) / 16 * 16;
        PIC_CUDA(cudaMalloc(&v.e, bytes));
        M.allocs.push_back(v.e);
        PIC_CUDA(cudaMalloc(&v.eu, bytes));
        M.allocs.push_back(v.eu);
        PIC_CUDA(cudaMalloc(&v.g, bytes));
        M.allocs.push_back(v.g);
        PIC_CUDA(cudaMemset(v.e, 0, bytes));
        PIC_CUDA(cudaMemset(v.eu, 0, bytes));
        PIC_CUDA(cudaMemset(v.g, 0, bytes));
        v.ec = v.e;
        v.rz = nullptr;
        if (M.rz) {
            const std::vector<double> rd = rz_rows(v.ny, hx, hy);
            std::vector<T> rt(rd.begin(), rd.end());
            T* d = nullptr;
            PIC_CUDA(cudaMalloc(&d, rt.size() * sizeof(T)));
            M.allocs.push_back(d);
            PIC_CUDA(cudaMemcpy(d, rt.data(), rt.size() * sizeof(T), cudaMemcpyHostToDevice));
            v.rz = d;
            if (l == 0) {
                PIC_CUDA(cudaMalloc(&M.rz0, rd.size() * sizeof(double)));
                M.allocs.push_back(M.rz0);
                PIC_CUDA(cudaMemcpy(M.rz0, rd.data(), rd.size() * sizeof(double), cudaMemcpyHostToDevice));
            }
        }
        lv.push_back(v);
    }
    return PIC_OK;
}

// Gauss-Jordan inverse with partial pivoting (coarsest level, a few hundred unknowns).
static bool invert(std::vector<double>& a, int n) {
    std::vector<double> inv(size_t(n) * n, 0.0);
    for (int i = 0; i < n; ++i) inv[size_t(i) * n + i] = 1.0;
    for (int c = 0; c < n; ++c) {
        int p = c;
        for (int r = c + 1; r < n; ++r)
            if (std::fabs(a[size_t(r) * n + c]) > std::fabs(a[size_t(p) * n + c])) p = r;
        if (std::fabs(a[size_t(p) * n + c]) < 1e-300) return false;
        if (p != c)
            for (int k = 0; k < n; ++k) {
                std::swap(a[size_t(p) * n + k], a[size_t(c) * n + k]);
                std::swap(inv[size_t(p) * n + k], inv[size_t(c) * n + k]);
            }
        const double d = 1.0 / a[size_t(c) * n + c];
        for (int k = 0; k < n; ++k) {
            a[size_t(c) * n + k] *= d;
            inv[size_t(c) * n + k] *= d;
        }
        for (int r = 0; r < n; ++r) {
            if (r == c) continue;
            const double f = a[size_t(r) * n + c];
            if (f == 0.0) continue;
            for (int k = 0; k < n; ++k) {
                a[size_t(r) * n + k] -= f * a[size_t(c) * n + k];
                inv[size_t(r) * n + k] -= f * inv[size_t(c) * n + k];
            }
        }
    }
    a.swap(inv);
    return true;
}

// The dense operator of level l (spacings dx 2^l, dy 2^l) on its free nodes:
// not Dirichlet, not on the grid edges (in r-z geometry the axis row is free).
// idx lists the free nodes in row-major order; bw is the largest distance
// between a row and the column of one of its couplings.  With more than
// max_n free nodes only idx is filled.
static std::vector<double> dense_operator(const MgImpl& M, int l, int nx, int ny, const std::vector<uint8_t>& mask,
                                          std::vector<int>& idx, int& bw, int max_n) {
    std::vector<int> where(size_t(nx) * ny, -1);
    idx.clear();
    for (int j = M.rz ? 0 : 1; j < ny - 1; ++j)
        for (int i = 1; i < nx - 1; ++i)
            if (!mask[size_t(j) * nx + i]) {
                where[size_t(j) * nx + i] = int(idx.size());
                idx.push_back(j * nx + i);
            }
    const int n = int(idx.size());
    bw = 0;
    if (n > max_n) return {};
    const double hx = M.dx * double(1 << l), hy = M.dy * double(1 << l);
    const double ccx = 1.0 / (hx * hx), ccy = 1.0 / (hy * hy);
    const std::vector<double> rows = M.rz ? rz_rows(ny, hx, hy) : std::vector<double>();
    std::vector<double> A(size_t(n) * n, 0.0);
    for (int a = 0; a < n; ++a) {
        const int k = idx[a], j = k / nx;
        const double wn = M.rz ? rows[4 * j] : ccy, ws = M.rz ? rows[4 * j + 1] : ccy;
        A[size_t(a) * n + a] = -(2.0 * ccx + wn + ws);
        const int nb[4] = {k - 1, k + 1, j > 0 ? k - nx : -1, k + nx};
        const double w[4] = {ccx, ccx, ws, wn};
        for (int q = 0; q < 4; ++q) {
            const int b = nb[q] >= 0 ? where[nb[q]] : -1;
            if (b >= 0) {
                A[size_t(a) * n + b] += w[q];
                bw = std::max(bw, std::abs(b - a));
            }
        }
    }
    return A;
}

// The two-level launches (k_mg_down2, k_mg_up2) for levels Lc-2 and Lc-1,
// where their shared memory fits.
template <class T>
static int configure_fuse2(MgImpl& M) {
    const size_t d = down2_smem<T>(M.o.pre_sweeps), u = up2_smem<T>(M.o.post_sweeps);
    if (d > 227 * 1024 || u > 227 * 1024) return PIC_OK;
    PIC_TRY(raise_smem_limit(reinterpret_cast<const void*>(down2_kernel<T>(M.o.pre_sweeps)), d));
    PIC_TRY(raise_smem_limit(reinterpret_cast<const void*>(up2_kernel<T>(M.o.post_sweeps)), u));
    M.fuse2 = true;
    return PIC_OK;
}

// The direct solve of level Lc (see k_mg_direct); left off (the coarse
// V-cycle kernel runs) when the level has no free node or too many.
static int configure_direct(MgImpl& M, const std::vector<int>& nxs, const std::vector<int>& nys,
                            const std::vector<std::vector<uint8_t>>& masks) {
    const int l = M.Lc, nx = nxs[l], ny = nys[l];
    std::vector<int> idx;
    int bw = 0;
    std::vector<double> A = dense_operator(M, l, nx, ny, masks[l], idx, bw, kDirectMaxFree);
    const int n = int(idx.size());
    if (n == 0 || n > kDirectMaxFree) return PIC_OK;
    if (!band_inverse(A, n, bw)) return fail(PIC_ERR_NUMERIC, "pic_mg_create: singular coarse system");
    std::vector<char> fr(size_t(nx) * ny, 0);
    for (int k : idx) fr[k] = 1;
    std::vector<int> all(idx);
    for (int k = 0; k < nx * ny; ++k)
        if (!fr[k]) all.push_back(k);
    // the inverse in FP32 only for a mixed-precision V-cycle that asked for it
    const bool f32 = M.precision == PIC_MG_MIXED && M.o.coarse_fp32;
    M.dinv64 = !f32;
    const size_t bytes = A.size() * (f32 ? sizeof(float) : sizeof(double));
    PIC_CUDA(cudaMalloc(&M.dinv, bytes));
    M.allocs.push_back(M.dinv);
    if (f32) {
        const std::vector<float> af(A.begin(), A.end());
        PIC_CUDA(cudaMemcpy(M.dinv, af.data(), bytes, cudaMemcpyHostToDevice));
    } else {
        PIC_CUDA(cudaMemcpy(M.dinv, A.data(), bytes, cudaMemcpyHostToDevice));
    }
    PIC_CUDA(cudaMalloc(&M.didx, all.size() * sizeof(int)));
    M.allocs.push_back(M.didx);
    PIC_CUDA(cudaMemcpy(M.didx, all.data(), all.size() * sizeof(int), cudaMemcpyHostToDevice));
    M.dn = n;
    M.dnz = int(all.size()) - n;
    M.direct = true;
    return PIC_OK;
}

template <class T>
static int configure_kernels(MgImpl& M) {
    const size_t down = down_smem<T>(M.o.pre_sweeps, M.rz), up = up_smem<T>(M.o.post_sweeps, M.rz);
    const size_t upr = up_smem<T>(M.o.post_sweeps, M.rz, true);
    if (down > 227 * 1024 || upr > 227 * 1024 || M.cl[0].smem > 227 * 1024 || M.cl[1].smem > 227 * 1024)
        return fail(PIC_ERR_BAD_ARG, "multigrid: shared memory too large (sweeps %d/%d)", M.o.pre_sweeps,
                    M.o.post_sweeps);
    if (M.rz) {
        PIC_TRY(raise_smem_limit(reinterpret_cast<const void*>(down_kernel<T, true>(M.o.pre_sweeps)), down));
        PIC_TRY(raise_smem_limit(reinterpret_cast<const void*>(up_kernel<T, true>(M.o.post_sweeps)), up));
        PIC_TRY(raise_smem_limit(reinterpret_cast<const void*>(up_res_kernel<T, true>(M.o.post_sweeps)), upr));
        PIC_TRY(raise_smem_limit(reinterpret_cast<const void*>(k_mg_coarse<T, true>), M.cl[0].smem));
        return PIC_OK;  // r-z solves use the graph and host loops only
    }
    PIC_TRY(raise_smem_limit(reinterpret_cast<const void*>(down_kernel<T, false>(M.o.pre_sweeps)), down));
    PIC_TRY(raise_smem_limit(reinterpret_cast<const void*>(up_kernel<T, false>(M.o.post_sweeps)), up));
    PIC_TRY(raise_smem_limit(reinterpret_cast<const void*>(up_res_kernel<T, false>(M.o.post_sweeps)), upr));
    PIC_TRY(raise_smem_limit(reinterpret_cast<const void*>(k_mg_coarse<T, false>), M.cl[0].smem));
    M.solve_smem = std::max(std::max(down, up), M.cl[1].smem);
    PIC_TRY(raise_smem_limit(reinterpret_cast<const void*>(k_mg_solve<T>), M.solve_smem));
    int per_sm = 0;
    PIC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_mg_solve<T>, kMgThreads, M.solve_smem));
    if (per_sm < 1) return fail(PIC_ERR_CUDA, "multigrid: the persistent kernel does not fit on an SM");
    M.solve_grid = std::min(per_sm, 2) * num_sms();
    return PIC_OK;
}

static size_t pad16(size_t n) { return (n + 15) / 16 * 16; }

// Shared-memory layout of levels [first, L) for the single-block coarse
// V-cycle, and the device image of their masks (grid edges included).
static int build_layout(MgImpl& M, int first, const std::vector<int>& nxs, const std::vector<int>& nys,
                        const std::vector<std::vector<uint8_t>>& masks, size_t esz, CoarseLayout& C) {
    C.first = first;
    size_t off = 0;
    for (int l = first; l < M.L; ++l) {
        C.off_e[l - first] = int(off);
        off += pad16(size_t(nxs[l]) * nys[l] * esz);
    }
    C.e_bytes = int(off);
    for (int l = first; l < M.L; ++l) {
        C.off_g[l - first] = int(off);
        off += pad16(size_t(nxs[l]) * nys[l] * esz);
    }
    C.m_off = int(off);
    std::vector<uint8_t> img;
    for (int l = first; l < M.L; ++l) {
        C.off_m[l - first] = int(off);
        const int nx = nxs[l], ny = nys[l];
        const size_t G = size_t(nx) * ny;
        std::vector<uint8_t> m(pad16(G), 1);
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i)
                m[size_t(j) * nx + i] = (i == 0 || (j == 0 && !M.rz) || i == nx - 1 || j == ny - 1 ||
                                         masks[l][size_t(j) * nx + i]);
        img.insert(img.end(), m.begin(), m.end());
        off += m.size();
    }
    C.m_vec = int(img.size() / 16);
    if (cudaMalloc(&C.mimg, img.size()) != cudaSuccess) return PIC_ERR_CUDA;
    M.allocs.push_back(C.mimg);
    if (cudaMemcpy(C.mimg, img.data(), img.size(), cudaMemcpyHostToDevice) != cudaSuccess) return PIC_ERR_CUDA;
    C.g_vec = int(pad16(size_t(nxs[first]) * nys[first] * esz) / 16);
    const size_t nf = size_t(M.nfree_c), ab = pad16(nf * nf * sizeof(double)), cb = pad16(nf * sizeof(int));
    if (nf > 0 && off + ab + cb <= 200 * 1024) {
        C.a_off = int(off);
        off += ab;
        C.c_off = int(off);
        off += cb;
        C.a_vec = int(ab / 16);
        C.c_vec = int(cb / 16);
    } else {
        C.a_off = C.c_off = -1;
        C.a_vec = C.c_vec = 0;
    }
    C.smem = off;
    return PIC_OK;
}

template <class T>
static void fill_coarse(const MgImpl& M, const CoarseLayout& C, const std::vector<LevelDev<T>>& lv, double* phi,
                        CoarseDesc<T>& D) {
    D.nlev = M.L - C.first;
    for (int c = 0; c < D.nlev; ++c) {
        D.lv[c] = lv[C.first + c];
        D.off_e[c] = C.off_e[c];
        D.off_g[c] = C.off_g[c];
        D.off_m[c] = C.off_m[c];
    }
    D.e_bytes = C.e_bytes;
    D.m_off = C.m_off;
    D.a_off = C.a_off;
    D.c_off = C.c_off;
    D.mimg = C.mimg;
    D.g16 = reinterpret_cast<const uint4*>(lv[C.first].g);
    D.ainv16 = reinterpret_cast<const uint4*>(M.ainv);
    D.cidx16 = reinterpret_cast<const uint4*>(M.cidx);
    D.m_vec = C.m_vec;
    D.g_vec = C.g_vec;
    D.a_vec = C.a_vec;
    D.c_vec = C.c_vec;
    D.ainv = M.ainv;
    D.cidx = M.cidx;
    D.nf = M.nfree_c;
    D.omega = T(M.o.omega);
    D.pre = M.o.pre_sweeps;
    D.post = M.o.post_sweeps;
    D.phi0 = C.first == 0 ? phi : nullptr;
}

// Picks the cluster size (16 CTAs where the device allows, else 8) whose
// band phases fit in shared memory; leaves cluster_ok false (the graph loop
// is used instead) for FP64 levels or bands that do not fit.
static int configure_cluster(MgImpl& M, const std::vector<int>& nxs, const std::vector<int>& nys, int first = 0) {
    M.cluster_ok = false;
    if (M.precision != PIC_MG_MIXED) return PIC_OK;
    const int pre = M.o.pre_sweeps, post = M.o.post_sweeps;
    for (int cs : {16, 8}) {
        size_t need = M.cl[1].smem;
        for (int l = first; l < M.Lp; ++l) {
            const size_t per = size_t((nys[l] + cs - 1) / cs);
            const size_t Rd = per + 2 * size_t(2 * pre + 2), Ru = per + 4 * size_t(post);
            const size_t down = Rd * nxs[l] * (2 * sizeof(float) + 1);
            const size_t CR = Ru / 2 + 3;
            const size_t up = Ru * nxs[l] * (2 * sizeof(float) + 1) + CR * nxs[l + 1] * sizeof(float);
            need = std::max(need, std::max(down, up));
        }
        if (need > 227 * 1024) continue;
        if (cs > 8 &&
            cudaFuncSetAttribute(k_mg_cluster, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) {
            cudaGetLastError();
            continue;
        }
        PIC_TRY(raise_smem_limit(reinterpret_cast<const void*>(k_mg_cluster), need));
        cudaLaunchConfig_t cfg{};
        cfg.gridDim = dim3(cs);
        cfg.blockDim = dim3(kClusterThreads);
        cfg.dynamicSmemBytes = need;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = cs;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        int n = 0;
        if (cudaOccupancyMaxActiveClusters(&n, k_mg_cluster, &cfg) != cudaSuccess) {
            cudaGetLastError();
            continue;
        }
        if (n >= 1) {
            M.cluster_ok = true;
            M.cluster_size = cs;
            M.cluster_smem = need;
            return PIC_OK;
        }
    }
    return PIC_OK;
}

static void mg_release(pic_mg* mg) {
    if (!mg) return;
    MgImpl& M = mg->m;
    if (M.exec) cudaGraphExecDestroy(M.exec);
    if (M.side) cudaStreamDestroy(M.side);
    if (M.cap) cudaStreamDestroy(M.cap);
    if (M.dst) dst_destroy(M.dst);
    for (void* p : M.allocs) cudaFree(p);
    delete mg;
}

int mg_create(int nx, int ny, double dx, double dy, const uint8_t* h_mask, const pic_mg_options* opts,
              pic_mg** out) {
    if (!out || !h_mask || nx < 3 || ny < 3 || !(dx > 0) || !(dy > 0))
        return fail(PIC_ERR_BAD_ARG, "pic_mg_create: bad arguments");
    pic_mg* mg = new pic_mg;
    MgImpl& M = mg->m;
    M.o.precision = PIC_MG_MIXED;
    M.o.pre_sweeps = 2;
    M.o.post_sweeps = 2;
    M.o.omega = 1.15;
    M.o.coarsest_max = 9;
    if (opts) {
        M.o.precision = opts->precision;
        if (opts->pre_sweeps > 0) M.o.pre_sweeps = opts->pre_sweeps;
        if (opts->post_sweeps > 0) M.o.post_sweeps = opts->post_sweeps;
        if (opts->omega > 0) M.o.omega = opts->omega;
        if (opts->coarsest_max >= 3) M.o.coarsest_max = opts->coarsest_max;
        M.o.launch_mode = opts->launch_mode;
        M.o.geometry = opts->geometry;
        M.o.coarse_fp32 = opts->coarse_fp32 ? 1 : 0;
    }
    auto bail = [&](int code) {
        mg_release(mg);
        return code;
    };
    if (M.o.precision != PIC_MG_MIXED && M.o.precision != PIC_MG_FP64)
        return bail(fail(PIC_ERR_BAD_ARG, "pic_mg_create: unknown precision %d", M.o.precision));
    if (M.o.pre_sweeps > kMgMaxSweeps || M.o.post_sweeps > kMgMaxSweeps)
        return bail(fail(PIC_ERR_BAD_ARG, "pic_mg_create: at most 8 pre/post sweeps"));
    if (M.o.launch_mode < PIC_MG_PERSISTENT || M.o.launch_mode > PIC_MG_HYBRID)
        return bail(fail(PIC_ERR_BAD_ARG, "pic_mg_create: unknown launch mode %d", M.o.launch_mode));
    if (M.o.geometry != PIC_GEOM_CARTESIAN && M.o.geometry != PIC_GEOM_RZ)
        return bail(fail(PIC_ERR_BAD_ARG, "pic_mg_create: unknown geometry %d", M.o.geometry));
    M.rz = M.o.geometry == PIC_GEOM_RZ;
    // r-z solves run in the graph or host loop (the persistent and cluster
    // kernels are Cartesian)
    if (M.rz && (M.o.launch_mode == PIC_MG_PERSISTENT || M.o.launch_mode == PIC_MG_CLUSTER ||
                 M.o.launch_mode == PIC_MG_HYBRID))
        M.o.launch_mode = PIC_MG_GRAPH_LOOP;
    M.precision = M.o.precision;
    M.nx = nx;
    M.ny = ny;
    M.dx = dx;
    M.dy = dy;
    std::vector<int> nxs{nx}, nys{ny};
    std::vector<std::vector<uint8_t>> masks(1, std::vector<uint8_t>(h_mask, h_mask + size_t(nx) * ny));
    for (auto& v : masks[0]) v = v ? 1 : 0;
    while (nxs.back() > M.o.coarsest_max && nys.back() > M.o.coarsest_max && ((nxs.back() - 1) % 2 == 0) &&
           ((nys.back() - 1) % 2 == 0)) {
        const int fx = nxs.back(), fy = nys.back();
        const int cx = (fx - 1) / 2 + 1, cy = (fy - 1) / 2 + 1;
        const std::vector<uint8_t>& mf = masks.back();
        // A coarse node is Dirichlet if the fine node it injects from is, or if
        // an internal Dirichlet node (an electrode; not the grid edges, which
        // are Dirichlet on every level) lies in its 3 x 3 fine neighbourhood:
        // an electrode on an odd line would otherwise vanish from the coarse
        // grid, whose correction then spans it, and the cycle can diverge.
        auto inner = [&](int i, int j) {
            return i > 0 && i < fx - 1 && j < fy - 1 && (j > 0 || M.rz) && mf[size_t(j) * fx + i] != 0;
        };
        std::vector<uint8_t> mc(size_t(cx) * cy);
        for (int J = 0; J < cy; ++J)
            for (int I = 0; I < cx; ++I) {
                uint8_t v = mf[size_t(2 * J) * fx + 2 * I];
                for (int dj = -1; dj <= 1 && !v; ++dj)
                    for (int di = -1; di <= 1 && !v; ++di) {
                        const int i = 2 * I + di, j = 2 * J + dj;
                        if (i >= 0 && j >= 0 && i < fx && j < fy && inner(i, j)) v = 1;
                    }
                mc[size_t(J) * cx + I] = v;
            }
        nxs.push_back(cx);
        nys.push_back(cy);
        masks.push_back(std::move(mc));
    }
    M.L = int(nxs.size());
    if (M.L > kMgMaxLevels) return bail(fail(PIC_ERR_BAD_ARG, "pic_mg_create: more than %d levels", kMgMaxLevels));
    const long coarse_max = M.precision == PIC_MG_MIXED ? kCoarseMaxNodes32 : kCoarseMaxNodes64;
    M.Lc = 0;
    while (M.Lc < M.L && long(nxs[M.Lc]) * nys[M.Lc] > coarse_max) ++M.Lc;
    if (M.L - M.Lc > kMgMaxCoarseLevels) M.Lc = M.L - kMgMaxCoarseLevels;
    if (M.Lc >= M.L)
        return bail(fail(PIC_ERR_BAD_ARG,
                         "pic_mg_create: grid %dx%d does not coarsen below %ld nodes; node counts must be 2^k*c+1", nx,
                         ny, coarse_max));
    const int ncx = nxs.back(), ncy = nys.back();
    std::vector<int> idx;
    int bw = 0;
    std::vector<double> A = dense_operator(M, M.L - 1, ncx, ncy, masks.back(), idx, bw, 4096);
    M.nfree_c = int(idx.size());
    if (M.nfree_c > 4096)
        return bail(fail(PIC_ERR_BAD_ARG, "pic_mg_create: coarsest level %dx%d has %d unknowns", ncx, ncy, M.nfree_c));
    if (M.nfree_c > 0) {
        const int n = M.nfree_c;
        if (!invert(A, n)) return bail(fail(PIC_ERR_NUMERIC, "pic_mg_create: singular coarsest system"));
        // padded to 16 bytes: the coarse kernel reads both in 16-byte words
        const size_t ab = (A.size() * sizeof(double) + 15) / 16 * 16, cb = (idx.size() * sizeof(int) + 15) / 16 * 16;
        if (cudaMalloc(&M.ainv, ab) != cudaSuccess)
            return bail(fail(PIC_ERR_CUDA, "pic_mg_create: out of device memory"));
        M.allocs.push_back(M.ainv);
        cudaMemset(M.ainv, 0, ab);
        cudaMemcpy(M.ainv, A.data(), A.size() * sizeof(double), cudaMemcpyHostToDevice);
        if (cudaMalloc(&M.cidx, cb) != cudaSuccess)
            return bail(fail(PIC_ERR_CUDA, "pic_mg_create: out of device memory"));
        M.allocs.push_back(M.cidx);
        cudaMemset(M.cidx, 0, cb);
        cudaMemcpy(M.cidx, idx.data(), idx.size() * sizeof(int), cudaMemcpyHostToDevice);
    }
    const size_t esz = M.precision == PIC_MG_MIXED ? sizeof(float) : sizeof(double);
    M.Lp = 0;
    while (M.Lp < M.L && long(nxs[M.Lp]) * nys[M.Lp] > kPersistCoarseMax) ++M.Lp;
    if (M.L - M.Lp > kMgMaxCoarseLevels) M.Lp = M.L - kMgMaxCoarseLevels;
    if (build_layout(M, M.Lc, nxs, nys, masks, esz, M.cl[0]) != PIC_OK ||
        build_layout(M, M.Lp, nxs, nys, masks, esz, M.cl[1]) != PIC_OK)
        return bail(fail(PIC_ERR_CUDA, "pic_mg_create: out of device memory"));
    int st = M.precision == PIC_MG_MIXED ? alloc_levels(M, M.lf, masks, nxs, nys)
                                         : alloc_levels(M, M.ld, masks, nxs, nys);
    if (st == PIC_OK) st = M.precision == PIC_MG_MIXED ? configure_kernels<float>(M) : configure_kernels<double>(M);
    if (st == PIC_OK && M.o.launch_mode == PIC_MG_CLUSTER) st = configure_cluster(M, nxs, nys);
    if (st == PIC_OK && M.o.launch_mode == PIC_MG_HYBRID) {
        // tile kernels for the levels above kHybridBandMax nodes, one cluster
        // launch for the rest; FP32 Cartesian levels only, else the graph loop
        M.Lt = 0;
        while (M.Lt < M.L && long(nxs[M.Lt]) * nys[M.Lt] > kHybridBandMax) ++M.Lt;
        if (M.precision == PIC_MG_MIXED && !M.rz && M.Lt >= 1 && M.Lt < M.Lp) {
            st = configure_cluster(M, nxs, nys, M.Lt);
            M.hybrid = st == PIC_OK && M.cluster_ok;
        }
        if (!M.hybrid) M.o.launch_mode = PIC_MG_GRAPH_LOOP;
    }
    if (st == PIC_OK && M.o.launch_mode == PIC_MG_DST) {
        // the sine-transform solve applies to Cartesian grids of 2^q + 1 nodes
        // whose Dirichlet nodes are the edges alone; otherwise the graph loop
        bool edges_only = !M.rz;
        for (int j = 1; j < ny - 1 && edges_only; ++j)
            for (int i = 1; i < nx - 1; ++i)
                if (masks[0][size_t(j) * nx + i]) {
                    edges_only = false;
                    break;
                }
        const bool pow2 = nx - 1 >= 4 && ny - 1 >= 4 && nx - 1 <= 2048 && ny - 1 <= 2048 &&
                          ((nx - 1) & (nx - 2)) == 0 && ((ny - 1) & (ny - 2)) == 0;
        if (edges_only && pow2) st = dst_create(nx, ny, dx, dy, &M.dst);
        if (st == PIC_OK && !M.dst) M.o.launch_mode = PIC_MG_GRAPH_LOOP;
    }
    if (st == PIC_OK && M.Lc >= 1 &&
        (M.o.launch_mode == PIC_MG_GRAPH_LOOP || M.o.launch_mode == PIC_MG_HOST_LOOP))
        st = configure_direct(M, nxs, nys, masks);
    if (st == PIC_OK && M.direct && !M.rz && M.Lc >= 3)
        st = M.precision == PIC_MG_MIXED ? configure_fuse2<float>(M) : configure_fuse2<double>(M);
    if (st != PIC_OK) return bail(st);
    M.grd0 = dim3(div_up(nx, M.blk0.x), div_up(ny, M.blk0.y * kR0Rows));
    // block partials of the residual norm: one pair per block of the level-0
    // tiling (k_mg_r0, k_mg_up_res) or of the persistent grid (k_mg_solve),
    // whichever is larger
    const int nb = std::max(std::max(int(M.grd0.x * M.grd0.y), div_up(nx, kMgTile) * div_up(ny, kMgTile)),
                            M.solve_grid);
    if (cudaMalloc(&M.N.partial, sizeof(double) * 2 * nb) != cudaSuccess)
        return bail(fail(PIC_ERR_CUDA, "pic_mg_create: out of device memory"));
    M.allocs.push_back(M.N.partial);
    if (cudaMalloc(&M.r64, sizeof(double) * size_t(nx) * ny) != cudaSuccess)
        return bail(fail(PIC_ERR_CUDA, "pic_mg_create: out of device memory"));
    M.allocs.push_back(M.r64);
    cudaMemset(M.r64, 0, sizeof(double) * size_t(nx) * ny);
    char* small = nullptr;
    if (cudaMalloc(&small, 256) != cudaSuccess) return bail(fail(PIC_ERR_CUDA, "pic_mg_create: out of device memory"));
    M.allocs.push_back(small);
    cudaMemset(small, 0, 256);
    M.N.norms = reinterpret_cast<double*>(small);
    M.N.total = reinterpret_cast<long long*>(small + 16);
    M.N.done = reinterpret_cast<unsigned*>(small + 24);
    M.N.converged = reinterpret_cast<int*>(small + 28);
    M.N.cycles = reinterpret_cast<int*>(small + 32);
    M.bar = reinterpret_cast<GridBar*>(small + 40);
    M.error = reinterpret_cast<int*>(small + 48);
    if (cudaStreamCreateWithFlags(&M.side, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&M.cap, cudaStreamNonBlocking) != cudaSuccess)
        return bail(fail(PIC_ERR_CUDA, "pic_mg_create: stream creation failed"));
    *out = mg;
    return PIC_OK;
}

static int launch_cluster_tail(MgImpl& M, const std::vector<LevelDev<float>>& lv, cudaStream_t st);

// The FP64 residual and the loop decision (k_mg_r0) of either geometry.
template <class T>
static void launch_r0(MgImpl& M, const std::vector<LevelDev<T>>& lv, double* phi, const double* f, double tol,
                      int max_cycles, int initial, cudaGraphConditionalHandle cond, int use_cond, cudaStream_t st) {
    const double cx = 1.0 / (M.dx * M.dx), cy = 1.0 / (M.dy * M.dy);
    const double* nul = nullptr;
    if (M.rz)
        launch_pdl(k_mg_r0<T, true>, M.grd0, M.blk0, 0, st, phi, f, lv[0].mask, M.nx, M.ny, cx, cy, lv[0].g, M.N,
                   tol * tol, max_cycles, initial, cond, use_cond, (const double*)M.rz0, M.r64);
    else
        launch_pdl(k_mg_r0<T, false>, M.grd0, M.blk0, 0, st, phi, f, lv[0].mask, M.nx, M.ny, cx, cy, lv[0].g, M.N,
                   tol * tol, max_cycles, initial, cond, use_cond, nul, M.r64);
}

// One V-cycle followed by the residual check, launched on stream st.  With
// tile levels, the finest down phase reads the FP64 residual (r64, from
// k_mg_r0 or the previous cycle) and the finest up phase updates it and takes
// the loop decision (k_mg_up_res); a cycle of the coarse kernel alone ends
// with k_mg_r0.
template <class T>
static int launch_cycle(MgImpl& M, std::vector<LevelDev<T>>& lv_in, double* phi, const double* f, double tol,
                        int max_cycles, cudaGraphConditionalHandle cond, int use_cond, cudaStream_t st, int& count) {
    // the hybrid cycle's coarse end starts at Lt (tiles above it); its
    // cluster kernel's bands write eu like the tile up phases, its CTA 0 the
    // levels from Lp
    const bool hyb = std::is_same<T, float>::value && M.hybrid;
    const int Ltile = hyb ? M.Lt : M.Lc;
    const std::vector<LevelDev<T>> lv = with_corrections(lv_in, hyb ? M.Lp : M.Lc);
    const T omega = T(M.o.omega);
    const size_t down = down_smem<T>(M.o.pre_sweeps, M.rz), up = up_smem<T>(M.o.post_sweeps, M.rz);
    const DownKernel<T> kdown = M.rz ? down_kernel<T, true>(M.o.pre_sweeps) : down_kernel<T, false>(M.o.pre_sweeps);
    const UpKernel<T> kup = M.rz ? up_kernel<T, true>(M.o.post_sweeps) : up_kernel<T, false>(M.o.post_sweeps);
    count = 0;
    // levels Lc-2 and Lc-1 in one launch each way where that applies
    const bool f2 = M.fuse2 && !hyb;
    const int Lsingle = f2 ? Ltile - 2 : Ltile;
    for (int l = 0; l < Lsingle; ++l) {
        const dim3 g(div_up(lv[l].nx, kMgTile), div_up(lv[l].ny, kMgTile));
        // the finest down phase waits for its predecessor to finish before it
        // is placed: launched ahead, its CTAs would take the SMs its
        // predecessor leaves free first, several to an SM (measured 8.5 us
        // instead of 4.8 at 513^2)
        if (l == 0) kdown<<<g, dim3(kMgThreads), down, st>>>(lv[0], lv[1], omega, (const double*)M.r64);
        else launch_pdl(kdown, g, dim3(kMgThreads), down, st, lv[l], lv[l + 1], omega, (const double*)nullptr);
        ++count;
    }
    if (f2) {
        const int l = Lsingle;
        const dim3 g(div_up(lv[l].nx, kMgTile), div_up(lv[l].ny, kMgTile));
        launch_pdl(down2_kernel<T>(M.o.pre_sweeps), g, dim3(kMgThreads), down2_smem<T>(M.o.pre_sweeps), st, lv[l],
                   lv[l + 1], lv[l + 2], omega);
        ++count;
    }
    if constexpr (std::is_same<T, float>::value) {
        if (hyb) {
            PIC_TRY(launch_cluster_tail(M, lv, st));
            ++count;
        }
    }
    if (!hyb && M.direct) {
        const DirectDesc<T> D{M.dinv, M.didx, M.didx + M.dn, lv[M.Lc].g, lv[M.Lc].e, M.dn, M.dnz};
        if (M.dinv64) launch_pdl(k_mg_direct<T, double>, dim3(div_up(M.dn, kDirectRows)), dim3(kDirectRows * 32), 0, st, D);
        else launch_pdl(k_mg_direct<T, T>, dim3(div_up(M.dn, kDirectRows)), dim3(kDirectRows * 32), 0, st, D);
        ++count;
    } else if (!hyb) {
        CoarseDesc<T> D{};
        fill_coarse(M, M.cl[0], lv, phi, D);
        if (M.rz) launch_pdl(k_mg_coarse<T, true>, dim3(1), dim3(kCoarseThreads), M.cl[0].smem, st, D);
        else launch_pdl(k_mg_coarse<T, false>, dim3(1), dim3(kCoarseThreads), M.cl[0].smem, st, D);
        ++count;
    }
    if (f2) {
        const int l = Lsingle;
        const dim3 g(div_up(lv[l].nx, kMgTile), div_up(lv[l].ny, kMgTile));
        launch_pdl(up2_kernel<T>(M.o.post_sweeps), g, dim3(kMgThreads), up2_smem<T>(M.o.post_sweeps), st, lv[l],
                   lv[l + 1], lv[l + 2], omega);
        ++count;
    }
    for (int l = Lsingle - 1; l >= 1; --l) {
        const dim3 g(div_up(lv[l].nx, kMgTile), div_up(lv[l].ny, kMgTile));
        launch_pdl(kup, g, dim3(kMgThreads), up, st, lv[l], lv[l + 1], omega, (double*)nullptr);
        ++count;
    }
    if (Ltile >= 1) {
        ResArgs R{};
        R.r64 = M.r64;
        R.rz0 = M.rz ? (const double*)M.rz0 : nullptr;
        R.cx = 1.0 / (M.dx * M.dx);
        R.cy = 1.0 / (M.dy * M.dy);
        R.N = M.N;
        R.tol2 = tol * tol;
        R.max_cycles = max_cycles;
        R.cond = cond;
        R.use_cond = use_cond;
        const UpResKernel<T> kres =
            M.rz ? up_res_kernel<T, true>(M.o.post_sweeps) : up_res_kernel<T, false>(M.o.post_sweeps);
        const dim3 g(div_up(lv[0].nx, kMgTile), div_up(lv[0].ny, kMgTile));
        launch_pdl(kres, g, dim3(kMgThreads), up_smem<T>(M.o.post_sweeps, M.rz, true), st, lv[0], lv[1], omega, phi,
                   R);
    } else {
        launch_r0(M, lv, phi, f, tol, max_cycles, 0, cond, use_cond, st);
    }
    ++count;
    PIC_LAUNCH_CHECK();
    return PIC_OK;
}

// min_cycles: V-cycles chained in the capturing graph itself before the WHILE
// node, which only then tests for convergence (each iteration of a WHILE
// node costs a launch of its body graph).
template <class T>
static int capture_solve(MgImpl& M, std::vector<LevelDev<T>>& lv, double* phi, const double* f, double tol,
                         int max_cycles, int min_cycles, cudaStream_t st) {
    cudaStreamCaptureStatus cs;
    cudaGraph_t g = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t nd = 0;
    PIC_CUDA(cudaStreamGetCaptureInfo(st, &cs, nullptr, &g, &deps, &nd));
    if (cs != cudaStreamCaptureStatusActive) return fail(PIC_ERR_BAD_ARG, "multigrid: stream is not capturing");
    cudaGraphConditionalHandle h;
    PIC_CUDA(cudaGraphConditionalHandleCreate(&h, g, 0, cudaGraphCondAssignDefault));
    const int K = std::max(0, std::min(min_cycles, max_cycles));
    launch_r0(M, lv, phi, f, tol, max_cycles, 1, h, K == 0, st);
    PIC_LAUNCH_CHECK();
    for (int k = 0; k < K; ++k) {
        int count = 0;
        PIC_TRY(launch_cycle(M, lv, phi, f, tol, max_cycles, h, k == K - 1, st, count));
    }
    PIC_CUDA(cudaStreamGetCaptureInfo(st, &cs, nullptr, &g, &deps, &nd));
    cudaGraphNodeParams p{};
    p.type = cudaGraphNodeTypeConditional;
    p.conditional.handle = h;
    p.conditional.type = cudaGraphCondTypeWhile;
    p.conditional.size = 1;
    cudaGraphNode_t cn;
    PIC_CUDA(cudaGraphAddNode(&cn, g, deps, nd, &p));
    cudaGraph_t body = p.conditional.phGraph_out[0];
    PIC_CUDA(cudaStreamUpdateCaptureDependencies(st, &cn, 1, cudaStreamSetCaptureDependencies));
    PIC_CUDA(cudaStreamBeginCaptureToGraph(M.side, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
    int count = 0;
    const int rc = launch_cycle(M, lv, phi, f, tol, max_cycles, h, 1, M.side, count);
    cudaGraph_t body_out = nullptr;
    const cudaError_t ec = cudaStreamEndCapture(M.side, &body_out);
    if (rc != PIC_OK) return rc;
    if (ec != cudaSuccess) return fail(PIC_ERR_CUDA, "multigrid body capture: %s", cudaGetErrorString(ec));
    M.body_launches = count;
    return PIC_OK;
}

template <class T>
static int launch_persistent(MgImpl& M, std::vector<LevelDev<T>>& lv_in, double* phi, const double* f, double tol,
                             int max_cycles, cudaStream_t st) {
    const std::vector<LevelDev<T>> lv = with_corrections(lv_in, M.Lp);
    SolveDesc<T> S{};
    S.L = M.L;
    S.Lp = M.Lp;
    for (int l = 0; l < M.L; ++l) S.lv[l] = lv[l];
    fill_coarse(M, M.cl[1], lv, phi, S.coarse);
    S.f = f;
    S.phi = phi;
    S.nx = M.nx;
    S.ny = M.ny;
    S.cx = 1.0 / (M.dx * M.dx);
    S.cy = 1.0 / (M.dy * M.dy);
    S.N = M.N;
    S.tol2 = tol * tol;
    S.max_cycles = max_cycles;
    S.omega = T(M.o.omega);
    S.pre = M.o.pre_sweeps;
    S.post = M.o.post_sweeps;
    S.bar = M.bar;
    S.error = M.error;
    S.polls = M.wait_polls;
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(M.solve_grid);
    cfg.blockDim = dim3(kMgThreads);
    cfg.dynamicSmemBytes = M.solve_smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    PIC_CUDA(cudaLaunchKernelEx(&cfg, k_mg_solve<T>, S));
    return PIC_OK;
}

static int launch_cluster(MgImpl& M, double* phi, const double* f, double tol, int max_cycles, cudaStream_t st) {
    ClusterDesc S{};
    S.L = M.L;
    S.Lb = M.Lp;
    const std::vector<LevelDev<float>> lv = with_corrections(M.lf, M.Lp);
    for (int l = 0; l < M.L; ++l) S.lv[l] = lv[l];
    fill_coarse(M, M.cl[1], lv, phi, S.coarse);
    S.f = f;
    S.phi = phi;
    S.nx = M.nx;
    S.ny = M.ny;
    S.cx = 1.0 / (M.dx * M.dx);
    S.cy = 1.0 / (M.dy * M.dy);
    S.N = M.N;
    S.tol2 = tol * tol;
    S.max_cycles = max_cycles;
    S.omega = float(M.o.omega);
    S.pre = M.o.pre_sweeps;
    S.post = M.o.post_sweeps;
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(M.cluster_size);
    cfg.blockDim = dim3(kClusterThreads);
    cfg.dynamicSmemBytes = M.cluster_smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = M.cluster_size;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    PIC_CUDA(cudaLaunchKernelEx(&cfg, k_mg_cluster, S));
    return PIC_OK;
}

// The coarse end of a PIC_MG_HYBRID V-cycle: levels [Lt, Lp) in bands over the
// cluster, [Lp, L) in its CTA 0, in one launch (lv: with eu corrections below Lp).
static int launch_cluster_tail(MgImpl& M, const std::vector<LevelDev<float>>& lv, cudaStream_t st) {
    ClusterDesc S{};
    S.L = M.L;
    S.Lb = M.Lp;
    S.Lt = M.Lt;
    S.tail = 1;
    for (int l = 0; l < M.L; ++l) S.lv[l] = lv[l];
    fill_coarse(M, M.cl[1], lv, nullptr, S.coarse);
    S.omega = float(M.o.omega);
    S.pre = M.o.pre_sweeps;
    S.post = M.o.post_sweeps;
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(M.cluster_size);
    cfg.blockDim = dim3(kClusterThreads);
    cfg.dynamicSmemBytes = M.cluster_smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = M.cluster_size;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    PIC_CUDA(cudaLaunchKernelEx(&cfg, k_mg_cluster, S));
    return PIC_OK;
}

// Appends the whole solve to a capture in progress on `st`: the persistent or
// cluster kernel, or the residual and a WHILE node over V-cycles.
// The sine-transform solve, then the FP64 residual and its norms for pic_mg_info.
static int launch_dst(MgImpl& M, double* phi, const double* f, double tol, int max_cycles, cudaStream_t st) {
    PIC_TRY(dst_launch(M.dst, phi, f, st));
    if (M.precision == PIC_MG_MIXED) launch_r0(M, M.lf, phi, f, tol, max_cycles, 1, cudaGraphConditionalHandle{}, 0, st);
    else launch_r0(M, M.ld, phi, f, tol, max_cycles, 1, cudaGraphConditionalHandle{}, 0, st);
    PIC_LAUNCH_CHECK();
    return PIC_OK;
}

int mg_capture(MgImpl& M, double* phi, const double* f, double tol, int max_cycles, int min_cycles, cudaStream_t st) {
    if (M.dst) return launch_dst(M, phi, f, tol, max_cycles, st);
    if (M.o.launch_mode == PIC_MG_CLUSTER && M.cluster_ok) return launch_cluster(M, phi, f, tol, max_cycles, st);
    if (M.o.launch_mode == PIC_MG_PERSISTENT)
        return M.precision == PIC_MG_MIXED ? launch_persistent(M, M.lf, phi, f, tol, max_cycles, st)
                                           : launch_persistent(M, M.ld, phi, f, tol, max_cycles, st);
    if (M.o.launch_mode == PIC_MG_HOST_LOOP)
        return fail(PIC_ERR_BAD_ARG, "multigrid: the host-driven loop cannot be captured in a graph");
    return M.precision == PIC_MG_MIXED ? capture_solve(M, M.lf, phi, f, tol, max_cycles, min_cycles, st)
                                       : capture_solve(M, M.ld, phi, f, tol, max_cycles, min_cycles, st);
}

static int ensure_graph(MgImpl& M, double* phi, const double* f, double tol, int max_cycles, int min_cycles) {
    if (M.exec && M.g_phi == phi && M.g_f == f && M.g_tol == tol && M.g_max == max_cycles && M.g_min == min_cycles)
        return PIC_OK;
    if (M.exec) {
        cudaGraphExecDestroy(M.exec);
        M.exec = nullptr;
    }
    PIC_CUDA(cudaStreamBeginCapture(M.cap, cudaStreamCaptureModeThreadLocal));
    const int rc = mg_capture(M, phi, f, tol, max_cycles, min_cycles, M.cap);
    cudaGraph_t g = nullptr;
    const cudaError_t ec = cudaStreamEndCapture(M.cap, &g);
    if (rc != PIC_OK) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    if (ec != cudaSuccess) return fail(PIC_ERR_CUDA, "multigrid capture: %s", cudaGetErrorString(ec));
    const cudaError_t ei = cudaGraphInstantiate(&M.exec, g, 0);
    cudaGraphDestroy(g);
    if (ei != cudaSuccess) return fail(PIC_ERR_CUDA, "multigrid graph instantiate: %s", cudaGetErrorString(ei));
    M.g_phi = phi;
    M.g_f = f;
    M.g_tol = tol;
    M.g_max = max_cycles;
    M.g_min = min_cycles;
    return PIC_OK;
}

int mg_read_info(MgImpl& M, pic_mg_info* info) {
    unsigned char small[72];
    PIC_CUDA(cudaMemcpy(small, M.N.norms, sizeof small, cudaMemcpyDeviceToHost));
    int err[6];
    memcpy(err, small + 48, sizeof err);
    if (err[0]) {
        // the solve gave up (no kernel of it is still running: the stream was
        // synchronised): clear the flag and the barrier, so that the solver
        // can be used again, and report the timeout
        PIC_CUDA(cudaMemset(M.bar, 0, sizeof(GridBar)));
        PIC_CUDA(cudaMemset(M.error, 0, 6 * sizeof(int)));
        return fail(PIC_ERR_TIMEOUT,
                    "multigrid: grid barrier %d of the persistent solve timed out (block %d saw count %d, "
                    "generation %d, waited on %d)",
                    err[1], err[2], err[3], err[4], err[5]);
    }
    double norms[2];
    int conv, cycles;
    memcpy(norms, small, 16);
    memcpy(&conv, small + 28, 4);
    memcpy(&cycles, small + 32, 4);
    info->rhs_norm = std::sqrt(norms[0]);
    const double fn = norms[0] > 0 ? std::sqrt(norms[0]) : 1.0;
    info->rel_res = std::sqrt(norms[1]) / fn;
    info->cycles = cycles;
    info->converged = conv ? 1 : 0;
    return PIC_OK;
}

long long mg_total_cycles(pic_mg* mg) {
    long long t = 0;
    if (mg) cudaMemcpy(&t, mg->m.N.total, sizeof t, cudaMemcpyDeviceToHost);
    return t;
}

int mg_read_info(MgImpl& M, pic_mg_info* info);

// Host-driven solve: one launch per kernel and a synchronisation per cycle
// (the first min_cycles cycles run whatever the residual).
template <class T>
static int solve_eager(MgImpl& M, std::vector<LevelDev<T>>& lv, double* phi, const double* f, double tol,
                       int max_cycles, int min_cycles, cudaStream_t st) {
    launch_r0(M, lv, phi, f, tol, max_cycles, 1, cudaGraphConditionalHandle{}, 0, st);
    PIC_LAUNCH_CHECK();
    pic_mg_info info{};
    for (;;) {
        PIC_CUDA(cudaStreamSynchronize(st));
        PIC_TRY(mg_read_info(M, &info));
        if ((info.converged && info.cycles >= min_cycles) || info.cycles >= max_cycles) break;
        int count = 0;
        PIC_TRY(launch_cycle(M, lv, phi, f, tol, max_cycles, cudaGraphConditionalHandle{}, 0, st, count));
        M.body_launches = count;
    }
    return PIC_OK;
}

int mg_launch(MgImpl& M, double* phi, const double* f, double tol, int max_cycles, int min_cycles, cudaStream_t st) {
    if (M.dst) return launch_dst(M, phi, f, tol, max_cycles, st);
    if (M.o.launch_mode == PIC_MG_CLUSTER && M.cluster_ok) return launch_cluster(M, phi, f, tol, max_cycles, st);
    if (M.o.launch_mode == PIC_MG_PERSISTENT)
        return M.precision == PIC_MG_MIXED ? launch_persistent(M, M.lf, phi, f, tol, max_cycles, st)
                                           : launch_persistent(M, M.ld, phi, f, tol, max_cycles, st);
    if (M.o.launch_mode == PIC_MG_HOST_LOOP)
        return M.precision == PIC_MG_MIXED ? solve_eager(M, M.lf, phi, f, tol, max_cycles, min_cycles, st)
                                           : solve_eager(M, M.ld, phi, f, tol, max_cycles, min_cycles, st);
    PIC_TRY(ensure_graph(M, phi, f, tol, max_cycles, min_cycles));
    PIC_CUDA(cudaGraphLaunch(M.exec, st));
    return PIC_OK;
}

int mg_solve(MgImpl& M, double* phi, const double* f, double tol, int max_cycles, pic_mg_info* info,
             cudaStream_t st) {
    PIC_TRY(mg_launch(M, phi, f, tol, max_cycles, 0, st));
    PIC_CUDA(cudaStreamSynchronize(st));
    pic_mg_info loc{};
    PIC_TRY(mg_read_info(M, &loc));
    const bool one_kernel = M.o.launch_mode == PIC_MG_PERSISTENT || (M.o.launch_mode == PIC_MG_CLUSTER && M.cluster_ok);
    M.launches += M.dst ? 4 : 1 + (one_kernel ? 0 : (long long)(loc.cycles) * M.body_launches);
    if (info) *info = loc;
    if (!loc.converged)
        return fail(PIC_ERR_NOT_CONVERGED, "multigrid: relative residual %.3e after %d cycles (tol %.1e)", loc.rel_res,
                    loc.cycles, tol);
    return PIC_OK;
}

long long mg_launches(pic_mg* mg) { return mg ? mg->m.launches : 0; }
int mg_body_launches(pic_mg* mg) {
    if (!mg) return 0;
    const MgImpl& M = mg->m;
    const bool one_kernel = M.dst || M.o.launch_mode == PIC_MG_PERSISTENT ||
                            (M.o.launch_mode == PIC_MG_CLUSTER && M.cluster_ok);
    return one_kernel ? 0 : M.body_launches;
}
// Kernels a solve runs besides its V-cycles: the residual, or the three
// sine-transform kernels and the residual.
int mg_fixed_launches(pic_mg* mg) { return mg && mg->m.dst ? 4 : 1; }
int mg_capture_into(pic_mg* mg, double* phi, const double* f, double tol, int max_cycles, int min_cycles,
                    cudaStream_t st) {
    return mg_capture(mg->m, phi, f, tol, max_cycles, min_cycles, st);
}
bool mg_uses_graph(pic_mg* mg) { return mg->m.o.launch_mode != PIC_MG_HOST_LOOP; }
bool mg_is_rz(pic_mg* mg) { return mg->m.rz; }
int mg_launch_graph(pic_mg* mg, double* phi, const double* f, double tol, int max_cycles, int min_cycles,
                    cudaStream_t st) {
    return mg_launch(mg->m, phi, f, tol, max_cycles, min_cycles, st);
}
int mg_info(pic_mg* mg, pic_mg_info* info) { return mg_read_info(mg->m, info); }
const int* mg_device_converged(pic_mg* mg) { return mg->m.N.converged; }

// The tile geometry of S sweeps (pic_mg_tile_geometry).
template <int S>
int tile_geometry(int* out) {
    const int g[] = {kMgTile,
                     DownGeom<S>::H,      DownGeom<S>::W,
                     UpGeom<S>::H,        UpGeom<S>::W,        UpGeom<S>::CW,
                     UpGeom<S, true>::H,  UpGeom<S, true>::W,  UpGeom<S, true>::CW,
                     Down2Geom<S>::HC,    Down2Geom<S>::WC,    Down2Geom<S>::HF,    Down2Geom<S>::WF,
                     Up2Geom<S>::HF,      Up2Geom<S>::WF,      Up2Geom<S>::CWF,     Up2Geom<S>::WC,
                     Up2Geom<S>::CWC};
    static_assert(sizeof(g) / sizeof(g[0]) == PIC_MG_GEOMETRY_VALUES, "geometry table");
    for (int k = 0; k < PIC_MG_GEOMETRY_VALUES; ++k) out[k] = g[k];
    return PIC_OK;
}
}  // namespace pic

using namespace pic;

extern "C" {

int pic_mg_create(int nx, int ny, double dx, double dy, const uint8_t* h_dirichlet, const pic_mg_options* opts,
                  pic_mg** out) {
    clear_error();
    return mg_create(nx, ny, dx, dy, h_dirichlet, opts, out);
}

int pic_mg_effective_launch_mode(pic_mg* mg, int* mode) {
    clear_error();
    if (!mg || !mode) return fail(PIC_ERR_BAD_ARG, "pic_mg_effective_launch_mode: bad arguments");
    const MgImpl& M = mg->m;
    *mode = (M.o.launch_mode == PIC_MG_CLUSTER && !M.cluster_ok) ? int(PIC_MG_GRAPH_LOOP) : M.o.launch_mode;
    if (M.dst) *mode = PIC_MG_DST;
    return PIC_OK;
}

int pic_mg_destroy(pic_mg* mg) {
    clear_error();
    if (!mg) return PIC_OK;
    cudaDeviceSynchronize();
    mg_release(mg);
    return PIC_OK;
}

int pic_mg_solve(pic_mg* mg, double* d_phi, const double* d_f, double tol, int max_cycles, pic_mg_info* info,
                 void* stream) {
    clear_error();
    if (!mg || !d_phi || !d_f || !(tol > 0) || max_cycles < 0) return fail(PIC_ERR_BAD_ARG, "pic_mg_solve: bad arguments");
    return mg_solve(mg->m, d_phi, d_f, tol, max_cycles, info, as_stream(stream));
}

int pic_mg_solve_async(pic_mg* mg, double* d_phi, const double* d_f, double tol, int cycles, void* stream) {
    clear_error();
    if (!mg || !d_phi || !d_f || !(tol > 0) || cycles < 0)
        return fail(PIC_ERR_BAD_ARG, "pic_mg_solve_async: bad arguments");
    return mg_launch(mg->m, d_phi, d_f, tol, cycles, 0, as_stream(stream));
}

int pic_mg_tile_geometry(int sweeps, int* out) {
    clear_error();
    if (!out) return fail(PIC_ERR_BAD_ARG, "pic_mg_tile_geometry: out is NULL");
    switch (sweeps) {
        case 1: return pic::tile_geometry<1>(out);
        case 2: return tile_geometry<2>(out);
        case 3: return tile_geometry<3>(out);
        case 4: return tile_geometry<4>(out);
        case 5: return tile_geometry<5>(out);
        case 6: return tile_geometry<6>(out);
        case 7: return tile_geometry<7>(out);
        case 8: return tile_geometry<8>(out);
        default: return fail(PIC_ERR_BAD_ARG, "pic_mg_tile_geometry: sweeps %d outside 1..8", sweeps);
    }
}

int pic_mg_set_wait_limit(pic_mg* mg, long long polls) {
    clear_error();
    if (!mg) return fail(PIC_ERR_BAD_ARG, "pic_mg_set_wait_limit: mg is NULL");
    mg->m.wait_polls = polls < 0 ? kBarrierPolls : (unsigned long long)polls;
    return PIC_OK;
}

int pic_mg_read_info(pic_mg* mg, double tol, pic_mg_info* info) {
    clear_error();
    (void)tol;
    if (!mg || !info) return fail(PIC_ERR_BAD_ARG, "pic_mg_read_info: bad arguments");
    PIC_CUDA(cudaDeviceSynchronize());
    return mg_read_info(mg->m, info);
}

}  // extern "C"
