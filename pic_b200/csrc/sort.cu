// Deterministic cell sort: the replacement of Particles2D.sort_particles_sparse
// (src/Particles.py:550-632), whose atomic slot claims give a run-to-run
// varying order.  Here the order is a stable least-significant-digit radix
// sort of tile-major cell keys, in as few passes of at most 10-bit digits as
// the key width allows (19 bits at 513^2: two passes of 10 and 9 bits); each
// pass is a stable counting sort over G CTAs (three per SM), each owning a
// contiguous index range:
//   upsweep    per-CTA digit histograms (one shared-memory increment per
//              distinct digit and warp: the keys are nearly sorted)
//   scan_rows  one warp per digit: exclusive scan of that digit's counts over
//              the CTAs, and the digit's total
//   downsweep  the digits' bases (exclusive scan of the totals), then stable
//              ranks inside each 4096-key sub-tile (warp match_any in index
//              order), scattered to their global slots
// then the first slot of every tile, from the sorted keys.  Dead particles
// (NaN position) get the largest key and are dropped.
#include <cuda.h>

#include <algorithm>
#include <atomic>
#include <mutex>
#include <vector>

#include "sort_internal.cuh"

namespace pic {

constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kSortIpt = 16;
constexpr int kSortSub = kSortThreads * kSortIpt;
constexpr int kRadixMax = 1 << kSortDigitMax;
constexpr int kSortCtasPerSm = 3;  // the downsweep holds 80 registers a thread: three CTAs fit an SM

__global__ void k_sort_keys(const float* __restrict__ x, const float* __restrict__ y, const int* __restrict__ n_dev,
                            int ncx, int ncy, int tile, int tiles_x, uint32_t dead_key, uint32_t* __restrict__ keys,
                            uint32_t* __restrict__ vals, int* __restrict__ live) {
    const int n = n_dev[0];
    int mine = 0;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        const uint32_t k = tile_key(x[p], y[p], ncx, ncy, tile, tiles_x, dead_key);
        keys[p] = k;
        vals[p] = uint32_t(p);
        mine += k != dead_key;
    }
    mine = __reduce_add_sync(0xffffffffu, mine);
    if ((threadIdx.x & 31) == 0 && mine) atomicAdd(live, mine);
}

__device__ __forceinline__ void cta_range(int n, int G, int g, int& b, int& e) {
    const int per = (n + G - 1) / G;
    b = min(n, g * per);
    e = min(n, b + per);
}

__global__ void __launch_bounds__(kSortThreads) k_upsweep(const uint32_t* __restrict__ keys,
                                                          const int* __restrict__ n_dev, int shift, int bits, int G,
                                                          int* __restrict__ cnt) {
    __shared__ int h[kRadixMax];
    const int radix = 1 << bits;
    const uint32_t mask = uint32_t(radix - 1);
    for (int d = threadIdx.x; d < radix; d += blockDim.x) h[d] = 0;
    __syncthreads();
    int b, e;
    cta_range(n_dev[0], G, blockIdx.x, b, e);
    const int lane = threadIdx.x & 31;
    // keys are nearly sorted, so a warp's 32 digits are mostly equal: one
    // shared-memory increment per distinct digit and warp.  A thread loads
    // kSortIpt keys before it uses the first, so that the loads overlap.
    for (int base = b; base < e; base += kSortSub) {
        uint32_t k[kSortIpt];
#pragma unroll
        for (int it = 0; it < kSortIpt; ++it) {
            const int i = base + it * kSortThreads + int(threadIdx.x);
            k[it] = i < e ? __ldg(keys + i) : 0xffffffffu;
        }
#pragma unroll
        for (int it = 0; it < kSortIpt; ++it) {
            const int i = base + it * kSortThreads + int(threadIdx.x);
            const int d = i < e ? int((k[it] >> shift) & mask) : kRadixMax;
            const unsigned peers = __match_any_sync(0xffffffffu, d);
            if (d < kRadixMax && lane == __ffs(peers) - 1) atomicAdd(&h[d], __popc(peers));
        }
    }
    __syncthreads();
    for (int d = threadIdx.x; d < radix; d += blockDim.x) cnt[d * G + blockIdx.x] = h[d];
}

// Exclusive block scan of v (one value per thread, 256 threads); returns the
// thread's prefix and leaves the block total in *total.
__device__ __forceinline__ int block_exclusive_scan(int v, int* warp_tot, int* total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) warp_tot[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        const int w = lane < kSortWarps ? warp_tot[lane] : 0;
        int wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi += t;
        }
        if (lane < kSortWarps) warp_tot[lane] = wi - w;
        if (lane == kSortWarps - 1) *total = wi;
    }
    __syncthreads();
    const int r = warp_tot[warp] + incl - v;
    __syncthreads();  // warp_tot may be reused
    return r;
}

// One warp per digit d: exclusive scan of cnt[d*G .. d*G+G) in place over the
// CTAs (32 counts at a time, carried), and the digit's total in tot[d].
__global__ void __launch_bounds__(kSortThreads) k_scan_rows(int* __restrict__ cnt, int G, int radix,
                                                            int* __restrict__ tot) {
    const int d = blockIdx.x * kSortWarps + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (d >= radix) return;
    int* row = cnt + long(d) * G;
    int carry = 0;
    for (int base = 0; base < G; base += 32) {
        const int i = base + lane;
        const int v = i < G ? row[i] : 0;
        int incl = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += t;
        }
        if (i < G) row[i] = carry + incl - v;
        carry += __shfl_sync(0xffffffffu, incl, 31);
    }
    if (lane == 0) tot[d] = carry;
}

__global__ void __launch_bounds__(kSortThreads) k_downsweep(const uint32_t* __restrict__ kin,
                                                            const uint32_t* __restrict__ vin,
                                                            uint32_t* __restrict__ kout, uint32_t* __restrict__ vout,
                                                            const int* __restrict__ n_dev, int shift, int bits, int G,
                                                            const int* __restrict__ offs,
                                                            const int* __restrict__ tot) {
    __shared__ int running[kRadixMax];
    __shared__ int wc[kSortWarps][kRadixMax];
    __shared__ int subtotal[kRadixMax];
    __shared__ int warp_tot[kSortWarps];
    __shared__ int total;
    const int radix = 1 << bits;
    const uint32_t mask = uint32_t(radix - 1);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    int b, e;
    cta_range(n_dev[0], G, blockIdx.x, b, e);
    {
        // the digits' global bases: exclusive scan of the totals (each thread
        // four consecutive digits), plus this CTA's offset within each digit
        constexpr int kPer = kRadixMax / kSortThreads;
        int v[kPer], sum = 0;
#pragma unroll
        for (int k = 0; k < kPer; ++k) {
            const int d = int(threadIdx.x) * kPer + k;
            v[k] = d < radix ? tot[d] : 0;
            sum += v[k];
        }
        int run = block_exclusive_scan(sum, warp_tot, &total);
#pragma unroll
        for (int k = 0; k < kPer; ++k) {
            const int d = int(threadIdx.x) * kPer + k;
            if (d < radix) running[d] = run + offs[d * G + blockIdx.x];
            run += v[k];
        }
    }
    for (int base = b; base < e; base += kSortSub) {
        for (int q = threadIdx.x; q < kSortWarps * radix; q += blockDim.x) wc[q >> bits][q & (radix - 1)] = 0;
        __syncthreads();
        uint32_t key[kSortIpt], val[kSortIpt];
        int rank[kSortIpt];
        // every load of the sub-tile issued before the ranking uses the first
#pragma unroll
        for (int it = 0; it < kSortIpt; ++it) {
            const int idx = base + warp * (32 * kSortIpt) + it * 32 + lane;
            const bool valid = idx < e;
            key[it] = valid ? __ldg(kin + idx) : 0u;
            val[it] = valid ? __ldg(vin + idx) : 0u;
        }
#pragma unroll
        for (int it = 0; it < kSortIpt; ++it) {
            const int idx = base + warp * (32 * kSortIpt) + it * 32 + lane;
            const bool valid = idx < e;
            const int d = valid ? int((key[it] >> shift) & mask) : kRadixMax;
            const unsigned peers = __match_any_sync(0xffffffffu, d);
            const int leader = __ffs(peers) - 1;
            int basecnt = 0;
            if (lane == leader && valid) {
                basecnt = wc[warp][d];
                wc[warp][d] = basecnt + __popc(peers);
            }
            basecnt = __shfl_sync(0xffffffffu, basecnt, leader);
            rank[it] = valid ? basecnt + __popc(peers & lt) : -1;
        }
        __syncthreads();
        for (int d = threadIdx.x; d < radix; d += blockDim.x) {
            int run = 0;
#pragma unroll
            for (int w = 0; w < kSortWarps; ++w) {
                const int t = wc[w][d];
                wc[w][d] = run;
                run += t;
            }
            subtotal[d] = run;
        }
        __syncthreads();
#pragma unroll
        for (int it = 0; it < kSortIpt; ++it) {
            if (rank[it] < 0) continue;
            const int d = int((key[it] >> shift) & mask);
            const int pos = running[d] + wc[warp][d] + rank[it];
            kout[pos] = key[it];
            vout[pos] = val[it];
        }
        __syncthreads();
        for (int d = threadIdx.x; d < radix; d += blockDim.x) running[d] += subtotal[d];
        __syncthreads();
    }
}

// First sorted slot of each tile (the lower bound of its first key; empty
// tiles get the next tile's start, the end the live count) and the live
// count: position k writes the starts of the tiles after its predecessor's,
// up to its own.
__global__ void k_tile_starts(const uint32_t* __restrict__ keys, const int* __restrict__ live, int ntiles, int tt,
                              int* __restrict__ tile_start, int* __restrict__ count_out) {
    const int n = *live;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k <= n; k += gridDim.x * blockDim.x) {
        if (k == n && count_out) *count_out = n;
        if (!tile_start) continue;
        const int t1 = k < n ? int(keys[k] / uint32_t(tt)) : ntiles;
        const int t0 = k > 0 ? int(keys[k - 1] / uint32_t(tt)) : -1;
        for (int t = t0 + 1; t <= t1; ++t) tile_start[t] = k;
    }
}

__global__ void k_gather5(const uint32_t* __restrict__ perm, const int* __restrict__ live,
                          const float* __restrict__ a0, const float* __restrict__ a1, const float* __restrict__ a2,
                          const float* __restrict__ a3, const float* __restrict__ a4, float* __restrict__ b0,
                          float* __restrict__ b1, float* __restrict__ b2, float* __restrict__ b3,
                          float* __restrict__ b4, uint32_t* __restrict__ perm_out) {
    const int n = *live;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const uint32_t s = perm[k];
        b0[k] = a0[s];
        b1[k] = a1[s];
        b2[k] = a2[s];
        b3[k] = a3[s];
        if (a4) b4[k] = a4[s];
        if (perm_out) perm_out[k] = s;
    }
}

// The permutation alone (no arrays gathered): its first *live entries.
__global__ void k_copy_perm(const uint32_t* __restrict__ perm, const int* __restrict__ live,
                            uint32_t* __restrict__ perm_out) {
    const int n = *live;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) perm_out[k] = perm[k];
}

__global__ void k_set_n(int* n_dev, int n) {
    n_dev[0] = n;
    n_dev[1] = 0;
}

__global__ void k_copy_n(int* n_dev, const int* src) {
    n_dev[0] = *src;
    n_dev[1] = 0;
}

int grid_blocks(long n, int threads);

int sort_geometry(int capacity, int nx, int ny, int tile, int max_ctas, SortImpl* S) {
    S->capacity = capacity;
    S->nx = nx;
    S->ny = ny;
    S->tile = tile;
    S->tiles_x = (nx - 1 + tile - 1) / tile;
    S->tiles_y = (ny - 1 + tile - 1) / tile;
    S->ntiles = S->tiles_x * S->tiles_y;
    const unsigned long long nkeys = (unsigned long long)S->ntiles * tile * tile;
    if (nkeys >= 0xffffffffull) return fail(PIC_ERR_BAD_ARG, "cell sort: grid too large for 32-bit keys");
    S->dead_key = uint32_t(nkeys);
    int bits = 0;
    while ((1ull << bits) <= nkeys) ++bits;
    // the fewest passes of at most kSortDigitMax bits, the widths as even as possible
    S->passes = (bits + kSortDigitMax - 1) / kSortDigitMax;
    int rem = bits;
    for (int p = 0; p < S->passes; ++p) {
        S->digit[p] = (rem + (S->passes - p) - 1) / (S->passes - p);
        rem -= S->digit[p];
    }
    S->G = std::max(1, std::min(max_ctas, div_up(capacity, kSortSub)));
    return PIC_OK;
}

int sorter_create(int capacity, int nx, int ny, int tile, SortImpl* S) {
    if (capacity < 1 || nx < 2 || ny < 2 || tile < 1) return fail(PIC_ERR_BAD_ARG, "pic_sorter_create: bad arguments");
    PIC_TRY(sort_geometry(capacity, nx, ny, tile, kSortCtasPerSm * num_sms(), S));
    const size_t bytes = sizeof(uint32_t) * size_t(capacity);
    for (uint32_t** p : {&S->k0, &S->k1, &S->v0, &S->v1}) {
        PIC_CUDA(cudaMalloc(p, bytes));
        S->allocs.push_back(*p);
    }
    PIC_CUDA(cudaMalloc(&S->cnt, sizeof(int) * kRadixMax * S->G));
    S->allocs.push_back(S->cnt);
    PIC_CUDA(cudaMalloc(&S->tot, sizeof(int) * kRadixMax));
    S->allocs.push_back(S->tot);
    PIC_CUDA(cudaMalloc(&S->n_dev, sizeof(int) * 2));
    S->allocs.push_back(S->n_dev);
    return PIC_OK;
}

void sorter_free(SortImpl* S) {
    for (void* p : S->allocs) cudaFree(p);
    S->allocs.clear();
}

// Radix passes over S.k0/S.v0 (filled by a key kernel; S.n_dev = {n, live}),
// then tile starts and the live count.  *perm receives the buffer holding the
// sorted source slots.
int sort_passes(SortImpl& S, int* tile_start, int* count_out, const uint32_t** perm, cudaStream_t st) {
    uint32_t *ki = S.k0, *vi = S.v0, *ko = S.k1, *vo = S.v1;
    int shift = 0;
    for (int p = 0; p < S.passes; ++p) {
        const int w = S.digit[p];
        k_upsweep<<<S.G, kSortThreads, 0, st>>>(ki, S.n_dev, shift, w, S.G, S.cnt);
        k_scan_rows<<<div_up(1 << w, kSortWarps), kSortThreads, 0, st>>>(S.cnt, S.G, 1 << w, S.tot);
        k_downsweep<<<S.G, kSortThreads, 0, st>>>(ki, vi, ko, vo, S.n_dev, shift, w, S.G, S.cnt, S.tot);
        std::swap(ki, ko);
        std::swap(vi, vo);
        shift += w;
    }
    k_tile_starts<<<grid_blocks(long(S.capacity) + 1, 256), 256, 0, st>>>(ki, S.n_dev + 1, S.ntiles,
                                                                           S.tile * S.tile, tile_start, count_out);
    *perm = vi;
    PIC_LAUNCH_CHECK();
    return PIC_OK;
}

int sort_set_n(SortImpl& S, const int* d_n, cudaStream_t st) {
    k_copy_n<<<1, 1, 0, st>>>(S.n_dev, d_n);
    PIC_LAUNCH_CHECK();
    return PIC_OK;
}

// Sorts the live particles of [0, *d_n) (device count); see pic_sort.
int sort_run(SortImpl& S, const int* d_n, const float* x, const float* y, const float* vx, const float* vy,
             const float* vz, float* xo, float* yo, float* vxo, float* vyo, float* vzo, uint32_t* perm_out,
             int* count_out, int* tile_start, cudaStream_t st) {
    PIC_TRY(sort_set_n(S, d_n, st));
    const int cap = S.capacity;
    k_sort_keys<<<grid_blocks(cap, 256), 256, 0, st>>>(x, y, S.n_dev, S.nx - 1, S.ny - 1, S.tile, S.tiles_x,
                                                       S.dead_key, S.k0, S.v0, S.n_dev + 1);
    const uint32_t* perm = nullptr;
    PIC_TRY(sort_passes(S, tile_start, count_out, &perm, st));
    if (xo) k_gather5<<<grid_blocks(cap, 256), 256, 0, st>>>(perm, S.n_dev + 1, x, y, vx, vy, vz, xo, yo, vxo, vyo,
                                                             vzo, perm_out);
    else if (perm_out)
        k_copy_perm<<<grid_blocks(cap, 256), 256, 0, st>>>(perm, S.n_dev + 1, perm_out);
    PIC_LAUNCH_CHECK();
    return PIC_OK;
}

// ---- sort without allocation: scratch in a fixed device array -----------------------
//
// pic_sort_static keeps its scratch (key and slot ping-pong buffers, the
// digit-count table and the count pair) in one file-scope device array of
// kStaticSortBytes, which every GPU that loads the library holds until the
// process exits.  Every call shares it: calls that overlap on the GPU race.
// The first call on a device, with that device current, looks up the array's
// address (cudaGetSymbolAddress) and caches it with the device's context (a
// call after a device reset looks it up again); that first call should come
// before any stream capture.
constexpr int kStaticSortCtas = 256;  // upper bound of the radix passes' CTA count
constexpr size_t kStaticSortKeyBytes = sizeof(uint32_t) * size_t(PIC_SORT_STATIC_MAX);
constexpr size_t kStaticSortCntBytes = sizeof(int) * size_t(kRadixMax) * kStaticSortCtas;
constexpr size_t kStaticSortTotBytes = sizeof(int) * size_t(kRadixMax);
constexpr size_t kStaticSortBytes = 4 * kStaticSortKeyBytes + kStaticSortCntBytes + kStaticSortTotBytes + 256;

static __device__ __align__(256) unsigned char g_sort_scratch[kStaticSortBytes];

constexpr int kStaticMaxDevices = 64;

// Per device: the context the scratch address was looked up in, the address
// and the device's SM count.  A device reset (cudaDeviceReset) gives the
// device a new primary context in which the module, and the array, are
// loaded anew: the address is then looked up again.
struct StaticScratch {
    CUcontext ctx = nullptr;
    unsigned char* ptr = nullptr;
    int sms = 0;
};
static StaticScratch g_sort_scratch_at[kStaticMaxDevices];
static std::mutex g_sort_scratch_mu;

// Address of the current device's scratch array and its SM count.
static int static_scratch(unsigned char** out, int* sms) {
    int dev = 0;
    PIC_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kStaticMaxDevices)
        return fail(PIC_ERR_BAD_ARG, "pic_sort_static: device %d beyond the supported %d", dev, kStaticMaxDevices);
    PIC_CUDA(cudaFree(nullptr));  // makes the device's primary context current
    // cuCtxGetCurrent through the runtime's entry-point lookup, so that the
    // library does not link the driver library itself
    using CtxGetCurrent = CUresult (*)(CUcontext*);
    static CtxGetCurrent get_ctx = nullptr;
    if (!get_ctx) {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q{};
        PIC_CUDA(cudaGetDriverEntryPoint("cuCtxGetCurrent", &fn, cudaEnableDefault, &q));
        if (q != cudaDriverEntryPointSuccess || !fn)
            return fail(PIC_ERR_CUDA, "pic_sort_static: cuCtxGetCurrent not found");
        get_ctx = reinterpret_cast<CtxGetCurrent>(fn);
    }
    CUcontext ctx = nullptr;
    if (get_ctx(&ctx) != CUDA_SUCCESS || !ctx)
        return fail(PIC_ERR_CUDA, "pic_sort_static: no current context on device %d", dev);
    std::lock_guard<std::mutex> lock(g_sort_scratch_mu);
    StaticScratch& S = g_sort_scratch_at[dev];
    if (S.ctx != ctx || !S.ptr) {
        void* addr = nullptr;
        PIC_CUDA(cudaGetSymbolAddress(&addr, g_sort_scratch));
        int n = 0;
        PIC_CUDA(cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev));
        S.ctx = ctx;
        S.ptr = static_cast<unsigned char*>(addr);
        S.sms = n;
    }
    *out = S.ptr;
    *sms = S.sms;
    return PIC_OK;
}

}  // namespace pic

struct pic_sorter {
    pic::SortImpl s;
};

using namespace pic;

extern "C" {

int pic_sorter_create(int capacity, int nx, int ny, int tile, pic_sorter** out) {
    clear_error();
    if (!out) return fail(PIC_ERR_BAD_ARG, "pic_sorter_create: out is NULL");
    pic_sorter* s = new pic_sorter;
    const int st = sorter_create(capacity, nx, ny, tile, &s->s);
    if (st != PIC_OK) {
        sorter_free(&s->s);
        delete s;
        return st;
    }
    *out = s;
    return PIC_OK;
}

int pic_sorter_destroy(pic_sorter* s) {
    clear_error();
    if (!s) return PIC_OK;
    sorter_free(&s->s);
    delete s;
    return PIC_OK;
}

int pic_sort(pic_sorter* s, const float* d_x, const float* d_y, const float* d_vx, const float* d_vy,
             const float* d_vz, int n, float* d_x_out, float* d_y_out, float* d_vx_out, float* d_vy_out,
             float* d_vz_out, uint32_t* d_perm, int* d_count_out, int* d_tile_start, void* stream) {
    clear_error();
    if (!s || n < 0 || n > s->s.capacity || !d_x || !d_y)
        return fail(PIC_ERR_BAD_ARG, "pic_sort: bad arguments (n=%d, capacity=%d)", n, s ? s->s.capacity : 0);
    if (d_x_out && (!d_y_out || !d_vx_out || !d_vy_out || !d_vx || !d_vy || (d_vz && !d_vz_out)))
        return fail(PIC_ERR_BAD_ARG, "pic_sort: output arrays incomplete");
    cudaStream_t st = as_stream(stream);
    k_set_n<<<1, 1, 0, st>>>(s->s.n_dev, n);
    // sort_run copies the count from a device int; n_dev itself holds it here
    return sort_run(s->s, s->s.n_dev, d_x, d_y, d_vx, d_vy, d_vz, d_x_out, d_y_out, d_vx_out, d_vy_out, d_vz_out,
                    d_perm, d_count_out, d_tile_start, st);
}

int pic_sort_static(const float* d_x, const float* d_y, const float* d_vx, const float* d_vy, const float* d_vz,
                    int n, int nx, int ny, int tile, float* d_x_out, float* d_y_out, float* d_vx_out,
                    float* d_vy_out, float* d_vz_out, uint32_t* d_perm, int* d_count_out, int* d_tile_start,
                    void* stream) {
    clear_error();
    if (n < 0 || n > PIC_SORT_STATIC_MAX)
        return fail(PIC_ERR_BAD_ARG, "pic_sort_static: n=%d outside [0, %d] (the fixed scratch holds %d slots)", n,
                    PIC_SORT_STATIC_MAX, PIC_SORT_STATIC_MAX);
    if (!d_x || !d_y || nx < 2 || ny < 2 || tile < 1)
        return fail(PIC_ERR_BAD_ARG, "pic_sort_static: bad arguments");
    if (d_x_out && (!d_y_out || !d_vx_out || !d_vy_out || !d_vx || !d_vy || (d_vz && !d_vz_out)))
        return fail(PIC_ERR_BAD_ARG, "pic_sort_static: output arrays incomplete");
    // the geometry and passes of sorter_create, without its allocations
    unsigned char* base = nullptr;
    int sms = 0;
    PIC_TRY(static_scratch(&base, &sms));
    SortImpl S;
    PIC_TRY(sort_geometry(std::max(n, 1), nx, ny, tile, std::min(kSortCtasPerSm * sms, kStaticSortCtas), &S));
    S.k0 = reinterpret_cast<uint32_t*>(base);
    S.k1 = reinterpret_cast<uint32_t*>(base + kStaticSortKeyBytes);
    S.v0 = reinterpret_cast<uint32_t*>(base + 2 * kStaticSortKeyBytes);
    S.v1 = reinterpret_cast<uint32_t*>(base + 3 * kStaticSortKeyBytes);
    S.cnt = reinterpret_cast<int*>(base + 4 * kStaticSortKeyBytes);
    S.tot = reinterpret_cast<int*>(base + 4 * kStaticSortKeyBytes + kStaticSortCntBytes);
    S.n_dev = reinterpret_cast<int*>(base + 4 * kStaticSortKeyBytes + kStaticSortCntBytes + kStaticSortTotBytes);
    cudaStream_t st = as_stream(stream);
    // n_dev = {n, 0}: the live count starts at zero whatever the last call left
    k_set_n<<<1, 1, 0, st>>>(S.n_dev, n);
    return sort_run(S, S.n_dev, d_x, d_y, d_vx, d_vy, d_vz, d_x_out, d_y_out, d_vx_out, d_vy_out, d_vz_out, d_perm,
                    d_count_out, d_tile_start, st);
}

}  // extern "C"
