// The fused time step (SimulationManager._init_step / _step,
// src/simulation.py:622-660).
//
// Reference order per step: drift (update_R), deposit, solve, E, kick
// (update_V), MCC.  Moving the loop boundary gives the same operator sequence
// with one particle pass per step:
//     [kick + MCC + drift + absorb + deposit]  ->  RHS  ->  multigrid  ->  E
// The kick and MCC of the last step stay pending until the next step or
// pic_sim_sync, so after a sync the state equals the reference's.
//
// Particle pass: persistent CTAs take work items (species, tile, [begin,end))
// from an atomic counter.  Items of sorted particles belong to one tile of
// tile x tile cells: the CTA stages the tile's E field (with a halo) and a
// charge accumulator (2^-19 fixed point) in shared memory, pushes the item's
// particles and flushes the charge tile once with global atomics.  Particles
// that left the staged region since the last sort gather from and deposit to
// global memory directly.  Particles born since the last sort are processed
// as untiled items.  Null-collision candidates are kicked in the pass and
// listed with their kicked state; k_collide finishes them (collision,
// products, drift, deposit) after the pass.  k_push, one ring of bulk copies
// per block, is the default (the fastest measured); three more streaming
// schemes with the same per-particle arithmetic are kept as options
// (k_push_pipe, k_push_warp with and without warp-aggregated deposits).
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstddef>
#include <vector>

#include <cuda.h>

#include "mcc_host.cuh"
#include "sort_internal.cuh"

namespace pic {

int grid_blocks(long n, int threads);
int launch_update_E(const double* phi, float* Ex, float* Ey, float2* E2, int ep, int nx, int ny, double dx, double dy,
                    cudaStream_t st, bool axis);
int launch_form_rhs(const float* rho, const uint8_t* dirichlet, double eps0, double* f, float* snapshot, float* zero,
                    double* phi, double* phi_prev, long G, cudaStream_t st, const double* rowf, int nx);
int mg_create(int nx, int ny, double dx, double dy, const uint8_t* h_mask, const pic_mg_options* opts, pic_mg** out);
int mg_body_launches(pic_mg* mg);
int mg_fixed_launches(pic_mg* mg);
long long mg_total_cycles(pic_mg* mg);
int mg_capture_into(pic_mg* mg, double* phi, const double* f, double tol, int max_cycles, int min_cycles,
                    cudaStream_t st);
int mg_launch_graph(pic_mg* mg, double* phi, const double* f, double tol, int max_cycles, int min_cycles,
                    cudaStream_t st);
int mg_info(pic_mg* mg, pic_mg_info* info);
int diagnostics(const DiagSpecies* sp, const double* mass, const double* np2c, int ns, const double* phi,
                const float* rho, const float* Ex, const float* Ey, int nx, int ny, double dx, double dy, double eps0,
                const double* rowv, double* scratch, pic_sim_diag* out, cudaStream_t st);
size_t diagnostics_scratch_doubles();
bool mg_uses_graph(pic_mg* mg);

constexpr int kPushThreads = 256;
constexpr int kPushP = 3;  // particles per thread per chunk (odd: conflict-free blocked access to shared memory;
                           // 3 keeps a CTA at 45 KB of shared memory, so that four fit on an SM)
// Warp 0 takes no particles: its thread 0 runs the ring (bulk stores, the next
// load, work claims) while warps 1-7 push, so the per-chunk barrier does not
// wait on that bookkeeping (7 % faster than spreading the chunk over all warps).
constexpr int kChunk = (kPushThreads - 32) * kPushP;
constexpr int kBufStride = kChunk + 8;  // floats per array per buffer: room for the 16-byte alignment window
// candidate-bit words staged with a chunk: its kChunk / 32 words, widened to
// 16-byte boundaries at both ends
constexpr int kCbWords = 32;
static_assert(kChunk / 32 + 8 <= kCbWords, "a chunk's candidate words fit their stage");
// collision candidates a k_push block lists in shared memory during a work
// unit and appends to the global list at the unit's end (about P_null * 8160
// per unit: 20 at the 513^2 workload's electrons); more go to it one by one
constexpr int kCandUnit = 64;
constexpr int kUnitMax = 8160;          // particles per work unit (one E tile staging, one charge flush)
// The charge tile accumulates CIC weights as unsigned fixed point, 2^-19 per
// unit: integer shared-memory atomics are native (float ones retry), the sum
// is independent of the order, and 8160 weights <= 1 stay below 2^32
// (8160 * 2^19 = 2^32 - 2^24).
constexpr float kFixScale = 524288.0f;  // 2^19
constexpr float kFixInv = 1.0f / 524288.0f;
constexpr int kHalo = 4;                // cells staged around a tile
constexpr int kArraySlack = 16;         // floats allocated past each species' capacity (bulk-copy window)
constexpr unsigned long long kWaitLimit = 1ull << 24;  // bounded mbarrier wait

// Device-resident per-species state (the sort swaps the buffers).
struct SpeciesState {
    float* cur[5];  // x, y, vx, vy, vz
    float* alt[5];
    int count;       // slots in use
    int sorted_end;  // slots covered by tile items
    int capacity;
    int stride;      // cur[k] = cur[0] + k * stride (the five arrays share one allocation)
};

struct SpeciesConst {
    float kq;          // q/m dt (times the kick factor)
    float dtdx, dtdy;  // dt/dx, dt/dy
    float scale;       // q np2c / (dx dy)
};

struct alignas(64) PushArgs {
    CUtensorMap emap;  // E (interleaved Ex, Ey as 8-byte elements, nx x ny, rows ep apart): the E tiles' bulk loads
    SpeciesState* state;
    SpeciesConst sp[PIC_MAX_SPECIES];
    const int4* items;
    const int* n_items;
    int* item_next;
    const float2* E;
    float* rho;
    int nx, ny, tile, tiles_x, rw;
    int ep;  // row pitch of E in nodes (nx rounded up to even: 16-byte row strides for the tensor map)
    int ew;  // row width of k_push_warp's E tile (rw rounded up to even)
    int do_kick, do_mcc, do_drift, do_deposit;
    const MccDev* mcc;  // device copy of the tables' descriptor
    uint2 key;
    const uint32_t* step;
    const unsigned* cbits[PIC_MAX_SPECIES];  // null-collision candidate bit per slot (k_mcc_bits), or null
    const unsigned *vbits, *hbits;           // internal electrode edges (hits_electrode), when `electrodes`
    int electrodes;
    int rz;           // r-z geometry: drift_rz (y radial, vz azimuthal)
    int2* cand;          // collision candidates (species, slot), finished by k_collide after the pass
    float4* cand_state;  // their kicked (x, y, vx, vy)
    int* cand_count;
    int cand_cap;
    unsigned long long* ctr;
    int* error;  // set when a bounded wait gives up
    unsigned long long wait_limit;  // polls of a chunk wait (kWaitLimit unless changed)
    // one pass over an ensemble's members (k_push<..., true>): the members'
    // own arguments, and the first work item of each member in the pass's
    // flat item numbering (nmembers + 1 entries, the last the total)
    const PushArgs* members;
    const int* member_items;
    int nmembers;
};

// The arguments of member m: the pass's own unless it runs an ensemble.
template <bool ENS>
__device__ __forceinline__ const PushArgs& member(const PushArgs& A, int m) {
    if constexpr (ENS) return A.members[m];
    else return A;
}
// A chunk's species field holds the species plus 256 x the ensemble member.
template <bool ENS>
__device__ __forceinline__ int chunk_species(int s) { return ENS ? (s & 0xff) : s; }
template <bool ENS>
__device__ __forceinline__ int chunk_member(int s) { return ENS ? (s >> 8) : 0; }

// ---- TMA bulk copies and mbarriers (inline PTX, no multicast) -------------------

__device__ __forceinline__ unsigned smem_u32(const void* p) { return unsigned(__cvta_generic_to_shared(p)); }

__device__ __forceinline__ void mbar_init(unsigned long long* m, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(m)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_expect_tx(unsigned long long* m, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(m)), "r"(bytes) : "memory");
}

__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, unsigned long long* m) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(m))
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(unsigned long long* m, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(smem_u32(m)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Waits for the phase with the given parity; false after `limit` polls.
__device__ __forceinline__ bool mbar_wait(unsigned long long* m, unsigned parity, unsigned long long limit) {
    for (unsigned long long k = 0; k < limit; ++k)
        if (mbar_try_wait(m, parity)) return true;
    return false;
}

// One chunk of a work unit, as the producer thread hands it to the CTA.
struct ChunkDesc {
    int valid;
    int s, tile, b, e;  // species (+ 256 x the ensemble member), tile (-1: untiled), slot range of the chunk
    int unit_e;         // end of the unit's slot range
    int first;          // first chunk of its unit
};

// The chunk's first candidate-bit word, rounded down to a 16-byte boundary.
__device__ __forceinline__ int cb_word0(int b) { return (b >> 5) & ~3; }

// Issues the bulk copies of slots [b, e) of species s into `buf` (one
// thread), and, when `cbuf` is given and the species collides, the words of
// its candidate bits that cover the slots into `cbuf`.
template <bool ENS>
__device__ __forceinline__ void issue_chunk(const PushArgs& A, const ChunkDesc& c, float* buf, unsigned* cbuf,
                                            unsigned long long* bar) {
    const int a0 = c.b & ~3, a1 = (c.e + 3) & ~3;
    const unsigned bytes = unsigned(a1 - a0) * 4u;
    const PushArgs& M = member<ENS>(A, chunk_member<ENS>(c.s));
    const int sp = chunk_species<ENS>(c.s);
    const unsigned* const cb = (cbuf && M.do_mcc) ? M.cbits[sp] : nullptr;
    const int w0 = cb_word0(c.b), w1 = (((c.e - 1) >> 5) + 4) & ~3;
    const unsigned cbytes = cb ? unsigned(w1 - w0) * 4u : 0u;
    // x, y, vx, vy: vz is touched only by collision candidates (finish_candidate)
    mbar_expect_tx(bar, 4u * bytes + cbytes);
    const SpeciesState& S = M.state[sp];
#pragma unroll
    for (int k = 0; k < 4; ++k) bulk_g2s(buf + k * kBufStride, S.cur[k] + a0, bytes, bar);
    if (cb) bulk_g2s(cbuf, cb + w0, cbytes, bar);
}

// The chunk after `c`: the rest of its unit, else the first chunk of a newly
// claimed unit (one thread).  In an ensemble pass the claimed number runs over
// every member's items: the member is found in member_items.
template <bool ENS>
__device__ __forceinline__ ChunkDesc next_chunk(const PushArgs& A, const ChunkDesc& c, int n_items) {
    ChunkDesc d;
    if (c.valid && c.e < c.unit_e) {
        d = c;
        d.b = c.e;
        d.e = min(c.unit_e, c.e + kChunk);
        d.first = 0;
        return d;
    }
    int it = atomicAdd(A.item_next, 1);
    d.valid = it < n_items;
    if (!d.valid) return d;
    int m = 0;
    if constexpr (ENS) {
        int lo = 0, hi = A.nmembers - 1;  // the last member whose first item is <= it
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (__ldg(A.member_items + mid) <= it) lo = mid;
            else hi = mid - 1;
        }
        m = lo;
        it -= __ldg(A.member_items + lo);
    }
    const int4 u = member<ENS>(A, m).items[it];
    d.s = u.x + (m << 8);
    d.tile = u.y;
    d.b = u.z;
    d.unit_e = u.w;
    d.e = min(u.w, u.z + kChunk);
    d.first = 1;
    return d;
}

// Null-collision candidates of a step, one bit per slot: one thread per
// 256-slot segment draws the segment's geometric gaps (mcc_mark_segment) into
// its eight words.  The draws depend only on (segment, step, species), not on
// the particles, so the mask is ready before the particle pass reads it.
__global__ void __launch_bounds__(256) k_mcc_bits(const MccDev* __restrict__ M, int nspecies,
                                                  const uint32_t* __restrict__ step_ptr, uint2 key,
                                                  unsigned* const* __restrict__ bits, const int* __restrict__ nseg) {
    __shared__ unsigned w[256 * (kMccSegment / 32)];
    constexpr int kW = kMccSegment / 32;
    const uint32_t step = *step_ptr;
    int g = blockIdx.x * blockDim.x + threadIdx.x, s = 0;
    while (s < nspecies && g >= nseg[s]) g -= nseg[s++];
    unsigned* mine = w + threadIdx.x * kW;
#pragma unroll
    for (int q = 0; q < kW; ++q) mine[q] = 0u;
    if (s < nspecies && M->sp[s].nproc > 0) {
        const int b = g * int(kMccSegment);
        mcc_mark_segment(M->sp[s], uint32_t(s), long(g), INT_MAX, b, b + int(kMccSegment), step, key, mine);
    }
    if (s < nspecies) {
        unsigned* out = bits[s] + long(g) * kW;
#pragma unroll
        for (int q = 0; q < kW; ++q) out[q] = mine[q];
    }
}

// Asynchronous copies into shared memory (cp.async), completed per thread.
__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
// 8 bytes, or zeros when `bytes` is 0 (the source is then not read)
__device__ __forceinline__ void cp_async8(void* dst, const void* src, unsigned bytes) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(smem_u32(dst)), "l"(src), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }
// Waits until at most n (0..2) of this thread's copy groups are still in flight.
__device__ __forceinline__ void cp_async_wait_pending(int n) {
    if (n <= 0) asm volatile("cp.async.wait_group 0;" ::: "memory");
    else if (n == 1) asm volatile("cp.async.wait_group 1;" ::: "memory");
    else asm volatile("cp.async.wait_group 2;" ::: "memory");
}

// Stages the E tile of a unit's tile and zeroes its charge tile.  The E tile
// holds node pairs along x, et[q] = (E at node q, E at its east neighbour
// i1 = min(i + 1, nx - 1)), so that a particle reads its four E values with
// two 16-byte loads.  (The charge tile stays one word per node: 64-bit
// shared-memory atomics on pairs made the pass 1.7x slower, measured.)
__device__ __forceinline__ void stage_tile(const PushArgs& A, int tile, float4* et, unsigned* rt, int& ox, int& oy) {
    const int RW = A.rw;
    ox = (tile % A.tiles_x) * A.tile - kHalo;
    oy = (tile / A.tiles_x) * A.tile - kHalo;
    for (int q = threadIdx.x; q < RW * RW; q += kPushThreads) {
        const int gi = ox + q % RW, gj = oy + q / RW;
        float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
        if (gi >= 0 && gj >= 0 && gi < A.nx && gj < A.ny) {
            const long k = long(gj) * A.ep + gi;
            const float2 e0 = __ldg(A.E + k), e1 = __ldg(A.E + k + (gi + 1 < A.nx ? 1 : 0));
            v = make_float4(e0.x, e0.y, e1.x, e1.y);
        }
        et[q] = v;
        rt[q] = 0u;
    }
}

// stage_tile's E tile by asynchronous copies (two 8-byte copies per node
// pair, zeros outside the grid), committed as one group; the charge tile is
// left as the last flush zeroed it.  The caller waits (cp_async_wait_all)
// and meets the block at a barrier before the tile is read.
__device__ __forceinline__ void stage_etile_async(const PushArgs& A, int tile, float4* et, int& ox, int& oy) {
    const int RW = A.rw;
    ox = (tile % A.tiles_x) * A.tile - kHalo;
    oy = (tile / A.tiles_x) * A.tile - kHalo;
    for (int q = threadIdx.x; q < RW * RW; q += kPushThreads) {
        const int gi = ox + q % RW, gj = oy + q / RW;
        const bool in = gi >= 0 && gj >= 0 && gi < A.nx && gj < A.ny;
        const float2* p0 = in ? A.E + long(gj) * A.ep + gi : A.E;
        const float2* p1 = (in && gi + 1 < A.nx) ? p0 + 1 : p0;
        float* d = reinterpret_cast<float*>(et + q);
        cp_async8(d, p0, in ? 8u : 0u);
        cp_async8(d + 2, p1, in ? 8u : 0u);
    }
    cp_async_commit();
}

// Bulk copies from shared memory back to global memory (one bulk group per
// commit; wait_group.read N returns once at most N groups still read shared
// memory).
__device__ __forceinline__ void bulk_s2g(void* dst, const void* src, unsigned bytes) {
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst), "r"(smem_u32(src)),
                 "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_read1() { asm volatile("cp.async.bulk.wait_group.read 1;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

// Writes chunk c back from its buffer: the 16-byte-aligned middle of each
// array by bulk copies (one thread).  The slots outside it (fewer than 4 at
// each end) belong to neighbouring units on other CTAs' copies and go by
// plain stores (store_chunk_edges).
template <bool ENS>
__device__ __forceinline__ void store_chunk_bulk(const PushArgs& A, const ChunkDesc& c, const float* buf) {
    const int a0 = c.b & ~3, b4 = (c.b + 3) & ~3, e4 = c.e & ~3;
    if (e4 <= b4) return;
    const unsigned bytes = unsigned(e4 - b4) * 4u;
    const SpeciesState& S = member<ENS>(A, chunk_member<ENS>(c.s)).state[chunk_species<ENS>(c.s)];
    fence_proxy_async();  // the threads' shared-memory writes, visible to the bulk copy
#pragma unroll
    for (int k = 0; k < 4; ++k) bulk_s2g(S.cur[k] + b4, buf + k * kBufStride + (b4 - a0), bytes);
}

template <bool ENS>
__device__ __forceinline__ void store_chunk_edges(const PushArgs& A, const ChunkDesc& c, const float* buf, int tid) {
    if (tid >= 24) return;
    const int a0 = c.b & ~3, b4 = (c.b + 3) & ~3, e4 = c.e & ~3;
    const int k = tid / 6, j = tid % 6;
    const int slot = j < 3 ? c.b + j : max(e4, b4) + (j - 3);
    const int lim = j < 3 ? min(b4, c.e) : c.e;
    if (slot >= lim) return;
    member<ENS>(A, chunk_member<ENS>(c.s)).state[chunk_species<ENS>(c.s)].cur[k][slot] = buf[k * kBufStride + (slot - a0)];
}

// An ionisation product of this step's collisions, born at (x, y): its first
// drift with its own velocity, then, unless that takes it out of the domain
// or onto an electrode (it is then never stored), its slot at the end of its
// species and its deposit (global atomics).
__device__ __forceinline__ void place_product(const PushArgs& A, int s, float x, float y, float vx, float vy,
                                              float vz) {
    const SpeciesConst C = A.sp[s];
    if (A.do_drift) {
        const float x0 = x, y0 = y;
        if (A.rz) {
            drift_rz(x, y, vx, vy, vz, C.dtdx, C.dtdy);
        } else {
            x = __fmaf_rn(vx, C.dtdx, x);
            y = __fmaf_rn(vy, C.dtdy, y);
        }
        if (!(x >= 0.0f && x <= float(A.nx - 1) && y >= 0.0f && y <= float(A.ny - 1))) return;
        if (A.electrodes && hits_electrode(x0, y0, x, y, A.nx, A.ny, A.vbits, A.hbits)) return;
    }
    SpeciesState& S = A.state[s];
    const int slot = atomicAdd(&S.count, 1);
    if (slot >= S.capacity) {
        atomicSub(&S.count, 1);
        atomicAdd(A.ctr + kCtrDropped, 1ull);
        return;
    }
    S.cur[0][slot] = x;
    S.cur[1][slot] = y;
    S.cur[2][slot] = vx;
    S.cur[3][slot] = vy;
    S.cur[4][slot] = vz;
    atomicAdd(A.ctr + kCtrBorn + s, 1ull);
    if (A.do_deposit) {
        const Cic c = cic_weights(x, y, A.nx, A.ny);
        atomicAdd(A.rho + long(c.j0) * A.nx + c.i0, __fmul_rn(C.scale, c.w00));
        atomicAdd(A.rho + long(c.j0) * A.nx + c.i1, __fmul_rn(C.scale, c.w10));
        atomicAdd(A.rho + long(c.j1) * A.nx + c.i0, __fmul_rn(C.scale, c.w01));
        atomicAdd(A.rho + long(c.j1) * A.nx + c.i1, __fmul_rn(C.scale, c.w11));
    }
}

// The rest of a collision candidate's step, which the particle pass leaves
// after its kick: the null-collision test and scattering (mcc_collide), the
// ionisation products, then the drift, absorption and deposit (global
// atomics; a few candidates per thousand particles).  (x, y, vx, vy) is the
// kicked state; vz is read from the slot, which the pass does not touch.
__device__ __forceinline__ void finish_candidate(const PushArgs& A, const MccDev& MC, uint32_t step, int s, int p,
                                                 float x, float y, float vx, float vy) {
    const SpeciesState& S = A.state[s];
    const SpeciesConst C = A.sp[s];
    float vz = S.cur[4][p];
    const MccOutcome o = mcc_collide(MC, MC.sp[s], uint32_t(s), uint32_t(p), step, A.key, vx, vy, vz);
    if (o.overflow) atomicAdd(A.ctr + kCtrOverflow, 1ull);
    if (o.proc >= 0) {
        atomicAdd(A.ctr + kCtrCollisions + s * PIC_MAX_PROCESSES + o.proc, 1ull);
        if (o.born) {
            // born at the parent's position before its drift
            const MccSpeciesDev& M = MC.sp[s];
            place_product(A, M.born_e, x, y, o.be[0], o.be[1], o.be[2]);
            place_product(A, M.born_i, x, y, o.bi[0], o.bi[1], o.bi[2]);
        }
    }
    if (A.do_drift) {
        const float x0 = x, y0 = y;
        if (A.rz) {
            drift_rz(x, y, vx, vy, vz, C.dtdx, C.dtdy);
        } else {
            x = __fmaf_rn(vx, C.dtdx, x);
            y = __fmaf_rn(vy, C.dtdy, y);
        }
        if (!(x >= 0.0f && x <= float(A.nx - 1) && y >= 0.0f && y <= float(A.ny - 1))) {
            x = __int_as_float(0x7fc00000);
            y = x;
            atomicAdd(A.ctr + kCtrAbsorbed + s, 1ull);
        } else if (A.electrodes && hits_electrode(x0, y0, x, y, A.nx, A.ny, A.vbits, A.hbits)) {
            x = __int_as_float(0x7fc00000);
            y = x;
            atomicAdd(A.ctr + kCtrElectrode + s, 1ull);
        }
    }
    S.cur[0][p] = x;
    S.cur[1][p] = y;
    S.cur[2][p] = vx;
    S.cur[3][p] = vy;
    S.cur[4][p] = vz;
    if (A.do_deposit && is_live(x)) {
        const Cic w = cic_weights(x, y, A.nx, A.ny);
        atomicAdd(A.rho + long(w.j0) * A.nx + w.i0, __fmul_rn(C.scale, w.w00));
        atomicAdd(A.rho + long(w.j0) * A.nx + w.i1, __fmul_rn(C.scale, w.w10));
        atomicAdd(A.rho + long(w.j1) * A.nx + w.i0, __fmul_rn(C.scale, w.w01));
        atomicAdd(A.rho + long(w.j1) * A.nx + w.i1, __fmul_rn(C.scale, w.w11));
    }
}

constexpr int kStages = 3;  // chunk buffers: one loading, one in work, one draining to global memory

// Work units (species, tile, slot range) are claimed from an atomic counter
// and streamed through the CTA in chunks of kChunk particles over a ring of
// three shared-memory buffers: the bulk load of chunk k+1, the work on chunk
// k (results written back in place) and the bulk store of chunk k-1 overlap,
// with one CTA barrier per chunk (two more at the end of each unit, around
// the charge-tile flush).  The chunk after a non-final chunk is computed by
// every thread; only the first chunk of a new unit is published through
// shared memory, across the unit-end barrier.
// RZ: r-z geometry (drift_rz); a separate instance, so that the Cartesian
// pass carries none of it.  FULL: kick, drift and deposit all on (the step's
// pass), fixed at compile time.
template <bool RZ, bool FULL, bool ENS = false>
__global__ void __launch_bounds__(kPushThreads, 4) k_push(PushArgs A) {
    extern __shared__ __align__(128) unsigned char smem[];
    float* bufs = reinterpret_cast<float*>(smem);  // [kStages][4][kBufStride]
    unsigned* cbs = reinterpret_cast<unsigned*>(bufs + kStages * 4 * kBufStride);  // [kStages][kCbWords]
    // the tile side of the unit in work: an ensemble's members may differ
    // (A.rw is then their largest, which sizes shared memory)
    int RW = A.rw;
    float4* et = reinterpret_cast<float4*>(cbs + kStages * kCbWords);
    unsigned* rt = reinterpret_cast<unsigned*>(et + A.rw * A.rw);
    __shared__ __align__(8) unsigned long long bar[kStages];
    __shared__ ChunkDesc s_ch[kStages];
    __shared__ unsigned s_abs, s_cand, s_elec;
    // the unit's collision candidates: (species, slot) and kicked state
    __shared__ int2 s_cidx[kCandUnit];
    __shared__ float4 s_cst[kCandUnit];
    __shared__ int s_nc, s_nflush, s_cbase;
    const int tid = threadIdx.x;
    const int n_items = *A.n_items;
    if (tid == 0) {
        for (int k = 0; k < kStages; ++k) mbar_init(&bar[k], 1);
        fence_mbar_init();
        s_abs = 0;
        s_cand = 0;
        s_elec = 0;
        s_nc = 0;
        ChunkDesc none;
        none.valid = 0;
        const ChunkDesc c = next_chunk<ENS>(A, none, n_items);
        s_ch[0] = c;
        if (c.valid) issue_chunk<ENS>(A, c, bufs, cbs, &bar[0]);
    }
    __syncthreads();
    ChunkDesc ch = s_ch[0];
    ChunkDesc prev;  // the chunk processed before `ch`, still to be written back
    prev.valid = 0;
    unsigned phases = 0u;  // expected parity of each stage's mbarrier
    int cur = 0, ox = 0, oy = 0;
    // the charge tile starts at zero (every flush zeroes what it read)
    for (int q = tid; q < A.rw * A.rw; q += kPushThreads) rt[q] = 0u;
    if (ch.valid && ch.tile >= 0) {
        if constexpr (ENS) RW = member<ENS>(A, chunk_member<ENS>(ch.s)).rw;
        stage_tile(member<ENS>(A, chunk_member<ENS>(ch.s)), ch.tile, et, rt, ox, oy);
    }
    const bool do_kick = FULL || A.do_kick, do_drift = FULL || A.do_drift, do_deposit = FULL || A.do_deposit;
    // the unit's absorbed, candidate and electrode counts of this thread
    unsigned my_abs = 0, my_cand = 0, my_elec = 0;
    while (ch.valid) {
        const bool tiled = ch.tile >= 0;
        const int prv = cur == 0 ? kStages - 1 : cur - 1;
        const int nxt = cur == kStages - 1 ? 0 : cur + 1;
        const unsigned par = (phases >> cur) & 1u;
        const bool ok = mbar_wait(&bar[cur], par, A.wait_limit);
        phases ^= 1u << cur;
        if (__syncthreads_or(!ok)) {
            // give up on this launch: flag it, then wait (bounded) for the one
            // load in flight (the next chunk's load is issued only after a wait succeeds)
            if (tid == 0) {
                atomicExch(A.error, 1);
                mbar_wait(&bar[cur], par, kWaitLimit);
            }
            __syncthreads();
            break;
        }
        if (tid == 0) {
            // write back the previous chunk, then reuse the buffer of the one
            // before it (its store has been read) for the next chunk's load
            if (prev.valid) {
                store_chunk_bulk<ENS>(A, prev, bufs + prv * 4 * kBufStride);
                bulk_commit();
            }
            bulk_wait_read1();
            const ChunkDesc nc = next_chunk<ENS>(A, ch, n_items);
            s_ch[nxt] = nc;
            if (nc.valid) {
                fence_proxy_async();
                issue_chunk<ENS>(A, nc, bufs + nxt * 4 * kBufStride, cbs + nxt * kCbWords, &bar[nxt]);
            }
        }
        if (prev.valid) store_chunk_edges<ENS>(A, prev, bufs + prv * 4 * kBufStride, tid);
        const PushArgs& M = member<ENS>(A, chunk_member<ENS>(ch.s));  // this chunk's simulation
        const int s = chunk_species<ENS>(ch.s), b = ch.b, n = ch.e - ch.b;
        const int off = b & 3;
        float* const px = bufs + cur * 4 * kBufStride + off;
        float* const py = px + kBufStride;
        float* const pvx = py + kBufStride;
        float* const pvy = pvx + kBufStride;
        const SpeciesConst C = M.sp[s];
        // the chunk's candidate-bit words, staged with it (a species without
        // collision processes has no bits)
        const unsigned* const cbw = (M.do_mcc && M.cbits[s]) ? cbs + cur * kCbWords : nullptr;
        const int wb = cb_word0(b);
        // r-z: the azimuthal velocity is not staged; it is read and written in place
        float* const gvz = RZ ? M.state[s].cur[4] + b : nullptr;
        // the candidate bits of this thread's slots (at most two words), as a
        // 3-bit mask
        const int wt = tid - 32;  // particle lane (warp 0 has none)
        const int s0 = b + wt * kPushP, s_last = min(s0 + kPushP, b + n) - 1;
        unsigned cmask = 0u;
        if (wt >= 0 && cbw && s0 <= s_last) {
            const unsigned cw0 = cbw[(s0 >> 5) - wb];
            const unsigned cw1 = (s_last >> 5) != (s0 >> 5) ? cbw[(s_last >> 5) - wb] : 0u;
            cmask = __funnelshift_r(cw0, cw1, s0 & 31);
        }
        const unsigned tw = unsigned(RW - 1);  // staged tile: local cell index in [0, RW-2]
#pragma unroll
        for (int k = 0; k < kPushP; ++k) {
            const int l = wt * kPushP + k;
            if (wt < 0 || l >= n) break;
            const bool candidate = (cmask >> k) & 1u;
            float x = px[l], y = py[l];
            if (!is_live(x)) continue;
            float vx = pvx[l], vy = pvy[l];
            if (do_kick) {
                const Cic c = cic_weights(x, y, M.nx, M.ny);
                const int li = c.i0 - ox, lj = c.j0 - oy;
                float2 e00, e10, e01, e11;
                if (tiled && unsigned(li) < tw && unsigned(lj) < tw) {
                    const int q = lj * RW + li;
                    const float4 p0 = et[q], p1 = et[q + (c.j1 - c.j0) * RW];
                    e00 = make_float2(p0.x, p0.y);
                    e10 = make_float2(p0.z, p0.w);
                    e01 = make_float2(p1.x, p1.y);
                    e11 = make_float2(p1.z, p1.w);
                } else {
                    e00 = __ldg(M.E + long(c.j0) * M.ep + c.i0);
                    e10 = __ldg(M.E + long(c.j0) * M.ep + c.i1);
                    e01 = __ldg(M.E + long(c.j1) * M.ep + c.i0);
                    e11 = __ldg(M.E + long(c.j1) * M.ep + c.i1);
                }
                vx = __fmaf_rn(C.kq, cic_interp(c, e00.x, e10.x, e01.x, e11.x), vx);
                vy = __fmaf_rn(C.kq, cic_interp(c, e00.y, e10.y, e01.y, e11.y), vy);
            }
            if (candidate) {
                // kicked but not moved: listed here, appended to the global
                // list at the unit's end; k_collide finishes it after this pass
                ++my_cand;
                const int k = atomicAdd(&s_nc, 1);
                if (k < kCandUnit) {
                    s_cidx[k] = make_int2(s, b + l);
                    s_cst[k] = make_float4(x, y, vx, vy);
                    continue;
                }
                const int slot = atomicAdd(M.cand_count, 1);
                if (slot < M.cand_cap) {
                    M.cand[slot] = make_int2(s, b + l);
                    M.cand_state[slot] = make_float4(x, y, vx, vy);
                    continue;
                }
                atomicAdd(M.ctr + kCtrCandOverflow, 1ull);
            }
            if (do_drift) {
                const float x0 = x, y0 = y;
                if constexpr (RZ) {
                    float vz = gvz[l];
                    drift_rz(x, y, vx, vy, vz, C.dtdx, C.dtdy);
                    gvz[l] = vz;
                } else {
                    x = __fmaf_rn(vx, C.dtdx, x);
                    y = __fmaf_rn(vy, C.dtdy, y);
                }
                if (!(x >= 0.0f && x <= float(M.nx - 1) && y >= 0.0f && y <= float(M.ny - 1))) {
                    x = __int_as_float(0x7fc00000);
                    y = x;
                    ++my_abs;
                } else if (M.electrodes && hits_electrode(x0, y0, x, y, M.nx, M.ny, M.vbits, M.hbits)) {
                    x = __int_as_float(0x7fc00000);
                    y = x;
                    ++my_elec;
                }
            }
            px[l] = x;
            py[l] = y;
            pvx[l] = vx;
            pvy[l] = vy;
            if (do_deposit && is_live(x)) {
                // after the drift's domain test a live position lies in
                // [0, nx-1] x [0, ny-1], where cic_weights' clamp changes nothing
                const Cic c = FULL ? cic_weights_in_domain(x, y, M.nx, M.ny) : cic_weights(x, y, M.nx, M.ny);
                const int li = c.i0 - ox, lj = c.j0 - oy;
                if (tiled && unsigned(li) < tw && unsigned(lj) < tw) {
                    const int q = lj * RW + li;
                    const int dq = c.i1 - c.i0, dr = (c.j1 - c.j0) * RW;
                    atomicAdd(rt + q, __float2uint_rn(__fmul_rn(c.w00, kFixScale)));
                    atomicAdd(rt + q + dq, __float2uint_rn(__fmul_rn(c.w10, kFixScale)));
                    atomicAdd(rt + q + dr, __float2uint_rn(__fmul_rn(c.w01, kFixScale)));
                    atomicAdd(rt + q + dr + dq, __float2uint_rn(__fmul_rn(c.w11, kFixScale)));
                } else {
                    atomicAdd(M.rho + long(c.j0) * M.nx + c.i0, __fmul_rn(C.scale, c.w00));
                    atomicAdd(M.rho + long(c.j0) * M.nx + c.i1, __fmul_rn(C.scale, c.w10));
                    atomicAdd(M.rho + long(c.j1) * M.nx + c.i0, __fmul_rn(C.scale, c.w01));
                    atomicAdd(M.rho + long(c.j1) * M.nx + c.i1, __fmul_rn(C.scale, c.w11));
                }
            }
        }
        prev = ch;
        if (ch.e < ch.unit_e) {
            // the unit continues: every thread derives the next chunk itself
            ch.b = ch.e;
            ch.e = min(ch.unit_e, ch.e + kChunk);
            ch.first = 0;
        } else {
            // end of the unit: flush the charge tile and the counters
            my_abs = __reduce_add_sync(0xffffffffu, my_abs);
            my_cand = __reduce_add_sync(0xffffffffu, my_cand);
            my_elec = __reduce_add_sync(0xffffffffu, my_elec);
            if ((tid & 31) == 0) {
                if (my_abs) atomicAdd(&s_abs, my_abs);
                if (my_cand) atomicAdd(&s_cand, my_cand);
                if (my_elec) atomicAdd(&s_elec, my_elec);
            }
            my_abs = my_cand = my_elec = 0u;
            __syncthreads();
            // every particle of the unit is done with the E tile: the next
            // unit's tile is copied in while the charge tile is flushed
            const ChunkDesc nch = s_ch[nxt];
            int nox = ox, noy = oy;
            if (nch.valid && nch.tile >= 0)
                stage_etile_async(member<ENS>(A, chunk_member<ENS>(nch.s)), nch.tile, et, nox, noy);
            if (tiled && do_deposit) {
                for (int q = tid; q < RW * RW; q += kPushThreads) {
                    const unsigned sum = rt[q];
                    if (sum) {
                        rt[q] = 0u;
                        atomicAdd(M.rho + long(oy + q / RW) * M.nx + ox + q % RW,
                                  __fmul_rn(C.scale, __fmul_rn(float(sum), kFixInv)));
                    }
                }
            }
            if (tid == 0) {
                if (s_abs) atomicAdd(M.ctr + kCtrAbsorbed + s, (unsigned long long)s_abs);
                if (s_cand) atomicAdd(M.ctr + kCtrCandidates + s, (unsigned long long)s_cand);
                if (s_elec) atomicAdd(M.ctr + kCtrElectrode + s, (unsigned long long)s_elec);
                s_abs = 0;
                s_cand = 0;
                s_elec = 0;
                // the unit's listed candidates: one reservation in the global list
                const int nl = min(s_nc, kCandUnit);
                s_nflush = nl;
                s_cbase = nl ? atomicAdd(M.cand_count, nl) : 0;
                s_nc = 0;
            }
            cp_async_wait_all();
            __syncthreads();
            // (the list is refilled only after the next chunk's barrier)
            if (tid < s_nflush) {
                const int slot = s_cbase + tid;
                if (slot < M.cand_cap) {
                    M.cand[slot] = s_cidx[tid];
                    M.cand_state[slot] = s_cst[tid];
                } else {
                    // no room: the particle keeps its kick and is not moved this step
                    atomicAdd(M.ctr + kCtrCandOverflow, 1ull);
                }
            }
            ch = nch;
            if (ch.valid && ch.tile >= 0) {
                if constexpr (ENS) RW = member<ENS>(A, chunk_member<ENS>(ch.s)).rw;
                ox = nox;
                oy = noy;
            }
        }
        cur = nxt;
    }
    // write back the last chunk processed, then wait for every bulk store
    __syncthreads();
    if (prev.valid) {
        const int prv = cur == 0 ? kStages - 1 : cur - 1;
        if (tid == 0) {
            store_chunk_bulk<ENS>(A, prev, bufs + prv * 4 * kBufStride);
            bulk_commit();
        }
        store_chunk_edges<ENS>(A, prev, bufs + prv * 4 * kBufStride, tid);
    }
    if (tid == 0) bulk_wait_all();
}

// ---- particle pass, producer warp and consumer warps without block barriers ----------
//
// k_push_pipe: the work of k_push (same chunks, ring of three bulk-copied
// buffers, E tile and charge tile per unit, same per-particle arithmetic, in
// the same blocked order), with the per-chunk block barrier replaced by
// mbarriers, so that the consumer warps never wait for one another inside a
// unit:
//   warp 0 (producer)   claims chunks, publishes each chunk's descriptor,
//                       loads it (cp.async.bulk, completion on full[stage]),
//                       waits for done[stage] (one arrival per consumer warp),
//                       writes the chunk back (bulk stores, ragged edges by
//                       plain stores) and reloads the buffer two chunks ahead;
//                       past the last chunk it completes full[stage] with a
//                       plain arrival, the end marker
//   warps 1..7          wait full[stage], push their three particles each,
//                       arrive on done[stage]; at the end of a unit they meet
//                       on an mbarrier (cbar), flush the charge tile, stage
//                       the next unit's E tile and meet again
// Every wait is bounded: a thread whose wait gives up sets the error flag
// and leaves; the others' waits on it then give up in turn.  The producer
// waits, with the default limit, for every copy it started before it leaves.
__device__ __forceinline__ void mbar_arrive(unsigned long long* m) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(m)) : "memory");
}

// stage_tile's E staging by the consumer threads (ctid in [0, nc)); the
// charge tile is left as the last flush zeroed it.
__device__ __forceinline__ void stage_etile_c(const PushArgs& A, int tile, float4* et, int& ox, int& oy, int ctid,
                                              int nc) {
    const int RW = A.rw;
    ox = (tile % A.tiles_x) * A.tile - kHalo;
    oy = (tile / A.tiles_x) * A.tile - kHalo;
    for (int q = ctid; q < RW * RW; q += nc) {
        const int gi = ox + q % RW, gj = oy + q / RW;
        float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
        if (gi >= 0 && gj >= 0 && gi < A.nx && gj < A.ny) {
            const long k = long(gj) * A.ep + gi;
            const float2 e0 = __ldg(A.E + k), e1 = __ldg(A.E + k + (gi + 1 < A.nx ? 1 : 0));
            v = make_float4(e0.x, e0.y, e1.x, e1.y);
        }
        et[q] = v;
    }
}

constexpr int kConsumerWarps = kPushThreads / 32 - 1;
constexpr int kConsumers = kConsumerWarps * 32;

// Consumer warps: arrive on cbar and wait for the phase (bounded).
__device__ __forceinline__ bool consumer_meet(unsigned long long* cbar, unsigned& phase, unsigned long long limit) {
    __syncwarp();
    if ((threadIdx.x & 31) == 0) mbar_arrive(cbar);
    const bool ok = mbar_wait(cbar, phase, limit);
    phase ^= 1u;
    return ok;
}

template <bool RZ, bool FULL>
__global__ void __launch_bounds__(kPushThreads, 4) k_push_pipe(PushArgs A) {
    extern __shared__ __align__(128) unsigned char smem[];
    float* bufs = reinterpret_cast<float*>(smem);  // [kStages][4][kBufStride]
    const int RW = A.rw;
    float4* et = reinterpret_cast<float4*>(bufs + kStages * 4 * kBufStride);
    unsigned* rt = reinterpret_cast<unsigned*>(et + RW * RW);
    __shared__ __align__(8) unsigned long long full[kStages], done[kStages], cbar;
    __shared__ ChunkDesc s_ch[kStages];
    __shared__ unsigned s_abs, s_cand, s_elec;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int n_items = *A.n_items;
    for (int q = tid; q < RW * RW; q += kPushThreads) rt[q] = 0u;
    if (tid == 0) {
        for (int k = 0; k < kStages; ++k) {
            mbar_init(&full[k], 1);
            mbar_init(&done[k], kConsumerWarps);
        }
        mbar_init(&cbar, kConsumerWarps);
        fence_mbar_init();
        s_abs = s_cand = s_elec = 0u;
        // the first two chunks
        ChunkDesc none;
        none.valid = 0;
        for (int k = 0; k < 2; ++k) {
            const ChunkDesc c = (k == 0 || s_ch[0].valid) ? next_chunk<false>(A, k ? s_ch[0] : none, n_items) : none;
            s_ch[k] = c;
            if (c.valid) issue_chunk<false>(A, c, bufs + k * 4 * kBufStride, nullptr, &full[k]);
            else mbar_arrive(&full[k]);  // the end marker
        }
    }
    __syncthreads();
    if (warp == 0) {
        // ---- producer ----
        int j = 0;
        bool ok = true;
        for (;; ++j) {
            const int st = j % kStages;
            const ChunkDesc cj = s_ch[st];
            if (!cj.valid) break;
            // the consumers are done with chunk j: write it back
            ok = mbar_wait(&done[st], unsigned(j / kStages) & 1u, A.wait_limit);
            if (!ok) break;
            float* const buf = bufs + st * 4 * kBufStride;
            if (lane == 0) {
                store_chunk_bulk<false>(A, cj, buf);
                bulk_commit();
            }
            store_chunk_edges<false>(A, cj, buf, lane);
            // chunk j + 2 into the buffer of chunk j - 1, once its store has read it
            if (lane == 0) {
                const int s2 = (j + 2) % kStages;
                const ChunkDesc c1 = s_ch[(j + 1) % kStages];
                ChunkDesc c2;
                c2.valid = 0;
                if (c1.valid) c2 = next_chunk<false>(A, c1, n_items);
                bulk_wait_read1();
                s_ch[s2] = c2;
                if (c2.valid) {
                    fence_proxy_async();
                    issue_chunk<false>(A, c2, bufs + s2 * 4 * kBufStride, nullptr, &full[s2]);
                } else {
                    mbar_arrive(&full[s2]);  // the end marker
                }
            }
            __syncwarp();
        }
        if (lane == 0) {
            if (!ok) {
                atomicExch(A.error, 1);
                // the loads started for chunks j and j + 1 (chunk j + 2's was not)
                for (int k = 0; k <= 1; ++k) {
                    const int c = j + k, st = c % kStages;
                    if (s_ch[st].valid) mbar_wait(&full[st], unsigned(c / kStages) & 1u, kWaitLimit);
                }
            }
            bulk_wait_all();
        }
        return;
    }
    // ---- consumers ----
    const int ctid = tid - 32;
    const bool do_kick = FULL || A.do_kick, do_drift = FULL || A.do_drift, do_deposit = FULL || A.do_deposit;
    unsigned cphase = 0u;
    int ox = 0, oy = 0;
    if (!mbar_wait(&full[0], 0u, A.wait_limit)) {
        atomicExch(A.error, 1);
        return;
    }
    ChunkDesc ch = s_ch[0];
    if (!ch.valid) return;
    if (ch.tile >= 0) stage_etile_c(A, ch.tile, et, ox, oy, ctid, kConsumers);
    if (!consumer_meet(&cbar, cphase, A.wait_limit)) {
        atomicExch(A.error, 1);
        return;
    }
    unsigned my_abs = 0, my_cand = 0, my_elec = 0;
    const unsigned tw = unsigned(RW - 1);  // staged tile: local cell index in [0, RW-2]
    for (int j = 0;; ++j) {
        const int cur = j % kStages;
        const bool tiled = ch.tile >= 0;
        const int s = ch.s, b = ch.b, n = ch.e - ch.b;
        const int off = b & 3;
        float* const px = bufs + cur * 4 * kBufStride + off;
        float* const py = px + kBufStride;
        float* const pvx = py + kBufStride;
        float* const pvy = pvx + kBufStride;
        const SpeciesConst C = A.sp[s];
        const unsigned* const cbits = A.do_mcc ? A.cbits[s] : nullptr;
        float* const gvz = RZ ? A.state[s].cur[4] + b : nullptr;
        const int s0 = b + ctid * kPushP, s_last = min(s0 + kPushP, b + n) - 1;
        unsigned cmask = 0u;
        if (cbits && s0 <= s_last) {
            const unsigned cw0 = __ldg(cbits + (s0 >> 5));
            const unsigned cw1 = (s_last >> 5) != (s0 >> 5) ? __ldg(cbits + (s_last >> 5)) : 0u;
            cmask = __funnelshift_r(cw0, cw1, s0 & 31);
        }
#pragma unroll
        for (int k = 0; k < kPushP; ++k) {
            const int l = ctid * kPushP + k;
            if (l >= n) break;
            const bool candidate = (cmask >> k) & 1u;
            float x = px[l], y = py[l];
            if (!is_live(x)) continue;
            float vx = pvx[l], vy = pvy[l];
            if (do_kick) {
                const Cic c = cic_weights(x, y, A.nx, A.ny);
                const int li = c.i0 - ox, lj = c.j0 - oy;
                float2 e00, e10, e01, e11;
                if (tiled && unsigned(li) < tw && unsigned(lj) < tw) {
                    const int q = lj * RW + li;
                    const float4 p0 = et[q], p1 = et[q + (c.j1 - c.j0) * RW];
                    e00 = make_float2(p0.x, p0.y);
                    e10 = make_float2(p0.z, p0.w);
                    e01 = make_float2(p1.x, p1.y);
                    e11 = make_float2(p1.z, p1.w);
                } else {
                    e00 = __ldg(A.E + long(c.j0) * A.ep + c.i0);
                    e10 = __ldg(A.E + long(c.j0) * A.ep + c.i1);
                    e01 = __ldg(A.E + long(c.j1) * A.ep + c.i0);
                    e11 = __ldg(A.E + long(c.j1) * A.ep + c.i1);
                }
                vx = __fmaf_rn(C.kq, cic_interp(c, e00.x, e10.x, e01.x, e11.x), vx);
                vy = __fmaf_rn(C.kq, cic_interp(c, e00.y, e10.y, e01.y, e11.y), vy);
            }
            if (candidate) {
                // kicked but not moved: k_collide finishes it after this pass
                ++my_cand;
                const int slot = atomicAdd(A.cand_count, 1);
                if (slot < A.cand_cap) {
                    A.cand[slot] = make_int2(s, b + l);
                    A.cand_state[slot] = make_float4(x, y, vx, vy);
                    continue;
                }
                atomicAdd(A.ctr + kCtrCandOverflow, 1ull);
            }
            if (do_drift) {
                const float x0 = x, y0 = y;
                if constexpr (RZ) {
                    float vz = gvz[l];
                    drift_rz(x, y, vx, vy, vz, C.dtdx, C.dtdy);
                    gvz[l] = vz;
                } else {
                    x = __fmaf_rn(vx, C.dtdx, x);
                    y = __fmaf_rn(vy, C.dtdy, y);
                }
                if (!(x >= 0.0f && x <= float(A.nx - 1) && y >= 0.0f && y <= float(A.ny - 1))) {
                    x = __int_as_float(0x7fc00000);
                    y = x;
                    ++my_abs;
                } else if (A.electrodes && hits_electrode(x0, y0, x, y, A.nx, A.ny, A.vbits, A.hbits)) {
                    x = __int_as_float(0x7fc00000);
                    y = x;
                    ++my_elec;
                }
            }
            px[l] = x;
            py[l] = y;
            pvx[l] = vx;
            pvy[l] = vy;
            if (do_deposit && is_live(x)) {
                const Cic c = FULL ? cic_weights_in_domain(x, y, A.nx, A.ny) : cic_weights(x, y, A.nx, A.ny);
                const int li = c.i0 - ox, lj = c.j0 - oy;
                if (tiled && unsigned(li) < tw && unsigned(lj) < tw) {
                    const int q = lj * RW + li;
                    const int dq = c.i1 - c.i0, dr = (c.j1 - c.j0) * RW;
                    atomicAdd(rt + q, __float2uint_rn(__fmul_rn(c.w00, kFixScale)));
                    atomicAdd(rt + q + dq, __float2uint_rn(__fmul_rn(c.w10, kFixScale)));
                    atomicAdd(rt + q + dr, __float2uint_rn(__fmul_rn(c.w01, kFixScale)));
                    atomicAdd(rt + q + dr + dq, __float2uint_rn(__fmul_rn(c.w11, kFixScale)));
                } else {
                    atomicAdd(A.rho + long(c.j0) * A.nx + c.i0, __fmul_rn(C.scale, c.w00));
                    atomicAdd(A.rho + long(c.j0) * A.nx + c.i1, __fmul_rn(C.scale, c.w10));
                    atomicAdd(A.rho + long(c.j1) * A.nx + c.i0, __fmul_rn(C.scale, c.w01));
                    atomicAdd(A.rho + long(c.j1) * A.nx + c.i1, __fmul_rn(C.scale, c.w11));
                }
            }
        }
        // this warp is done with chunk j (its results are in the buffer)
        __syncwarp();
        if (lane == 0) mbar_arrive(&done[cur]);
        const bool unit_end = ch.e == ch.unit_e;
        const int nst = (j + 1) % kStages;
        if (!mbar_wait(&full[nst], unsigned((j + 1) / kStages) & 1u, A.wait_limit)) {
            atomicExch(A.error, 1);
            return;
        }
        const ChunkDesc nc = s_ch[nst];
        if (unit_end) {
            // the unit's deposits and counters are complete once every consumer has met
            my_abs = __reduce_add_sync(0xffffffffu, my_abs);
            my_cand = __reduce_add_sync(0xffffffffu, my_cand);
            my_elec = __reduce_add_sync(0xffffffffu, my_elec);
            if (lane == 0) {
                if (my_abs) atomicAdd(&s_abs, my_abs);
                if (my_cand) atomicAdd(&s_cand, my_cand);
                if (my_elec) atomicAdd(&s_elec, my_elec);
            }
            my_abs = my_cand = my_elec = 0u;
            if (!consumer_meet(&cbar, cphase, A.wait_limit)) {
                atomicExch(A.error, 1);
                return;
            }
            if (tiled && do_deposit) {
                // flush, and leave the tile zeroed for the next unit
                for (int q = ctid; q < RW * RW; q += kConsumers) {
                    const unsigned sum = rt[q];
                    if (sum) {
                        atomicAdd(A.rho + long(oy + q / RW) * A.nx + ox + q % RW,
                                  __fmul_rn(C.scale, __fmul_rn(float(sum), kFixInv)));
                        rt[q] = 0u;
                    }
                }
            }
            if (ctid == 0) {
                if (s_abs) atomicAdd(A.ctr + kCtrAbsorbed + s, (unsigned long long)s_abs);
                if (s_cand) atomicAdd(A.ctr + kCtrCandidates + s, (unsigned long long)s_cand);
                if (s_elec) atomicAdd(A.ctr + kCtrElectrode + s, (unsigned long long)s_elec);
                s_abs = s_cand = s_elec = 0u;
            }
            // every E-tile read of this unit is done: stage the next unit's
            if (nc.valid && nc.tile >= 0) stage_etile_c(A, nc.tile, et, ox, oy, ctid, kConsumers);
            if (!consumer_meet(&cbar, cphase, A.wait_limit)) {
                atomicExch(A.error, 1);
                return;
            }
        }
        if (!nc.valid) return;
        ch = nc;
    }
}

// ---- particle pass, per-warp pipeline --------------------------------------------
//
// The same work as k_push (same work units, E tile and charge tile per unit,
// same per-particle arithmetic), streamed differently: every warp runs its
// own pipeline of bulk copies instead of the CTA sharing one ring.  A unit's
// slots are cut into groups of kWarpGroup particles, dealt round-robin to the
// eight warps; lane 0 of each warp keeps up to kWarpStages - 1 of its groups
// in flight (cp.async.bulk of x, y, vx, vy into the warp's own stage buffers,
// completed on the warp's own mbarriers), running ahead into the next unit,
// whose descriptor is claimed one unit early.  Lane l of a group handles the
// particles l, l + 32, l + 64, ...: coalesced, conflict-free reads of the stage
// and coalesced stores of the results straight to global memory.  The only
// block barriers are the three per unit (E tile staged; deposits done; charge
// tile flushed), so a warp waits only on its own copies.
//
// The charge tile is deposited with warp-aggregated atomics when DEPOSIT_AGG:
// lanes whose particles fall in the same cell (sorted particles put runs of
// consecutive lanes in one cell) sum their four fixed-point weights with
// redux.sync over __match_any_sync's group, and the group's lowest lane adds
// the sums.  Integer sums are exact, so the tile holds the same values either way.
constexpr int kWarpGroup = 128;  // particles per group (four per lane)
constexpr int kWarpStages = 3;   // stage buffers per warp
constexpr int kPushWarps = kPushThreads / 32;

struct UnitDesc {
    const float* cur[4];  // x, y, vx, vy of the unit's species
    int valid;
    int s, tile, b, e;
};

__device__ __forceinline__ UnitDesc claim_unit(const PushArgs& A, int n_items) {
    UnitDesc u;
    const int it = atomicAdd(A.item_next, 1);
    u.valid = it < n_items;
    u.s = u.tile = u.b = u.e = 0;
    if (u.valid) {
        const int4 v = A.items[it];
        u.s = v.x;
        u.tile = v.y;
        u.b = v.z;
        u.e = v.w;
#pragma unroll
        for (int k = 0; k < 4; ++k) u.cur[k] = A.state[u.s].cur[k];
    }
    return u;
}

// Per-warp producer state (the same in every lane): the next group to load
// is the pj-th of this warp in unit pu; `issued` groups were loaded so far.
struct WarpFeed {
    int pu, pj, issued;
};

// Every lane: loads this warp's next groups (each lane 16 bytes of each of
// x, y, vx, vy: one asynchronous copy group per particle group) while stage
// buffers are free and the units are known (the current one and the next).
__device__ __forceinline__ void warp_feed(const UnitDesc* units, int kcur, int consumed, WarpFeed& f, int warp,
                                          int lane, float* wbuf) {
    while (f.issued - consumed < kWarpStages && f.pu <= kcur + 1) {
        const UnitDesc& U = units[f.pu & 1];
        if (!U.valid) return;
        const int w0 = (U.b & ~3) + (f.pj * kPushWarps + warp) * kWarpGroup;
        if (w0 >= U.e) {
            ++f.pu;
            f.pj = 0;
            continue;
        }
        const int w1 = min(w0 + kWarpGroup, (U.e + 3) & ~3);
        float* buf = wbuf + (f.issued % kWarpStages) * 4 * kWarpGroup;
        const int o = 4 * lane;
        if (w0 + o < w1) {
#pragma unroll
            for (int k = 0; k < 4; ++k) cp_async16(buf + k * kWarpGroup + o, U.cur[k] + w0 + o);
        }
        cp_async_commit();
        ++f.issued;
        ++f.pj;
    }
}

// The E tile of a unit: one bulk tensor load of the ew x RW nodes from
// (ox, oy) (zero outside the grid) into `dst`, completed on `bar` (one thread).
__device__ __forceinline__ void issue_etile(const PushArgs& A, int tile, float2* dst, unsigned long long* bar) {
    const int ox = (tile % A.tiles_x) * A.tile - kHalo, oy = (tile / A.tiles_x) * A.tile - kHalo;
    fence_proxy_async();  // the block's reads of this buffer (the unit before last) before the copy overwrites it
    mbar_expect_tx(bar, unsigned(A.ew * A.rw) * unsigned(sizeof(float2)));
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
        "[%4];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<unsigned long long>(&A.emap)), "r"(ox), "r"(oy), "r"(smem_u32(bar))
        : "memory");
}

template <bool RZ, bool FULL, bool DEPOSIT_AGG>
__global__ void __launch_bounds__(kPushThreads, 3) k_push_warp(const __grid_constant__ PushArgs A) {
    extern __shared__ __align__(128) unsigned char smem[];
    float* wbufs = reinterpret_cast<float*>(smem);  // [warp][stage][4][kWarpGroup]
    const int RW = A.rw, EW = A.ew;
    // two E tiles (the unit in work and the next one), 128-byte aligned
    const int ebuf = ((EW * RW * int(sizeof(float2)) + 127) / 128) * 128;
    unsigned char* ebase = smem + sizeof(float) * kPushWarps * kWarpStages * 4 * kWarpGroup;
    unsigned* rt = reinterpret_cast<unsigned*>(ebase + 2 * ebuf);
    __shared__ __align__(8) unsigned long long ebars[2];
    __shared__ UnitDesc units[2];
    __shared__ unsigned s_abs, s_cand, s_elec;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int n_items = *A.n_items;
    float* const wbuf = wbufs + warp * kWarpStages * 4 * kWarpGroup;
    unsigned epend = 0u;  // thread 0: E-tile buffers with a load issued and not yet waited for
    if (tid == 0) {
        mbar_init(&ebars[0], 1);
        mbar_init(&ebars[1], 1);
        fence_mbar_init();
        for (int b = 0; b < 2; ++b) {
            units[b] = claim_unit(A, n_items);
            if (units[b].valid && units[b].tile >= 0) {
                issue_etile(A, units[b].tile, reinterpret_cast<float2*>(ebase + b * ebuf), &ebars[b]);
                epend |= 1u << b;
            }
        }
        s_abs = s_cand = s_elec = 0u;
    }
    for (int q = tid; q < RW * RW; q += kPushThreads) rt[q] = 0u;  // the flush zeroes it after every unit
    __syncthreads();
    const bool do_kick = FULL || A.do_kick, do_drift = FULL || A.do_drift, do_deposit = FULL || A.do_deposit;
    WarpFeed feed{0, 0, 0};
    int consumed = 0;
    unsigned ephase = 0u;  // parity of each E buffer's next load
    bool failed = false;
    const unsigned tw = unsigned(RW - 1);  // staged tile: local cell index in [0, RW-2]
    for (int kcur = 0;; ++kcur) {
        const UnitDesc U = units[kcur & 1];
        if (!U.valid) break;
        const bool tiled = U.tile >= 0;
        const int eb = kcur & 1;
        const float2* const et = reinterpret_cast<const float2*>(ebase + eb * ebuf);
        int ox = 0, oy = 0;
        if (tiled) {
            ox = (U.tile % A.tiles_x) * A.tile - kHalo;
            oy = (U.tile / A.tiles_x) * A.tile - kHalo;
            if (mbar_wait(&ebars[eb], (ephase >> eb) & 1u, A.wait_limit)) {
                ephase ^= 1u << eb;
                if (tid == 0) epend &= ~(1u << eb);
            } else {
                failed = true;  // the load stays pending (thread 0 waits for it before exiting)
            }
        }
        warp_feed(units, kcur, consumed, feed, warp, lane, wbuf);
        const int s = U.s;
        const SpeciesConst C = A.sp[s];
        const SpeciesState& SS = A.state[s];
        float* const gx = SS.cur[0];
        float* const gy = SS.cur[1];
        float* const gvx = SS.cur[2];
        float* const gvy = SS.cur[3];
        float* const gvz = SS.cur[4];
        const unsigned* const cbits = A.do_mcc ? A.cbits[s] : nullptr;
        unsigned my_abs = 0, my_cand = 0, my_elec = 0;
        const int a0 = U.b & ~3;
        for (int j = 0; !failed; ++j) {
            const int w0 = a0 + (j * kPushWarps + warp) * kWarpGroup;
            if (w0 >= U.e) break;
            const int st = consumed % kWarpStages;
            cp_async_wait_pending(feed.issued - consumed - 1);
            __syncwarp();  // the other lanes' copies of this group are visible
            const float* const buf = wbuf + st * 4 * kWarpGroup;
#pragma unroll
            for (int m = 0; m < kWarpGroup / 32; ++m) {
                const int l = lane + 32 * m;
                const int p = w0 + l;
                const bool mine = p >= U.b && p < U.e;
                float x = buf[l], y = buf[kWarpGroup + l];
                const bool live = mine && is_live(x);
                float vx = buf[2 * kWarpGroup + l], vy = buf[3 * kWarpGroup + l];
                bool dep = false;
                if (live) {
                    if (do_kick) {
                        const Cic c = cic_weights(x, y, A.nx, A.ny);
                        const int li = c.i0 - ox, lj = c.j0 - oy;
                        float2 e00, e10, e01, e11;
                        if (tiled && unsigned(li) < tw && unsigned(lj) < tw) {
                            const int q = lj * EW + li, dq = c.i1 - c.i0, dr = (c.j1 - c.j0) * EW;
                            e00 = et[q];
                            e10 = et[q + dq];
                            e01 = et[q + dr];
                            e11 = et[q + dr + dq];
                        } else {
                            e00 = __ldg(A.E + long(c.j0) * A.ep + c.i0);
                            e10 = __ldg(A.E + long(c.j0) * A.ep + c.i1);
                            e01 = __ldg(A.E + long(c.j1) * A.ep + c.i0);
                            e11 = __ldg(A.E + long(c.j1) * A.ep + c.i1);
                        }
                        vx = __fmaf_rn(C.kq, cic_interp(c, e00.x, e10.x, e01.x, e11.x), vx);
                        vy = __fmaf_rn(C.kq, cic_interp(c, e00.y, e10.y, e01.y, e11.y), vy);
                    }
                    bool candidate = false;
                    if (cbits) candidate = (__ldg(cbits + (p >> 5)) >> (p & 31)) & 1u;
                    if (candidate) {
                        // kicked but not moved: k_collide finishes it after this pass
                        ++my_cand;
                        const int slot = atomicAdd(A.cand_count, 1);
                        if (slot < A.cand_cap) {
                            A.cand[slot] = make_int2(s, p);
                            A.cand_state[slot] = make_float4(x, y, vx, vy);
                        } else {
                            atomicAdd(A.ctr + kCtrCandOverflow, 1ull);
                            candidate = false;
                        }
                    }
                    if (candidate) {
                        gvx[p] = vx;
                        gvy[p] = vy;
                    } else {
                        if (do_drift) {
                            const float x0 = x, y0 = y;
                            if constexpr (RZ) {
                                float vz = gvz[p];
                                drift_rz(x, y, vx, vy, vz, C.dtdx, C.dtdy);
                                gvz[p] = vz;
                            } else {
                                x = __fmaf_rn(vx, C.dtdx, x);
                                y = __fmaf_rn(vy, C.dtdy, y);
                            }
                            if (!(x >= 0.0f && x <= float(A.nx - 1) && y >= 0.0f && y <= float(A.ny - 1))) {
                                x = __int_as_float(0x7fc00000);
                                y = x;
                                ++my_abs;
                            } else if (A.electrodes && hits_electrode(x0, y0, x, y, A.nx, A.ny, A.vbits, A.hbits)) {
                                x = __int_as_float(0x7fc00000);
                                y = x;
                                ++my_elec;
                            }
                        }
                        gx[p] = x;
                        gy[p] = y;
                        gvx[p] = vx;
                        gvy[p] = vy;
                        dep = do_deposit && is_live(x);
                    }
                }
                // deposit: the fixed-point tile for positions inside it, global atomics otherwise
                Cic c{};
                int q = -1;
                if (dep) {
                    c = FULL ? cic_weights_in_domain(x, y, A.nx, A.ny) : cic_weights(x, y, A.nx, A.ny);
                    const int li = c.i0 - ox, lj = c.j0 - oy;
                    if (tiled && unsigned(li) < tw && unsigned(lj) < tw) {
                        q = lj * RW + li;
                    } else {
                        atomicAdd(A.rho + long(c.j0) * A.nx + c.i0, __fmul_rn(C.scale, c.w00));
                        atomicAdd(A.rho + long(c.j0) * A.nx + c.i1, __fmul_rn(C.scale, c.w10));
                        atomicAdd(A.rho + long(c.j1) * A.nx + c.i0, __fmul_rn(C.scale, c.w01));
                        atomicAdd(A.rho + long(c.j1) * A.nx + c.i1, __fmul_rn(C.scale, c.w11));
                    }
                }
                const int dq = c.i1 - c.i0, dr = (c.j1 - c.j0) * RW;
                unsigned f00 = 0, f10 = 0, f01 = 0, f11 = 0;
                if (q >= 0) {
                    f00 = __float2uint_rn(__fmul_rn(c.w00, kFixScale));
                    f10 = __float2uint_rn(__fmul_rn(c.w10, kFixScale));
                    f01 = __float2uint_rn(__fmul_rn(c.w01, kFixScale));
                    f11 = __float2uint_rn(__fmul_rn(c.w11, kFixScale));
                }
                if constexpr (DEPOSIT_AGG) {
                    // lanes of one cell (and one neighbour layout) sum their weights; -1 - lane
                    // keys keep the lanes without a tile deposit apart
                    const int key = q >= 0 ? (q | (dq << 20) | ((dr != 0) << 21)) : -1 - lane;
                    const unsigned grp = __match_any_sync(0xffffffffu, key);
                    if (q >= 0) {
                        const unsigned s00 = __reduce_add_sync(grp, f00), s10 = __reduce_add_sync(grp, f10);
                        const unsigned s01 = __reduce_add_sync(grp, f01), s11 = __reduce_add_sync(grp, f11);
                        if (lane == __ffs(grp) - 1) {
                            atomicAdd(rt + q, s00);
                            atomicAdd(rt + q + dq, s10);
                            atomicAdd(rt + q + dr, s01);
                            atomicAdd(rt + q + dr + dq, s11);
                        }
                    }
                } else if (q >= 0) {
                    atomicAdd(rt + q, f00);
                    atomicAdd(rt + q + dq, f10);
                    atomicAdd(rt + q + dr, f01);
                    atomicAdd(rt + q + dr + dq, f11);
                }
            }
            __syncwarp();  // every lane is done with the stage before it is reloaded
            ++consumed;
            warp_feed(units, kcur, consumed, feed, warp, lane, wbuf);
        }
        my_abs = __reduce_add_sync(0xffffffffu, my_abs);
        my_cand = __reduce_add_sync(0xffffffffu, my_cand);
        my_elec = __reduce_add_sync(0xffffffffu, my_elec);
        if (lane == 0) {
            if (my_abs) atomicAdd(&s_abs, my_abs);
            if (my_cand) atomicAdd(&s_cand, my_cand);
            if (my_elec) atomicAdd(&s_elec, my_elec);
        }
        const bool abort = __syncthreads_or(failed);  // deposits and E-tile reads of the unit done
        if (tiled && do_deposit) {
            // flush, and leave the tile zeroed for the next unit
            for (int q = tid; q < RW * RW; q += kPushThreads) {
                const unsigned sum = rt[q];
                if (sum) {
                    atomicAdd(A.rho + long(oy + q / RW) * A.nx + ox + q % RW,
                              __fmul_rn(C.scale, __fmul_rn(float(sum), kFixInv)));
                    rt[q] = 0u;
                }
            }
        }
        if (tid == 0) {
            if (s_abs) atomicAdd(A.ctr + kCtrAbsorbed + s, (unsigned long long)s_abs);
            if (s_cand) atomicAdd(A.ctr + kCtrCandidates + s, (unsigned long long)s_cand);
            if (s_elec) atomicAdd(A.ctr + kCtrElectrode + s, (unsigned long long)s_elec);
            s_abs = s_cand = s_elec = 0u;
            if (abort) {
                atomicExch(A.error, 1);
            } else {
                // unit kcur + 2, and its E tile into the buffer this unit used
                const UnitDesc nu = claim_unit(A, n_items);
                units[kcur & 1] = nu;
                if (nu.valid && nu.tile >= 0) {
                    issue_etile(A, nu.tile, reinterpret_cast<float2*>(ebase + eb * ebuf), &ebars[eb]);
                    epend |= 1u << eb;
                }
            }
        }
        __syncthreads();  // charge tile flushed; the unit after next published
        if (abort) break;
    }
    // after a give-up, the copies still in flight (none otherwise): wait for them
    cp_async_wait_all();
    if (tid == 0)
        for (int b = 0; b < 2; ++b)
            if (epend & (1u << b)) mbar_wait(&ebars[b], (ephase >> b) & 1u, kWaitLimit);
}

// The collision candidates of the pass, one thread each, with their kicked
// state from the list; the tables' descriptor is a kernel parameter (no
// global load before the first table lookup).
__global__ void __launch_bounds__(128) k_collide(PushArgs A, const __grid_constant__ MccDev MC) {
    const int nc = min(*A.cand_count, A.cand_cap);
    const uint32_t step = *A.step;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nc; i += gridDim.x * blockDim.x) {
        const int2 c = A.cand[i];
        const float4 v = A.cand_state[i];
        finish_candidate(A, MC, step, c.x, c.y, v.x, v.y, v.z, v.w);
    }
}

// Per step: untiled items for slots past the last sort, item counter reset,
// RNG step advance, collision candidate list reset.
__global__ void k_build_items(SpeciesState* state, int nspecies, const int* n_tiled, int4* items, int* n_items,
                              int* item_next, uint32_t* step, int* cand_count, int advance_step) {
    __shared__ int off[PIC_MAX_SPECIES + 1];
    if (threadIdx.x == 0) {
        int o = *n_tiled;
        for (int s = 0; s < nspecies; ++s) {
            off[s] = o;
            const int u = state[s].count - state[s].sorted_end;
            o += u > 0 ? (u + kUnitMax - 1) / kUnitMax : 0;
        }
        off[nspecies] = o;
        *n_items = o;
        *item_next = 0;
        *cand_count = 0;
        if (advance_step) *step += 1u;
    }
    __syncthreads();
    for (int s = 0; s < nspecies; ++s) {
        const int b0 = state[s].sorted_end, e0 = state[s].count;
        for (int c = threadIdx.x; c < off[s + 1] - off[s]; c += blockDim.x) {
            const int b = b0 + c * kUnitMax;
            items[off[s] + c] = make_int4(s, -1, b, min(e0, b + kUnitMax));
        }
    }
}

// After a sort: items for every (species, tile), split into chunks.
__global__ void k_tile_items(const int* __restrict__ tile_start, int ntiles, int nspecies, int4* items,
                             int* n_tiled) {
    __shared__ int part[1024];
    const int total = ntiles * nspecies;
    const int per = (total + blockDim.x - 1) / blockDim.x;
    const int b = threadIdx.x * per, e = min(total, b + per);
    int sum = 0;
    for (int q = b; q < e; ++q) {
        const int s = q / ntiles, t = q % ntiles;
        const int* ts = tile_start + s * (ntiles + 1);
        sum += (ts[t + 1] - ts[t] + kUnitMax - 1) / kUnitMax;
    }
    part[threadIdx.x] = sum;
    __syncthreads();
    for (int o = 1; o < blockDim.x; o <<= 1) {
        const int v = threadIdx.x >= o ? part[threadIdx.x - o] : 0;
        __syncthreads();
        part[threadIdx.x] += v;
        __syncthreads();
    }
    int w = part[threadIdx.x] - sum;
    for (int q = b; q < e; ++q) {
        const int s = q / ntiles, t = q % ntiles;
        const int* ts = tile_start + s * (ntiles + 1);
        for (int c = ts[t]; c < ts[t + 1]; c += kUnitMax) items[w++] = make_int4(s, t, c, min(ts[t + 1], c + kUnitMax));
    }
    if (threadIdx.x == blockDim.x - 1) *n_tiled = part[threadIdx.x];
}

__global__ void k_sim_keys(const SpeciesState* __restrict__ state, int s, int ncx, int ncy, int tile, int tiles_x,
                           uint32_t dead_key, uint32_t* __restrict__ keys, uint32_t* __restrict__ vals,
                           int* __restrict__ n_dev) {
    const int n = state[s].count;
    const float* __restrict__ x = state[s].cur[0];
    const float* __restrict__ y = state[s].cur[1];
    int mine = 0;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        const uint32_t k = tile_key(x[p], y[p], ncx, ncy, tile, tiles_x, dead_key);
        keys[p] = k;
        vals[p] = uint32_t(p);
        mine += k != dead_key;
    }
    mine = __reduce_add_sync(0xffffffffu, mine);
    if ((threadIdx.x & 31) == 0 && mine) atomicAdd(n_dev + 1, mine);
}

__global__ void k_sim_gather(const SpeciesState* __restrict__ state, int s, const uint32_t* __restrict__ perm,
                             const int* __restrict__ n_dev) {
    const int n = n_dev[1];
    // the arrays' pointers in registers (a store through alt could otherwise
    // alias the state struct and force them to be reloaded per element)
    const SpeciesState& S = state[s];
    const float *__restrict__ c0 = S.cur[0], *__restrict__ c1 = S.cur[1], *__restrict__ c2 = S.cur[2],
                *__restrict__ c3 = S.cur[3], *__restrict__ c4 = S.cur[4];
    float *__restrict__ a0 = S.alt[0], *__restrict__ a1 = S.alt[1], *__restrict__ a2 = S.alt[2],
          *__restrict__ a3 = S.alt[3], *__restrict__ a4 = S.alt[4];
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const uint32_t p = __ldg(perm + k);
        const float v0 = c0[p], v1 = c1[p], v2 = c2[p], v3 = c3[p], v4 = c4[p];
        a0[k] = v0;
        a1[k] = v1;
        a2[k] = v2;
        a3[k] = v3;
        a4[k] = v4;
    }
}

__global__ void k_sim_flip(SpeciesState* state, int s, const int* n_dev) {
    SpeciesState& S = state[s];
#pragma unroll
    for (int c = 0; c < 5; ++c) {
        float* t = S.cur[c];
        S.cur[c] = S.alt[c];
        S.alt[c] = t;
    }
    S.count = n_dev[1];
    S.sorted_end = n_dev[1];
}

__global__ void k_set_count(SpeciesState* state, int s, int n) {
    state[s].count = n;
    state[s].sorted_end = 0;
}

// Loading particles invalidates the tile items of every species.
__global__ void k_untile_all(SpeciesState* state, int nspecies, int* n_tiled) {
    for (int s = 0; s < nspecies; ++s) state[s].sorted_end = 0;
    *n_tiled = 0;
}

// ---- host object -----------------------------------------------------------------

// ---- headless particle buffer ---------------------------------------------------------
//
// The particle vertex buffer of the reference's renderer (src/Render.py:544-571,
// an OpenGL VBO filled through CUDA interop) as a plain device buffer: for every
// live particle, in species order and slot order, (x, y) normalised to [-1, 1]
// over [x_min, x_max] x [y_min, y_max] and the species' type (index + 1), as
// float32 triples.  Dead slots are dropped by a stable compaction: per 1024-slot
// block a live count, one exclusive scan over all blocks, then each block writes
// its live particles at its offset plus their rank among the block's live slots.

constexpr int kRenderBlock = 1024;

struct RenderArgs {
    const SpeciesState* state;
    int ns;
    int first_block[PIC_MAX_SPECIES + 1];  // blocks of species s: [first_block[s], first_block[s+1])
    int* counts;                           // [blocks + 1]: live slots per block, then exclusive offsets
    float* out;                            // [capacity][3]
    int capacity;
    double dx, dy, x0, y0, wx, wy;         // x_ndc = 2 (x dx - x0) / wx - 1 (the reference's order)
};

__device__ __forceinline__ int render_species(const RenderArgs& R, int blk) {
    int s = 0;
    while (s + 1 < R.ns && blk >= R.first_block[s + 1]) ++s;
    return s;
}

__global__ void __launch_bounds__(kRenderBlock) k_render_count(RenderArgs R) {
    const int s = render_species(R, blockIdx.x);
    const SpeciesState& S = R.state[s];
    const int slot = (blockIdx.x - R.first_block[s]) * kRenderBlock + threadIdx.x;
    const bool live = slot < S.count && is_live(S.cur[0][slot]);
    const int n = __syncthreads_count(live);
    if (threadIdx.x == 0) R.counts[blockIdx.x] = n;
}

// One block: exclusive offsets of the block counts in place, the total in counts[nb].
__global__ void __launch_bounds__(1024) k_render_scan(int* counts, int nb) {
    __shared__ int warp_tot[32];
    __shared__ int carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int base = 0; base < nb; base += blockDim.x) {
        const int i = base + threadIdx.x;
        const int v = i < nb ? counts[i] : 0;
        int x = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) warp_tot[w] = x;
        __syncthreads();
        if (w == 0) {
            int t = warp_tot[lane];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, t, o);
                if (lane >= o) t += y;
            }
            warp_tot[lane] = t;  // inclusive over warps
        }
        __syncthreads();
        const int before = carry + (w ? warp_tot[w - 1] : 0) + x - v;
        if (i < nb) counts[i] = before;
        __syncthreads();
        if (threadIdx.x == 0) carry += warp_tot[31];
        __syncthreads();
    }
    if (threadIdx.x == 0) counts[nb] = carry;
}

__global__ void __launch_bounds__(kRenderBlock) k_render_emit(RenderArgs R) {
    __shared__ int warp_n[kRenderBlock / 32];
    const int s = render_species(R, blockIdx.x);
    const SpeciesState& S = R.state[s];
    const int slot = (blockIdx.x - R.first_block[s]) * kRenderBlock + threadIdx.x;
    const float x = slot < S.count ? S.cur[0][slot] : __int_as_float(0x7fc00000);
    const bool live = is_live(x);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const unsigned bal = __ballot_sync(0xffffffffu, live);
    if (lane == 0) warp_n[w] = __popc(bal);
    __syncthreads();
    int off = R.counts[blockIdx.x];
    for (int q = 0; q < w; ++q) off += warp_n[q];
    off += __popc(bal & ((1u << lane) - 1u));
    if (live && off < R.capacity) {
        const float y = S.cur[1][slot];
        float* o = R.out + 3L * off;
        o[0] = float(2.0 * (double(x) * R.dx - R.x0) / R.wx - 1.0);
        o[1] = float(2.0 * (double(y) * R.dy - R.y0) / R.wy - 1.0);
        o[2] = float(s + 1);
    }
}

struct SimImpl {
    pic_sim_desc d{};
    int nx = 0, ny = 0, ns = 0;
    long G = 0;
    SortImpl sorter;
    bool have_sorter = false;
    pic_mg* mg = nullptr;
    MccHost mcc;
    bool have_mcc = false;
    MccDev* mcc_dev = nullptr;  // device copy of mcc.dev
    unsigned* cbits[PIC_MAX_SPECIES]{};  // candidate bit per slot of each colliding species
    unsigned *vbits = nullptr, *hbits = nullptr;  // internal electrode edges
    double* diag = nullptr;                        // diagnostics scratch
    int* render_counts = nullptr;                  // particle-buffer block counts (render_blocks + 1)
    int render_blocks = 0;
    bool electrodes = false;
    bool rz = false;                               // r-z geometry (desc.mg.geometry)
    double* rowf = nullptr;  // r-z: per row dx*dy / V_j, deposit -> charge density (null: Cartesian)
    double* rowv = nullptr;  // r-z: per row V_j / (dx*dy)
    unsigned** d_cbits = nullptr;         // device copy of cbits
    int* d_nseg = nullptr;                // 256-slot segments per species (0: no collisions)
    int cbits_segments = 0;               // sum of d_nseg
    int2* cand = nullptr;       // collision candidates of one pass
    float4* cand_state = nullptr;  // their kicked state
    int* cand_count = nullptr;
    int cand_cap = 0;
    std::vector<void*> allocs;
    SpeciesState* d_state = nullptr;
    SpeciesState h_state[PIC_MAX_SPECIES]{};
    SpeciesConst sc[PIC_MAX_SPECIES]{};
    int4* items = nullptr;
    int item_cap = 0;
    int *n_items = nullptr, *item_next = nullptr, *n_tiled = nullptr;
    uint32_t* step_ctr = nullptr;
    int* tile_start = nullptr;
    unsigned long long* ctr = nullptr;
    int* error = nullptr;
    unsigned long long wait_limit = kWaitLimit;  // polls of k_push's chunk waits
    float2* E2 = nullptr;
    int ep = 0;          // row pitch of E2 (nodes)
    int ew = 0;          // row width of an E tile in k_push_warp's shared memory (rw rounded up to even)
    CUtensorMap emap{};  // tiles of E2 for k_push_warp's bulk tensor loads
    float *Ex = nullptr, *Ey = nullptr, *rho_acc = nullptr, *rho_out = nullptr;
    double *phi = nullptr, *f = nullptr, *phi_prev = nullptr;
    bool have_prev = false;  // phi_prev holds the potential of the previous solve
    uint8_t* dirichlet = nullptr;
    int push_grid = 0;
    size_t push_smem = 0;
    int push_kernel = PIC_PUSH_RING;  // pic_push_kernel
    int push_grid_w = 0;              // launch shape of k_push_warp
    size_t push_smem_w = 0;
    int rw = 0;
    bool kick_pending = false;
    long long steps = 0;
    long long launches = 0;  // launches outside the multigrid loop
    long long solves = 0;    // multigrid solves issued (each runs 1 + cycles * body kernels)
    bool profiling = false;
    cudaStream_t cap = nullptr, cap2 = nullptr;  // capture stream and the side branch of a captured step
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    // g_sort_step: the step whose side branch sorts for the next step
    cudaGraphExec_t g_step = nullptr, g_sort_step = nullptr;
    cudaGraphExec_t g_sort = nullptr;  // the cell sort alone (init, pic_sim_sort)
    long long sort_graph_launches = 0;
    // the next particle pass is prepared (its sort, items and candidate bits
    // done, the step counter advanced): set by a captured step, cleared by
    // anything that changes the particle state on the host's behalf
    bool prepared = false;
    std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> marks;
    std::vector<cudaEvent_t> event_pool;
    long long prof_cycles = 0;
    pic_mg_info last{};
    int last_status = PIC_OK;
};

// The tensor map of E2 for k_push_warp's E tiles: 8-byte elements (an
// (Ex, Ey) pair), nx x ny with rows ep elements apart, boxes of ew x RW
// elements (ew = RW rounded up to even, so that a box row is a multiple of 16
// bytes), zero fill outside the grid.  cuTensorMapEncodeTiled comes through the runtime's
// entry-point lookup, so the library does not link the driver library.
static int encode_e_map(SimImpl& S) {
    using Encode = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
    static Encode encode = nullptr;
    if (!encode) {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q{};
        PIC_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q));
        if (q != cudaDriverEntryPointSuccess || !fn) return fail(PIC_ERR_CUDA, "cuTensorMapEncodeTiled not found");
        encode = reinterpret_cast<Encode>(fn);
    }
    if (S.ew > 256 || S.rw > 256)
        return fail(PIC_ERR_BAD_ARG, "pic_sim_create: tile %d gives an E tile of %d nodes", S.d.tile, S.rw);
    const cuuint64_t dims[2] = {cuuint64_t(S.nx), cuuint64_t(S.ny)};
    const cuuint64_t strides[1] = {cuuint64_t(S.ep) * sizeof(float2)};
    const cuuint32_t box[2] = {cuuint32_t(S.ew), cuuint32_t(S.rw)};
    const cuuint32_t estr[2] = {1, 1};
    const CUresult r = encode(&S.emap, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, S.E2, dims, strides, box, estr,
                              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                              CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(PIC_ERR_CUDA, "cuTensorMapEncodeTiled: error %d", int(r));
    return PIC_OK;
}

template <class T>
static int dalloc(SimImpl& S, T** p, size_t n) {
    PIC_CUDA(cudaMalloc(p, sizeof(T) * std::max<size_t>(n, 1)));
    S.allocs.push_back(*p);
    PIC_CUDA(cudaMemset(*p, 0, sizeof(T) * std::max<size_t>(n, 1)));
    return PIC_OK;
}

// Phase timing: begin() records a start event, end() the matching stop event.
static cudaEvent_t take_event(SimImpl& S) {
    if (!S.event_pool.empty()) {
        cudaEvent_t e = S.event_pool.back();
        S.event_pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}

struct PhaseTimer {
    SimImpl& S;
    int phase;
    cudaStream_t st;
    cudaEvent_t a = nullptr;
    PhaseTimer(SimImpl& s, int p, cudaStream_t stream) : S(s), phase(p), st(stream) {
        if (S.profiling) {
            a = take_event(S);
            cudaEventRecord(a, st);
        }
    }
    ~PhaseTimer() {
        if (a) {
            cudaEvent_t b = take_event(S);
            cudaEventRecord(b, st);
            S.marks.push_back({phase, {a, b}});
        }
    }
};

static PushArgs push_args(SimImpl& S, int kick, int mcc, int drift, int deposit, double kick_factor) {
    PushArgs A{};
    A.state = S.d_state;
    for (int s = 0; s < S.ns; ++s) {
        A.sp[s] = S.sc[s];
        const pic_species_desc& sp = S.d.species[s];
        A.sp[s].kq = float(sp.charge / sp.mass * S.d.dt * kick_factor);
    }
    A.items = S.items;
    A.n_items = S.n_items;
    A.item_next = S.item_next;
    A.E = S.E2;
    A.ep = S.ep;
    A.ew = S.ew;
    A.emap = S.emap;
    A.rho = S.rho_acc;
    A.nx = S.nx;
    A.ny = S.ny;
    A.tile = S.d.tile;
    A.tiles_x = S.have_sorter ? S.sorter.tiles_x : 1;
    A.rw = S.rw;
    A.do_kick = kick;
    A.do_mcc = mcc && S.have_mcc;
    A.do_drift = drift;
    A.do_deposit = deposit;
    A.mcc = S.mcc_dev;
    A.key = make_uint2(uint32_t(S.d.seed), uint32_t(S.d.seed >> 32));
    A.step = S.step_ctr;
    for (int s = 0; s < S.ns; ++s) A.cbits[s] = S.cbits[s];
    A.vbits = S.vbits;
    A.hbits = S.hbits;
    A.electrodes = S.electrodes ? 1 : 0;
    A.rz = S.rz ? 1 : 0;
    A.cand = S.cand;
    A.cand_state = S.cand_state;
    A.cand_count = S.cand_count;
    A.cand_cap = S.cand_cap;
    A.ctr = S.ctr;
    A.error = S.error;
    A.wait_limit = S.wait_limit;
    return A;
}

// The preparation of a particle pass: work items for the current particle
// state (and the step counter, when advance_step), then, for a pass with
// collisions, the null-collision candidate bits of that step.  It reads only
// the particle state, so a captured step runs the next step's preparation
// beside its own field solve.
static int prepare_pass(SimImpl& S, cudaStream_t st, int mcc, int advance_step) {
    {
        PhaseTimer t(S, PIC_PHASE_BUILD, st);
        k_build_items<<<1, 256, 0, st>>>(S.d_state, S.ns, S.n_tiled, S.items, S.n_items, S.item_next, S.step_ctr,
                                         S.cand_count, advance_step);
        if (mcc && S.have_mcc) {
            const uint2 key = make_uint2(uint32_t(S.d.seed), uint32_t(S.d.seed >> 32));
            k_mcc_bits<<<div_up(S.cbits_segments, 256), 256, 0, st>>>(S.mcc_dev, S.ns, S.step_ctr, key, S.d_cbits,
                                                                     S.d_nseg);
            S.launches += 1;
        }
    }
    S.launches += 1;
    PIC_LAUNCH_CHECK();
    return PIC_OK;
}

// The particle pass itself, once prepare_pass has run for it.
static int run_pass_tail(SimImpl& S, cudaStream_t st, const PushArgs& A);

static int run_pass(SimImpl& S, cudaStream_t st, int kick, int mcc, int drift, int deposit, double kick_factor) {
    const PushArgs A = push_args(S, kick, mcc, drift, deposit, kick_factor);
    {
        PhaseTimer t(S, PIC_PHASE_PUSH, st);
        const bool full = kick && drift && deposit;
        if (S.push_kernel == PIC_PUSH_WARP || S.push_kernel == PIC_PUSH_WARP_AGG) {
            const int g = S.push_grid_w;
            const size_t sm = S.push_smem_w;
            const bool agg = S.push_kernel == PIC_PUSH_WARP_AGG;
            if (S.rz) {
                if (full) {
                    if (agg) k_push_warp<true, true, true><<<g, kPushThreads, sm, st>>>(A);
                    else k_push_warp<true, true, false><<<g, kPushThreads, sm, st>>>(A);
                } else {
                    if (agg) k_push_warp<true, false, true><<<g, kPushThreads, sm, st>>>(A);
                    else k_push_warp<true, false, false><<<g, kPushThreads, sm, st>>>(A);
                }
            } else {
                if (full) {
                    if (agg) k_push_warp<false, true, true><<<g, kPushThreads, sm, st>>>(A);
                    else k_push_warp<false, true, false><<<g, kPushThreads, sm, st>>>(A);
                } else {
                    if (agg) k_push_warp<false, false, true><<<g, kPushThreads, sm, st>>>(A);
                    else k_push_warp<false, false, false><<<g, kPushThreads, sm, st>>>(A);
                }
            }
        } else if (S.push_kernel == PIC_PUSH_PIPE) {
            if (S.rz) {
                if (full) k_push_pipe<true, true><<<S.push_grid, kPushThreads, S.push_smem, st>>>(A);
                else k_push_pipe<true, false><<<S.push_grid, kPushThreads, S.push_smem, st>>>(A);
            } else {
                if (full) k_push_pipe<false, true><<<S.push_grid, kPushThreads, S.push_smem, st>>>(A);
                else k_push_pipe<false, false><<<S.push_grid, kPushThreads, S.push_smem, st>>>(A);
            }
        } else if (S.rz) {
            if (full) k_push<true, true><<<S.push_grid, kPushThreads, S.push_smem, st>>>(A);
            else k_push<true, false><<<S.push_grid, kPushThreads, S.push_smem, st>>>(A);
        } else {
            if (full) k_push<false, true><<<S.push_grid, kPushThreads, S.push_smem, st>>>(A);
            else k_push<false, false><<<S.push_grid, kPushThreads, S.push_smem, st>>>(A);
        }
    }
    S.launches += 1;
    return run_pass_tail(S, st, A);
}

// What follows a particle pass with collisions: the collision candidates and
// their ionisation products (k_collide).
static int run_pass_tail(SimImpl& S, cudaStream_t st, const PushArgs& A) {
    if (A.do_mcc) {
        PhaseTimer t(S, PIC_PHASE_MERGE, st);
        // one thread per candidate: each is a long chain of dependent
        // table lookups and Philox rounds
        k_collide<<<4 * num_sms(), 128, 0, st>>>(A, S.mcc.dev);
        S.launches += 1;
    }
    PIC_LAUNCH_CHECK();
    return PIC_OK;
}

static int particle_pass(SimImpl& S, cudaStream_t st, int kick, int mcc, int drift, int deposit, double kick_factor,
                         int advance_step) {
    PIC_TRY(prepare_pass(S, st, mcc, advance_step));
    return run_pass(S, st, kick, mcc, drift, deposit, kick_factor);
}

static int field_solve(SimImpl& S, cudaStream_t st, bool capturing) {
    {
        PhaseTimer t(S, PIC_PHASE_RHS, st);
        // from the second solve on, the guess is extrapolated from the last two potentials
        PIC_TRY(launch_form_rhs(S.rho_acc, S.dirichlet, S.d.eps0, S.f, S.rho_out, S.rho_acc, S.phi,
                                S.have_prev ? S.phi_prev : nullptr, S.G, st, S.rowf, S.nx));
    }
    {
        PhaseTimer t(S, PIC_PHASE_SOLVE, st);
        if (capturing) PIC_TRY(mg_capture_into(S.mg, S.phi, S.f, S.d.tol, S.d.max_cycles, S.d.min_cycles, st));
        else PIC_TRY(mg_launch_graph(S.mg, S.phi, S.f, S.d.tol, S.d.max_cycles, S.d.min_cycles, st));
    }
    if (!S.have_prev) {
        PIC_CUDA(cudaMemcpyAsync(S.phi_prev, S.phi, sizeof(double) * S.G, cudaMemcpyDeviceToDevice, st));
        S.have_prev = true;
    }
    {
        PhaseTimer t(S, PIC_PHASE_EFIELD, st);
        PIC_TRY(launch_update_E(S.phi, S.Ex, S.Ey, S.E2, S.ep, S.nx, S.ny, S.d.dx, S.d.dy, st, S.rz));
    }
    S.launches += 2;
    S.solves += 1;
    return PIC_OK;
}

static int sort_all(SimImpl& S, cudaStream_t st) {
    PhaseTimer t(S, PIC_PHASE_SORT, st);
    SortImpl& R = S.sorter;
    S.launches += 1 + (long long)(S.ns) * (5 + 3 * R.passes);
    for (int s = 0; s < S.ns; ++s) {
        int* count_ptr = reinterpret_cast<int*>(reinterpret_cast<char*>(S.d_state + s) + offsetof(SpeciesState, count));
        PIC_TRY(sort_set_n(R, count_ptr, st));
        k_sim_keys<<<grid_blocks(S.d.species[s].capacity, 256), 256, 0, st>>>(
            S.d_state, s, S.nx - 1, S.ny - 1, R.tile, R.tiles_x, R.dead_key, R.k0, R.v0, R.n_dev);
        const uint32_t* perm = nullptr;
        PIC_TRY(sort_passes(R, S.tile_start + s * (R.ntiles + 1), nullptr, &perm, st));
        k_sim_gather<<<grid_blocks(S.d.species[s].capacity, 256), 256, 0, st>>>(S.d_state, s, perm, R.n_dev);
        k_sim_flip<<<1, 1, 0, st>>>(S.d_state, s, R.n_dev);
    }
    k_tile_items<<<1, 1024, 0, st>>>(S.tile_start, R.ntiles, S.ns, S.items, S.n_tiled);
    PIC_LAUNCH_CHECK();
    return PIC_OK;
}

// sort_all as one graph launch (captured at the first call): its forty-odd
// small launches are then enqueued by one call, so that the GPU does not wait
// on the host between them.  Profiling launches them one by one.
static int sort_all_graph(SimImpl& S, cudaStream_t st) {
    if (S.profiling) return sort_all(S, st);
    if (!S.g_sort) {
        const long long l0 = S.launches;
        PIC_CUDA(cudaStreamBeginCapture(S.cap, cudaStreamCaptureModeThreadLocal));
        const int rc = sort_all(S, S.cap);
        cudaGraph_t g = nullptr;
        const cudaError_t ec = cudaStreamEndCapture(S.cap, &g);
        S.sort_graph_launches = S.launches - l0;
        S.launches = l0;
        if (rc != PIC_OK) {
            if (g) cudaGraphDestroy(g);
            return rc;
        }
        if (ec != cudaSuccess) return fail(PIC_ERR_CUDA, "sort capture: %s", cudaGetErrorString(ec));
        const cudaError_t ei = cudaGraphInstantiate(&S.g_sort, g, 0);
        cudaGraphDestroy(g);
        if (ei != cudaSuccess) return fail(PIC_ERR_CUDA, "sort graph: %s", cudaGetErrorString(ei));
    }
    PIC_CUDA(cudaGraphLaunch(S.g_sort, st));
    S.launches += S.sort_graph_launches;
    return PIC_OK;
}

// The steady-state step captured once into a CUDA graph: the particle pass
// (kick + MCC + drift + deposit, prepared beforehand), then the field solve
// (RHS, multigrid, E) on the capture stream and, on a side branch beside it,
// the next step's preparation (its cell sort when sort_next, work items,
// candidate bits), which reads only the particle state.
static int capture_step(SimImpl& S, bool sort_next, cudaGraphExec_t* out) {
    const bool prof = S.profiling;
    S.profiling = false;
    const long long l0 = S.launches, s0 = S.solves;
    PIC_CUDA(cudaStreamBeginCapture(S.cap, cudaStreamCaptureModeThreadLocal));
    int rc = run_pass(S, S.cap, 1, 1, 1, 1, 1.0);
    bool forked = false;
    if (rc == PIC_OK && cudaEventRecord(S.ev_fork, S.cap) == cudaSuccess &&
        cudaStreamWaitEvent(S.cap2, S.ev_fork, 0) == cudaSuccess) {
        forked = true;
        if (sort_next) rc = sort_all(S, S.cap2);
        if (rc == PIC_OK) rc = prepare_pass(S, S.cap2, 1, 1);
        if (cudaEventRecord(S.ev_join, S.cap2) != cudaSuccess && rc == PIC_OK)
            rc = fail(PIC_ERR_CUDA, "step capture: join event");
    }
    if (rc == PIC_OK) rc = field_solve(S, S.cap, true);
    if (forked) cudaStreamWaitEvent(S.cap, S.ev_join, 0);
    cudaGraph_t g = nullptr;
    const cudaError_t ec = cudaStreamEndCapture(S.cap, &g);
    S.profiling = prof;
    S.launches = l0;  // counted when the graph is launched
    S.solves = s0;
    if (rc != PIC_OK) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    if (ec != cudaSuccess) return fail(PIC_ERR_CUDA, "step capture: %s", cudaGetErrorString(ec));
    const cudaError_t ei = cudaGraphInstantiate(out, g, 0);
    cudaGraphDestroy(g);
    if (ei != cudaSuccess) return fail(PIC_ERR_CUDA, "step graph instantiate: %s", cudaGetErrorString(ei));
    return PIC_OK;
}

static int sim_create(const pic_sim_desc* d, cudaStream_t st, SimImpl& S) {
    if (!d || d->nx < 3 || d->ny < 3 || !(d->dx > 0) || !(d->dy > 0) || !(d->dt > 0) || !(d->eps0 > 0) ||
        d->nspecies < 1 || d->nspecies > PIC_MAX_SPECIES || !d->h_dirichlet || !(d->tol > 0) || d->max_cycles < 1 ||
        d->min_cycles < 0)
        return fail(PIC_ERR_BAD_ARG, "pic_sim_create: bad descriptor");
    S.d = *d;
    if (S.d.tile <= 0) S.d.tile = 16;
    S.nx = d->nx;
    S.ny = d->ny;
    S.ns = d->nspecies;
    S.G = long(S.nx) * S.ny;
    S.rw = S.d.tile + 1 + 2 * kHalo;
    S.ew = (S.rw + 1) & ~1;
    PIC_TRY(mg_create(S.nx, S.ny, d->dx, d->dy, d->h_dirichlet, &d->mg, &S.mg));
    if (d->mg.geometry == PIC_GEOM_RZ) {
        // r-z: deposits become densities with the node volumes of each row
        S.rz = true;
        std::vector<double> f(size_t(S.ny)), v(size_t(S.ny));
        for (int j = 0; j < S.ny; ++j) {
            v[j] = rz_row_volume(j, S.ny, d->dy);
            f[j] = 1.0 / v[j];
        }
        PIC_TRY(dalloc(S, &S.rowf, size_t(S.ny)));
        PIC_TRY(dalloc(S, &S.rowv, size_t(S.ny)));
        PIC_CUDA(cudaMemcpy(S.rowf, f.data(), sizeof(double) * S.ny, cudaMemcpyHostToDevice));
        PIC_CUDA(cudaMemcpy(S.rowv, v.data(), sizeof(double) * S.ny, cudaMemcpyHostToDevice));
    }
    long max_cap = 0;
    for (int s = 0; s < S.ns; ++s) {
        const pic_species_desc& sp = d->species[s];
        if (sp.capacity < 1 || !(sp.mass > 0) || !(sp.np2c > 0))
            return fail(PIC_ERR_BAD_ARG, "pic_sim_create: species %d needs capacity, mass and np2c", s);
        max_cap = std::max<long>(max_cap, sp.capacity);
    }
    PIC_TRY(sorter_create(int(max_cap), S.nx, S.ny, S.d.tile, &S.sorter));
    S.have_sorter = true;
    if (d->mcc) {
        double mass[PIC_MAX_SPECIES];
        for (int s = 0; s < S.ns; ++s) mass[s] = d->species[s].mass;
        PIC_TRY(mcc_build(d->mcc, S.ns, mass, d->dt, &S.mcc));
        S.have_mcc = true;
    }
    PIC_TRY(dalloc(S, &S.mcc_dev, 1));
    if (S.have_mcc) PIC_CUDA(cudaMemcpy(S.mcc_dev, &S.mcc.dev, sizeof(MccDev), cudaMemcpyHostToDevice));
    // species buffers
    for (int s = 0; s < S.ns; ++s) {
        const pic_species_desc& sp = d->species[s];
        SpeciesState& H = S.h_state[s];
        // one allocation per buffer set; each array padded to a multiple of 4
        // floats so that every array starts 16-byte aligned
        const int stride = ((sp.capacity + kArraySlack + 3) / 4) * 4;
        float *cur = nullptr, *alt = nullptr;
        PIC_TRY(dalloc(S, &cur, size_t(stride) * 5));
        PIC_TRY(dalloc(S, &alt, size_t(stride) * 5));
        for (int c = 0; c < 5; ++c) {
            H.cur[c] = cur + size_t(c) * stride;
            H.alt[c] = alt + size_t(c) * stride;
        }
        H.stride = stride;
        H.count = 0;
        H.sorted_end = 0;
        H.capacity = sp.capacity;
        SpeciesConst& C = S.sc[s];
        C.kq = float(sp.charge / sp.mass * d->dt);
        C.dtdx = float(d->dt / d->dx);
        C.dtdy = float(d->dt / d->dy);
        C.scale = float(sp.charge * sp.np2c / (d->dx * d->dy));
    }
    PIC_TRY(dalloc(S, &S.d_state, size_t(S.ns)));
    PIC_CUDA(cudaMemcpy(S.d_state, S.h_state, sizeof(SpeciesState) * S.ns, cudaMemcpyHostToDevice));
    // work items
    S.item_cap = 4;
    for (int s = 0; s < S.ns; ++s) S.item_cap += S.sorter.ntiles + 2 * (d->species[s].capacity / kUnitMax + 2);
    PIC_TRY(dalloc(S, &S.items, size_t(S.item_cap)));
    PIC_TRY(dalloc(S, &S.n_items, 1));
    PIC_TRY(dalloc(S, &S.item_next, 1));
    PIC_TRY(dalloc(S, &S.n_tiled, 1));
    PIC_TRY(dalloc(S, &S.step_ctr, 1));
    PIC_TRY(dalloc(S, &S.tile_start, size_t(S.ns) * (S.sorter.ntiles + 1)));
    // candidates per pass: P_null N on average (binomial); eight times the mean plus a margin
    double expect = 0.0;
    if (S.have_mcc)
        for (int s = 0; s < S.ns; ++s) expect += S.mcc.p_null[s] * d->species[s].capacity;
    S.cand_cap = int(std::min(2.0e9, 8.0 * expect + 65536.0));
    PIC_TRY(dalloc(S, &S.cand, size_t(S.cand_cap)));
    PIC_TRY(dalloc(S, &S.cand_state, size_t(S.cand_cap)));
    // candidate bit masks, one bit per slot of every colliding species
    {
        int nseg[PIC_MAX_SPECIES] = {};
        S.cbits_segments = 0;
        for (int s = 0; s < S.ns; ++s) {
            if (!S.have_mcc || S.mcc.dev.sp[s].nproc == 0) continue;
            nseg[s] = div_up(d->species[s].capacity + kArraySlack, kMccSegment);
            PIC_TRY(dalloc(S, &S.cbits[s], size_t(nseg[s]) * (kMccSegment / 32)));
            S.cbits_segments += nseg[s];
        }
        PIC_TRY(dalloc(S, &S.d_cbits, size_t(PIC_MAX_SPECIES)));
        PIC_CUDA(cudaMemcpy(S.d_cbits, S.cbits, sizeof(unsigned*) * PIC_MAX_SPECIES, cudaMemcpyHostToDevice));
        PIC_TRY(dalloc(S, &S.d_nseg, size_t(PIC_MAX_SPECIES)));
        PIC_CUDA(cudaMemcpy(S.d_nseg, nseg, sizeof(int) * PIC_MAX_SPECIES, cudaMemcpyHostToDevice));
    }
    PIC_TRY(dalloc(S, &S.cand_count, 1));
    PIC_TRY(dalloc(S, &S.ctr, size_t(kCtrCount)));
    PIC_TRY(dalloc(S, &S.error, 1));
    // fields
    S.ep = (S.nx + 1) & ~1;
    PIC_TRY(dalloc(S, &S.E2, size_t(S.ep) * S.ny));
    PIC_TRY(encode_e_map(S));
    PIC_TRY(dalloc(S, &S.Ex, size_t(S.G)));
    PIC_TRY(dalloc(S, &S.Ey, size_t(S.G)));
    PIC_TRY(dalloc(S, &S.rho_acc, size_t(S.G)));
    PIC_TRY(dalloc(S, &S.rho_out, size_t(S.G)));
    PIC_TRY(dalloc(S, &S.phi, size_t(S.G)));
    PIC_TRY(dalloc(S, &S.phi_prev, size_t(S.G)));
    PIC_TRY(dalloc(S, &S.f, size_t(S.G)));
    PIC_TRY(dalloc(S, &S.dirichlet, size_t(S.G)));
    std::vector<uint8_t> mask(d->h_dirichlet, d->h_dirichlet + S.G);
    for (auto& v : mask) v = v ? 1 : 0;
    PIC_CUDA(cudaMemcpy(S.dirichlet, mask.data(), S.G, cudaMemcpyHostToDevice));
    // internal electrode edges: grid-line segments between two internal Dirichlet nodes
    {
        const int nx = S.nx, ny = S.ny;
        auto inner_dir = [&](int i, int j) {
            return i > 0 && j > 0 && i < nx - 1 && j < ny - 1 && mask[size_t(j) * nx + i];
        };
        const long nv = long(nx) * (ny - 1), nh = long(nx - 1) * ny;
        std::vector<unsigned> vb((nv + 31) / 32, 0u), hb((nh + 31) / 32, 0u);
        for (int X = 1; X < nx - 1; ++X)
            for (int j = 0; j + 1 < ny; ++j) {
                // an edge with one end on the domain boundary still belongs to the electrode
                const bool a = inner_dir(X, j) || (j == 0 && mask[size_t(j) * nx + X]);
                const bool b = inner_dir(X, j + 1) || (j + 1 == ny - 1 && mask[size_t(j + 1) * nx + X]);
                if (a && b && (inner_dir(X, j) || inner_dir(X, j + 1))) {
                    const long k = long(X) * (ny - 1) + j;
                    vb[k >> 5] |= 1u << (k & 31);
                    S.electrodes = true;
                }
            }
        for (int Y = 1; Y < ny - 1; ++Y)
            for (int i = 0; i + 1 < nx; ++i) {
                const bool a = inner_dir(i, Y) || (i == 0 && mask[size_t(Y) * nx + i]);
                const bool b = inner_dir(i + 1, Y) || (i + 1 == nx - 1 && mask[size_t(Y) * nx + i + 1]);
                if (a && b && (inner_dir(i, Y) || inner_dir(i + 1, Y))) {
                    const long k = long(Y) * (nx - 1) + i;
                    hb[k >> 5] |= 1u << (k & 31);
                    S.electrodes = true;
                }
            }
        PIC_TRY(dalloc(S, &S.vbits, vb.size()));
        PIC_TRY(dalloc(S, &S.hbits, hb.size()));
        PIC_CUDA(cudaMemcpy(S.vbits, vb.data(), sizeof(unsigned) * vb.size(), cudaMemcpyHostToDevice));
        PIC_CUDA(cudaMemcpy(S.hbits, hb.data(), sizeof(unsigned) * hb.size(), cudaMemcpyHostToDevice));
    }
    if (d->h_phi_bc) {
        std::vector<double> phi0(S.G, 0.0);
        for (long k = 0; k < S.G; ++k)
            if (mask[k]) phi0[k] = d->h_phi_bc[k];
        PIC_CUDA(cudaMemcpy(S.phi, phi0.data(), sizeof(double) * S.G, cudaMemcpyHostToDevice));
    }
    // launch shape of the particle pass
    S.push_smem = sizeof(float) * kStages * 4 * kBufStride + sizeof(unsigned) * kStages * kCbWords +
                  size_t(S.rw) * S.rw * (sizeof(float4) + sizeof(unsigned));
    const void* push_fns[4] = {reinterpret_cast<const void*>(k_push<false, false>),
                               reinterpret_cast<const void*>(k_push<false, true>),
                               reinterpret_cast<const void*>(k_push<true, false>),
                               reinterpret_cast<const void*>(k_push<true, true>)};
    for (const void* fn : push_fns) PIC_TRY(raise_smem_limit(fn, S.push_smem));
    const void* pipe_fns[4] = {reinterpret_cast<const void*>(k_push_pipe<false, false>),
                               reinterpret_cast<const void*>(k_push_pipe<false, true>),
                               reinterpret_cast<const void*>(k_push_pipe<true, false>),
                               reinterpret_cast<const void*>(k_push_pipe<true, true>)};
    for (const void* fn : pipe_fns) PIC_TRY(raise_smem_limit(fn, S.push_smem));
    // the grid of the step's instance (the others run the same grid)
    const void* push_fn = push_fns[S.rz ? 3 : 1];
    int per_sm = 0;
    PIC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, push_fn, kPushThreads, S.push_smem));
    S.push_grid = std::max(1, per_sm) * num_sms();
    if (d->push_kernel != PIC_PUSH_RING && d->push_kernel != PIC_PUSH_WARP && d->push_kernel != PIC_PUSH_WARP_AGG &&
        d->push_kernel != PIC_PUSH_PIPE)
        return fail(PIC_ERR_BAD_ARG, "pic_sim_create: push_kernel %d", d->push_kernel);
    // k_push_warp's E-tile loads start at x = tile * tx - 4, which the tensor
    // copy needs even (16-byte aligned): an odd tile takes the ring kernel
    S.push_kernel = (S.d.tile & 1) ? int(PIC_PUSH_RING) : d->push_kernel;
    S.push_smem_w = sizeof(float) * kPushWarps * kWarpStages * 4 * kWarpGroup +
                    2 * ((size_t(S.ew) * S.rw * sizeof(float2) + 127) / 128 * 128) +
                    size_t(S.rw) * S.rw * sizeof(unsigned);
    const void* warp_fns[8] = {reinterpret_cast<const void*>(k_push_warp<false, false, true>),
                               reinterpret_cast<const void*>(k_push_warp<false, true, true>),
                               reinterpret_cast<const void*>(k_push_warp<true, false, true>),
                               reinterpret_cast<const void*>(k_push_warp<true, true, true>),
                               reinterpret_cast<const void*>(k_push_warp<false, false, false>),
                               reinterpret_cast<const void*>(k_push_warp<false, true, false>),
                               reinterpret_cast<const void*>(k_push_warp<true, false, false>),
                               reinterpret_cast<const void*>(k_push_warp<true, true, false>)};
    for (const void* fn : warp_fns) PIC_TRY(raise_smem_limit(fn, S.push_smem_w));
    per_sm = 0;
    PIC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, warp_fns[S.rz ? 3 : 1], kPushThreads,
                                                           S.push_smem_w));
    S.push_grid_w = std::max(1, per_sm) * num_sms();
    PIC_CUDA(cudaStreamCreateWithFlags(&S.cap, cudaStreamNonBlocking));
    PIC_CUDA(cudaStreamCreateWithFlags(&S.cap2, cudaStreamNonBlocking));
    PIC_CUDA(cudaEventCreateWithFlags(&S.ev_fork, cudaEventDisableTiming));
    PIC_CUDA(cudaEventCreateWithFlags(&S.ev_join, cudaEventDisableTiming));
    (void)st;
    return PIC_OK;
}

static void sim_free(SimImpl& S) {
    if (S.g_step) cudaGraphExecDestroy(S.g_step);
    if (S.g_sort_step) cudaGraphExecDestroy(S.g_sort_step);
    if (S.g_sort) cudaGraphExecDestroy(S.g_sort);
    S.g_step = S.g_sort_step = S.g_sort = nullptr;
    if (S.cap) cudaStreamDestroy(S.cap);
    if (S.cap2) cudaStreamDestroy(S.cap2);
    if (S.ev_fork) cudaEventDestroy(S.ev_fork);
    if (S.ev_join) cudaEventDestroy(S.ev_join);
    S.cap = nullptr;
    for (auto& m : S.marks) {
        cudaEventDestroy(m.second.first);
        cudaEventDestroy(m.second.second);
    }
    S.marks.clear();
    for (cudaEvent_t e : S.event_pool) cudaEventDestroy(e);
    S.event_pool.clear();
    if (S.mg) pic_mg_destroy(S.mg);
    S.mg = nullptr;
    if (S.have_sorter) sorter_free(&S.sorter);
    if (S.have_mcc) mcc_free(&S.mcc);
    for (void* p : S.allocs) cudaFree(p);
    S.allocs.clear();
}

// ---- ensembles: many independent simulations in one graph --------------------------
//
// One CUDA graph holds a step of every member as independent branches and a
// conditional WHILE node repeats it, so n steps of the whole ensemble are one
// graph launch.  A member's branch:
//     k_ens_sort_cond -> IF { cell sort } -> particle pass -> field solve
//     (its multigrid loop is a nested WHILE node) -> k_ens_advance
// The IF condition is the member's own step counter (on the device) modulo
// its sort interval, so members with different intervals share one graph.

struct EnsControl {
    long long remaining;  // ensemble steps left in this launch
};

__global__ void k_ens_sort_cond(const long long* __restrict__ steps, int interval, cudaGraphConditionalHandle h) {
    cudaGraphSetConditional(h, (interval > 0 && *steps % interval == 0) ? 1u : 0u);
}

__global__ void k_ens_advance(long long* steps) { *steps += 1; }

__global__ void k_ens_loop(EnsControl* c, cudaGraphConditionalHandle h) {
    c->remaining -= 1;
    cudaGraphSetConditional(h, c->remaining > 0 ? 1u : 0u);
}

// The flat numbering of every member's work items for one particle pass over
// the ensemble, and its claim counter reset (one thread).
__global__ void k_ens_items(const PushArgs* __restrict__ members, int n, int* member_items, int* next) {
    int total = 0;
    for (int m = 0; m < n; ++m) {
        member_items[m] = total;
        total += *members[m].n_items;
    }
    member_items[n] = total;
    *next = 0;
}

struct EnsImpl {
    std::vector<SimImpl*> m;
    std::vector<cudaStream_t> branch, side;
    std::vector<cudaEvent_t> ev;
    cudaStream_t cap = nullptr;
    long long* d_steps = nullptr;
    EnsControl* d_ctl = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::vector<long long> per_step_launches;  // per member, without the sort
    std::vector<long long> sort_launches;
    // one particle pass over every member (when every member uses the ring
    // pass and the same geometry): the members' arguments, the flat item
    // numbering and its claim counter, the launch shape
    bool fused = false;
    bool rz = false;
    PushArgs* d_members = nullptr;
    int* d_member_items = nullptr;
    int* d_next = nullptr;
    int push_grid = 0;
    size_t push_smem = 0;
    int rw_max = 0;
};

// Decides whether the members' particle passes run as one launch, and sets it up.
static int ens_setup_fused(EnsImpl& E) {
    const int n = int(E.m.size());
    E.fused = true;
    E.rz = E.m[0]->rz;
    E.rw_max = 0;
    E.push_smem = 0;
    for (SimImpl* S : E.m) {
        if (S->push_kernel != PIC_PUSH_RING || S->rz != E.rz) E.fused = false;
        E.rw_max = std::max(E.rw_max, S->rw);
        E.push_smem = std::max(E.push_smem, S->push_smem);
    }
    if (!E.fused) return PIC_OK;
    std::vector<PushArgs> h(n);
    for (int i = 0; i < n; ++i) h[i] = push_args(*E.m[i], 1, 1, 1, 1, 1.0);
    PIC_CUDA(cudaMalloc(&E.d_members, sizeof(PushArgs) * n));
    PIC_CUDA(cudaMalloc(&E.d_member_items, sizeof(int) * (n + 1)));
    PIC_CUDA(cudaMalloc(&E.d_next, sizeof(int)));
    PIC_CUDA(cudaMemcpy(E.d_members, h.data(), sizeof(PushArgs) * n, cudaMemcpyHostToDevice));
    const void* fn = E.rz ? reinterpret_cast<const void*>(k_push<true, true, true>)
                          : reinterpret_cast<const void*>(k_push<false, true, true>);
    PIC_TRY(raise_smem_limit(fn, E.push_smem));
    int per_sm = 0;
    PIC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kPushThreads, E.push_smem));
    E.push_grid = std::max(1, per_sm) * num_sms();
    return PIC_OK;
}

// The arguments of the fused pass: the members' own, through d_members.
static PushArgs ens_push_args(const EnsImpl& E) {
    PushArgs A = push_args(*E.m[0], 1, 1, 1, 1, 1.0);
    A.members = E.d_members;
    A.member_items = E.d_member_items;
    A.nmembers = int(E.m.size());
    A.n_items = E.d_member_items + E.m.size();
    A.item_next = E.d_next;
    A.rw = E.rw_max;
    return A;
}

// Adds, to the graph that st is capturing into, a conditional IF node whose
// body is the member's cell sort, and moves st past it.
static int capture_sort_if(SimImpl& S, long long* d_step, cudaStream_t st, cudaStream_t side) {
    cudaStreamCaptureStatus cs;
    cudaGraph_t g = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t nd = 0;
    PIC_CUDA(cudaStreamGetCaptureInfo(st, &cs, nullptr, &g, &deps, &nd));
    if (cs != cudaStreamCaptureStatusActive) return fail(PIC_ERR_BAD_ARG, "ensemble: stream is not capturing");
    cudaGraphConditionalHandle h;
    PIC_CUDA(cudaGraphConditionalHandleCreate(&h, g, 0, cudaGraphCondAssignDefault));
    k_ens_sort_cond<<<1, 1, 0, st>>>(d_step, S.d.sort_interval, h);
    PIC_LAUNCH_CHECK();
    PIC_CUDA(cudaStreamGetCaptureInfo(st, &cs, nullptr, &g, &deps, &nd));
    cudaGraphNodeParams p{};
    p.type = cudaGraphNodeTypeConditional;
    p.conditional.handle = h;
    p.conditional.type = cudaGraphCondTypeIf;
    p.conditional.size = 1;
    cudaGraphNode_t cn;
    PIC_CUDA(cudaGraphAddNode(&cn, g, deps, nd, &p));
    cudaGraph_t body = p.conditional.phGraph_out[0];
    PIC_CUDA(cudaStreamUpdateCaptureDependencies(st, &cn, 1, cudaStreamSetCaptureDependencies));
    PIC_CUDA(cudaStreamBeginCaptureToGraph(side, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
    const int rc = sort_all(S, side);
    cudaGraph_t out = nullptr;
    const cudaError_t ec = cudaStreamEndCapture(side, &out);
    if (rc != PIC_OK) return rc;
    if (ec != cudaSuccess) return fail(PIC_ERR_CUDA, "ensemble sort capture: %s", cudaGetErrorString(ec));
    return PIC_OK;
}

static int ens_capture_body(EnsImpl& E);

static int ens_capture(EnsImpl& E) {
    // launches are counted when the graph runs; phase timing stays out of graphs
    std::vector<long long> l0, s0;
    std::vector<bool> prof;
    for (SimImpl* S : E.m) {
        l0.push_back(S->launches);
        s0.push_back(S->solves);
        prof.push_back(S->profiling);
        S->profiling = false;
    }
    const int rc = ens_capture_body(E);
    for (size_t i = 0; i < E.m.size(); ++i) {
        E.m[i]->launches = l0[i];
        E.m[i]->solves = s0[i];
        E.m[i]->profiling = prof[i];
    }
    return rc;
}

static int ens_capture_body(EnsImpl& E) {
    const int n = int(E.m.size());
    PIC_CUDA(cudaStreamBeginCapture(E.cap, cudaStreamCaptureModeThreadLocal));
    int rc = PIC_OK;
    cudaGraph_t g = nullptr;
    do {
        cudaStreamCaptureStatus cs;
        cudaGraph_t top = nullptr;
        const cudaGraphNode_t* deps = nullptr;
        size_t nd = 0;
        if (cudaStreamGetCaptureInfo(E.cap, &cs, nullptr, &top, &deps, &nd) != cudaSuccess) {
            rc = fail(PIC_ERR_CUDA, "ensemble: capture info");
            break;
        }
        cudaGraphConditionalHandle h;
        if (cudaGraphConditionalHandleCreate(&h, top, 1, cudaGraphCondAssignDefault) != cudaSuccess) {
            rc = fail(PIC_ERR_CUDA, "ensemble: conditional handle");
            break;
        }
        cudaGraphNodeParams p{};
        p.type = cudaGraphNodeTypeConditional;
        p.conditional.handle = h;
        p.conditional.type = cudaGraphCondTypeWhile;
        p.conditional.size = 1;
        cudaGraphNode_t cn;
        if (cudaGraphAddNode(&cn, top, deps, nd, &p) != cudaSuccess ||
            cudaStreamUpdateCaptureDependencies(E.cap, &cn, 1, cudaStreamSetCaptureDependencies) != cudaSuccess) {
            rc = fail(PIC_ERR_CUDA, "ensemble: loop node");
            break;
        }
        cudaGraph_t body = p.conditional.phGraph_out[0];
        // the loop body is captured on branch 0's stream as the root, forked to every member
        cudaStream_t root = E.side.back();
        if (cudaStreamBeginCaptureToGraph(root, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed) !=
            cudaSuccess) {
            rc = fail(PIC_ERR_CUDA, "ensemble: body capture");
            break;
        }
        if (cudaEventRecord(E.ev[n], root) != cudaSuccess) rc = fail(PIC_ERR_CUDA, "ensemble: fork event");
        if (E.fused) {
            // every member's sort and preparation as a branch, one particle
            // pass over all members, then every member's field solve as a branch
            for (int i = 0; i < n && rc == PIC_OK; ++i) {
                SimImpl& S = *E.m[i];
                cudaStream_t st = E.branch[i];
                if (cudaStreamWaitEvent(st, E.ev[n], 0) != cudaSuccess) rc = fail(PIC_ERR_CUDA, "ensemble: fork wait");
                if (rc == PIC_OK && S.d.sort_interval > 0) rc = capture_sort_if(S, E.d_steps + i, st, E.side[i]);
                if (rc == PIC_OK) rc = prepare_pass(S, st, 1, 1);
                if (rc == PIC_OK &&
                    (cudaEventRecord(E.ev[i], st) != cudaSuccess || cudaStreamWaitEvent(root, E.ev[i], 0) != cudaSuccess))
                    rc = fail(PIC_ERR_CUDA, "ensemble: join of member %d", i);
            }
            if (rc == PIC_OK) {
                k_ens_items<<<1, 1, 0, root>>>(E.d_members, n, E.d_member_items, E.d_next);
                const PushArgs A = ens_push_args(E);
                if (E.rz) k_push<true, true, true><<<E.push_grid, kPushThreads, E.push_smem, root>>>(A);
                else k_push<false, true, true><<<E.push_grid, kPushThreads, E.push_smem, root>>>(A);
                if (cudaGetLastError() != cudaSuccess || cudaEventRecord(E.ev[n], root) != cudaSuccess)
                    rc = fail(PIC_ERR_CUDA, "ensemble: particle pass");
            }
            for (int i = 0; i < n && rc == PIC_OK; ++i) {
                SimImpl& S = *E.m[i];
                cudaStream_t st = E.branch[i];
                if (cudaStreamWaitEvent(st, E.ev[n], 0) != cudaSuccess) rc = fail(PIC_ERR_CUDA, "ensemble: fork wait");
                if (rc == PIC_OK) rc = run_pass_tail(S, st, push_args(S, 1, 1, 1, 1, 1.0));
                if (rc == PIC_OK) rc = field_solve(S, st, true);
                if (rc == PIC_OK) {
                    k_ens_advance<<<1, 1, 0, st>>>(E.d_steps + i);
                    if (cudaEventRecord(E.ev[i], st) != cudaSuccess ||
                        cudaStreamWaitEvent(root, E.ev[i], 0) != cudaSuccess)
                        rc = fail(PIC_ERR_CUDA, "ensemble: join of member %d", i);
                }
            }
        }
        for (int i = 0; i < n && rc == PIC_OK && !E.fused; ++i) {
            SimImpl& S = *E.m[i];
            cudaStream_t st = E.branch[i];
            if (cudaStreamWaitEvent(st, E.ev[n], 0) != cudaSuccess) rc = fail(PIC_ERR_CUDA, "ensemble: fork wait");
            if (rc == PIC_OK && S.d.sort_interval > 0) rc = capture_sort_if(S, E.d_steps + i, st, E.side[i]);
            if (rc == PIC_OK) rc = particle_pass(S, st, 1, 1, 1, 1, 1.0, 1);
            if (rc == PIC_OK) rc = field_solve(S, st, true);
            if (rc == PIC_OK) {
                k_ens_advance<<<1, 1, 0, st>>>(E.d_steps + i);
                if (cudaEventRecord(E.ev[i], st) != cudaSuccess || cudaStreamWaitEvent(root, E.ev[i], 0) != cudaSuccess)
                    rc = fail(PIC_ERR_CUDA, "ensemble: join of member %d", i);
            }
        }
        if (rc == PIC_OK) k_ens_loop<<<1, 1, 0, root>>>(E.d_ctl, h);
        cudaGraph_t body_out = nullptr;
        const cudaError_t eb = cudaStreamEndCapture(root, &body_out);
        if (rc == PIC_OK && eb != cudaSuccess) rc = fail(PIC_ERR_CUDA, "ensemble body: %s", cudaGetErrorString(eb));
    } while (false);
    const cudaError_t ec = cudaStreamEndCapture(E.cap, &g);
    if (rc != PIC_OK) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    if (ec != cudaSuccess) return fail(PIC_ERR_CUDA, "ensemble capture: %s", cudaGetErrorString(ec));
    const cudaError_t ei = cudaGraphInstantiate(&E.exec, g, 0);
    cudaGraphDestroy(g);
    if (ei != cudaSuccess) return fail(PIC_ERR_CUDA, "ensemble graph instantiate: %s", cudaGetErrorString(ei));
    return PIC_OK;
}

static void ens_free(EnsImpl& E) {
    if (E.exec) cudaGraphExecDestroy(E.exec);
    E.exec = nullptr;
    for (cudaStream_t s : E.branch) cudaStreamDestroy(s);
    for (cudaStream_t s : E.side) cudaStreamDestroy(s);
    for (cudaEvent_t e : E.ev) cudaEventDestroy(e);
    E.branch.clear();
    E.side.clear();
    E.ev.clear();
    if (E.cap) cudaStreamDestroy(E.cap);
    E.cap = nullptr;
    if (E.d_steps) cudaFree(E.d_steps);
    if (E.d_ctl) cudaFree(E.d_ctl);
    if (E.d_members) cudaFree(E.d_members);
    if (E.d_member_items) cudaFree(E.d_member_items);
    if (E.d_next) cudaFree(E.d_next);
    E.d_steps = nullptr;
    E.d_ctl = nullptr;
    E.d_members = nullptr;
    E.d_member_items = nullptr;
    E.d_next = nullptr;
}

}  // namespace pic

struct pic_sim {
    pic::SimImpl s;
};

struct pic_ens {
    pic::EnsImpl e;
};

using namespace pic;

extern "C" {

int pic_sim_create(const pic_sim_desc* desc, void* stream, pic_sim** out) {
    clear_error();
    if (!out) return fail(PIC_ERR_BAD_ARG, "pic_sim_create: out is NULL");
    pic_sim* sim = new pic_sim;
    const int st = sim_create(desc, as_stream(stream), sim->s);
    if (st != PIC_OK) {
        sim_free(sim->s);
        delete sim;
        return st;
    }
    *out = sim;
    return PIC_OK;
}

int pic_sim_destroy(pic_sim* sim) {
    clear_error();
    if (!sim) return PIC_OK;
    cudaDeviceSynchronize();
    sim_free(sim->s);
    delete sim;
    return PIC_OK;
}

int pic_sim_load_species(pic_sim* sim, int s, const float* x, const float* y, const float* vx, const float* vy,
                         const float* vz, int n, int from_host, void* stream) {
    clear_error();
    if (!sim || s < 0 || s >= sim->s.ns || n < 0 || n > sim->s.d.species[s].capacity)
        return fail(PIC_ERR_BAD_ARG, "pic_sim_load_species: bad arguments");
    SimImpl& S = sim->s;
    S.prepared = false;
    cudaStream_t st = as_stream(stream);
    PIC_CUDA(cudaStreamSynchronize(st));
    PIC_CUDA(cudaMemcpy(&S.h_state[s], S.d_state + s, sizeof(SpeciesState), cudaMemcpyDeviceToHost));
    const float* src[5] = {x, y, vx, vy, vz};
    const cudaMemcpyKind kind = from_host ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
    for (int c = 0; c < 5; ++c) {
        if (src[c]) PIC_CUDA(cudaMemcpyAsync(S.h_state[s].cur[c], src[c], sizeof(float) * size_t(n), kind, st));
        else PIC_CUDA(cudaMemsetAsync(S.h_state[s].cur[c], 0, sizeof(float) * size_t(n), st));
    }
    k_set_count<<<1, 1, 0, st>>>(S.d_state, s, n);
    k_untile_all<<<1, 1, 0, st>>>(S.d_state, S.ns, S.n_tiled);
    PIC_LAUNCH_CHECK();
    PIC_CUDA(cudaStreamSynchronize(st));
    return PIC_OK;
}

int pic_sim_init(pic_sim* sim, void* stream) {
    clear_error();
    if (!sim) return fail(PIC_ERR_BAD_ARG, "pic_sim_init: sim is NULL");
    SimImpl& S = sim->s;
    cudaStream_t st = as_stream(stream);
    S.prepared = false;
    if (S.d.sort_interval > 0) PIC_TRY(sort_all_graph(S, st));
    PIC_TRY(particle_pass(S, st, 0, 0, 0, 1, 1.0, 0));
    PIC_TRY(field_solve(S, st, false));
    PIC_TRY(particle_pass(S, st, 1, 0, 0, 0, -0.5, 0));
    S.kick_pending = false;
    PIC_CUDA(cudaStreamSynchronize(st));
    PIC_TRY(mg_info(S.mg, &S.last));
    return S.last.converged ? PIC_OK : PIC_ERR_NOT_CONVERGED;
}

int pic_sim_step(pic_sim* sim, int n_steps, void* stream) {
    clear_error();
    if (!sim || n_steps < 0) return fail(PIC_ERR_BAD_ARG, "pic_sim_step: bad arguments");
    SimImpl& S = sim->s;
    cudaStream_t st = as_stream(stream);
    for (int i = 0; i < n_steps; ++i) {
        const bool sort = S.d.sort_interval > 0 && S.steps % S.d.sort_interval == 0;
        if (S.d.use_graph && S.kick_pending && !S.profiling && mg_uses_graph(S.mg)) {
            if (!S.prepared) {
                if (sort) PIC_TRY(sort_all_graph(S, st));
                PIC_TRY(prepare_pass(S, st, 1, 1));
            }
            if (!S.g_step) {
                // both graphs of the step are captured at the first captured step
                PIC_TRY(capture_step(S, false, &S.g_step));
                if (S.d.sort_interval > 0) PIC_TRY(capture_step(S, true, &S.g_sort_step));
            }
            const bool sort_next = S.d.sort_interval > 0 && (S.steps + 1) % S.d.sort_interval == 0;
            PIC_CUDA(cudaGraphLaunch(sort_next ? S.g_sort_step : S.g_step, st));
            // items and the pass (with collisions: candidate bits and k_collide), the RHS and E
            S.launches +=
                2 + (S.have_mcc ? 2 : 0) + 2 + (sort_next ? 1 + (long long)S.ns * (5 + 3 * S.sorter.passes) : 0);
            S.solves += 1;
            S.prepared = true;
        } else {
            const int k = S.kick_pending ? 1 : 0;
            if (S.prepared) {
                // this step's sort, items and counter were done by the last captured step
                PIC_TRY(run_pass(S, st, k, k, 1, 1, 1.0));
                S.prepared = false;
            } else {
                if (sort) PIC_TRY(sort_all(S, st));
                PIC_TRY(particle_pass(S, st, k, k, 1, 1, 1.0, 1));
            }
            PIC_TRY(field_solve(S, st, false));
        }
        S.kick_pending = true;
        ++S.steps;
    }
    return PIC_OK;
}

int pic_sim_sync(pic_sim* sim, void* stream) {
    clear_error();
    if (!sim) return fail(PIC_ERR_BAD_ARG, "pic_sim_sync: sim is NULL");
    SimImpl& S = sim->s;
    if (!S.kick_pending) return PIC_OK;
    // a prepared pass has its counter advanced already
    PIC_TRY(particle_pass(S, as_stream(stream), 1, 1, 0, 0, 1.0, S.prepared ? 0 : 1));
    S.prepared = false;
    S.kick_pending = false;
    return PIC_OK;
}

int pic_sim_species_arrays(pic_sim* sim, int s, float** x, float** y, float** vx, float** vy, float** vz) {
    clear_error();
    if (!sim || s < 0 || s >= sim->s.ns) return fail(PIC_ERR_BAD_ARG, "pic_sim_species_arrays: bad arguments");
    SimImpl& S = sim->s;
    PIC_CUDA(cudaDeviceSynchronize());
    PIC_CUDA(cudaMemcpy(&S.h_state[s], S.d_state + s, sizeof(SpeciesState), cudaMemcpyDeviceToHost));
    float** dst[5] = {x, y, vx, vy, vz};
    for (int c = 0; c < 5; ++c)
        if (dst[c]) *dst[c] = S.h_state[s].cur[c];
    return PIC_OK;
}

int pic_sim_read_particles(pic_sim* sim, int s, float* h_out, long long capacity, int* count, void* stream) {
    clear_error();
    if (!sim || s < 0 || s >= sim->s.ns || !h_out || !count || capacity < 0)
        return fail(PIC_ERR_BAD_ARG, "pic_sim_read_particles: bad arguments");
    SimImpl& S = sim->s;
    cudaStream_t st = as_stream(stream);
    PIC_CUDA(cudaStreamSynchronize(st));
    PIC_CUDA(cudaMemcpy(&S.h_state[s], S.d_state + s, sizeof(SpeciesState), cudaMemcpyDeviceToHost));
    const SpeciesState& H = S.h_state[s];
    *count = H.count;
    if (5LL * H.count > capacity)
        return fail(PIC_ERR_OUT_OF_CAPACITY, "pic_sim_read_particles: %d slots need %lld floats, capacity %lld",
                    H.count, 5LL * H.count, capacity);
    if (H.count == 0) return PIC_OK;
    // one contiguous copy per array
    const size_t w = sizeof(float) * size_t(H.count);
    for (int c = 0; c < 5; ++c)
        PIC_CUDA(cudaMemcpyAsync(h_out + size_t(c) * H.count, H.cur[c], w, cudaMemcpyDeviceToHost, st));
    return PIC_OK;
}

int pic_sim_sort(pic_sim* sim, void* stream) {
    clear_error();
    if (!sim) return fail(PIC_ERR_BAD_ARG, "pic_sim_sort: sim is NULL");
    SimImpl& S = sim->s;
    if (!S.have_sorter) return fail(PIC_ERR_BAD_ARG, "pic_sim_sort: the simulation was created without a sort");
    cudaStream_t st = as_stream(stream);
    PIC_TRY(sort_all_graph(S, st));
    // a pass prepared by the last captured step holds work items of the
    // unsorted order: rebuild them for the same step (the counter stays)
    if (S.prepared) PIC_TRY(prepare_pass(S, st, 1, 0));
    return PIC_OK;
}

int pic_sim_fields(pic_sim* sim, double** phi, float** rho, float** Ex, float** Ey) {
    clear_error();
    if (!sim) return fail(PIC_ERR_BAD_ARG, "pic_sim_fields: sim is NULL");
    if (phi) *phi = sim->s.phi;
    if (rho) *rho = sim->s.rho_out;
    if (Ex) *Ex = sim->s.Ex;
    if (Ey) *Ey = sim->s.Ey;
    return PIC_OK;
}

int pic_sim_diagnostics(pic_sim* sim, pic_sim_diag* out, void* stream) {
    clear_error();
    if (!sim || !out) return fail(PIC_ERR_BAD_ARG, "pic_sim_diagnostics: bad arguments");
    SimImpl& S = sim->s;
    cudaStream_t st = as_stream(stream);
    if (!S.diag) PIC_TRY(dalloc(S, &S.diag, diagnostics_scratch_doubles()));
    PIC_CUDA(cudaStreamSynchronize(st));
    PIC_CUDA(cudaMemcpy(S.h_state, S.d_state, sizeof(SpeciesState) * S.ns, cudaMemcpyDeviceToHost));
    DiagSpecies sp[PIC_MAX_SPECIES];
    double mass[PIC_MAX_SPECIES], np2c[PIC_MAX_SPECIES];
    for (int s = 0; s < S.ns; ++s) {
        const SpeciesState& H = S.h_state[s];
        sp[s] = DiagSpecies{H.cur[2], H.cur[3], H.cur[4], H.cur[0], H.count};
        mass[s] = S.d.species[s].mass;
        np2c[s] = S.d.species[s].np2c;
    }
    return diagnostics(sp, mass, np2c, S.ns, S.phi, S.rho_out, S.Ex, S.Ey, S.nx, S.ny, S.d.dx, S.d.dy, S.d.eps0,
                       S.rowv, S.diag, out, st);
}

int pic_sim_read_counters(pic_sim* sim, pic_sim_counters* out, void* stream) {
    clear_error();
    if (!sim || !out) return fail(PIC_ERR_BAD_ARG, "pic_sim_read_counters: bad arguments");
    SimImpl& S = sim->s;
    PIC_CUDA(cudaStreamSynchronize(as_stream(stream)));
    int err = 0;
    PIC_CUDA(cudaMemcpy(&err, S.error, sizeof err, cudaMemcpyDeviceToHost));
    if (err) {
        PIC_CUDA(cudaMemset(S.error, 0, sizeof err));
        return fail(PIC_ERR_TIMEOUT, "particle pass: a wait on a bulk copy into shared memory gave up after %llu polls",
                    S.wait_limit);
    }
    unsigned long long c[kCtrCount];
    PIC_CUDA(cudaMemcpy(c, S.ctr, sizeof c, cudaMemcpyDeviceToHost));
    SpeciesState hs[PIC_MAX_SPECIES];
    PIC_CUDA(cudaMemcpy(hs, S.d_state, sizeof(SpeciesState) * S.ns, cudaMemcpyDeviceToHost));
    *out = pic_sim_counters{};
    for (int s = 0; s < S.ns; ++s) {
        out->absorbed[s] = c[kCtrAbsorbed + s];
        out->null_candidates[s] = c[kCtrCandidates + s];
        out->born[s] = c[kCtrBorn + s];
        for (int k = 0; k < PIC_MAX_PROCESSES; ++k) out->collisions[s][k] = c[kCtrCollisions + s * PIC_MAX_PROCESSES + k];
        out->count[s] = hs[s].count;
    }
    for (int s = 0; s < S.ns; ++s) out->electrode_absorbed[s] = c[kCtrElectrode + s];
    out->dropped_births = c[kCtrDropped];
    out->nu_overflow = c[kCtrOverflow];
    out->candidate_overflow = c[kCtrCandOverflow];
    PIC_TRY(mg_info(S.mg, &S.last));
    out->last_cycles = S.last.cycles;
    out->last_rel_res = S.last.rel_res;
    out->steps = S.steps;
    return PIC_OK;
}

int pic_sim_set_wait_limit(pic_sim* sim, long long polls) {
    clear_error();
    if (!sim) return fail(PIC_ERR_BAD_ARG, "pic_sim_set_wait_limit: sim is NULL");
    SimImpl& S = sim->s;
    PIC_CUDA(cudaDeviceSynchronize());
    S.wait_limit = polls < 0 ? kWaitLimit : (unsigned long long)polls;
    PIC_TRY(pic_mg_set_wait_limit(S.mg, polls));  // the persistent solve's grid barriers
    // the captured steps hold the old limits in their kernel arguments
    if (S.g_step) cudaGraphExecDestroy(S.g_step);
    if (S.g_sort_step) cudaGraphExecDestroy(S.g_sort_step);
    S.g_step = S.g_sort_step = nullptr;
    return PIC_OK;
}

int pic_sim_particle_buffer(pic_sim* sim, float* d_out, int capacity, double x_min, double x_max, double y_min,
                            double y_max, int* count, void* stream) {
    clear_error();
    if (!sim || !count || capacity < 0 || (capacity > 0 && !d_out) || !(x_max > x_min) || !(y_max > y_min))
        return fail(PIC_ERR_BAD_ARG, "pic_sim_particle_buffer: bad arguments");
    SimImpl& S = sim->s;
    cudaStream_t st = as_stream(stream);
    RenderArgs R{};
    R.state = S.d_state;
    R.ns = S.ns;
    int nb = 0;
    for (int s = 0; s < S.ns; ++s) {
        R.first_block[s] = nb;
        nb += div_up(S.d.species[s].capacity, kRenderBlock);
    }
    R.first_block[S.ns] = nb;
    if (!S.render_counts) {
        PIC_TRY(dalloc(S, &S.render_counts, size_t(nb) + 1));
        S.render_blocks = nb;
    }
    R.counts = S.render_counts;
    R.out = d_out;
    R.capacity = capacity;
    R.dx = S.d.dx;
    R.dy = S.d.dy;
    R.x0 = x_min;
    R.y0 = y_min;
    R.wx = x_max - x_min;
    R.wy = y_max - y_min;
    k_render_count<<<nb, kRenderBlock, 0, st>>>(R);
    k_render_scan<<<1, 1024, 0, st>>>(S.render_counts, nb);
    k_render_emit<<<nb, kRenderBlock, 0, st>>>(R);
    PIC_LAUNCH_CHECK();
    PIC_CUDA(cudaMemcpyAsync(count, S.render_counts + nb, sizeof(int), cudaMemcpyDeviceToHost, st));
    PIC_CUDA(cudaStreamSynchronize(st));
    S.launches += 3;
    if (*count > capacity)
        return fail(PIC_ERR_OUT_OF_CAPACITY, "pic_sim_particle_buffer: %d live particles, buffer holds %d", *count,
                    capacity);
    return PIC_OK;
}

int pic_sim_solver_mode(pic_sim* sim, int* mode) {
    clear_error();
    if (!sim || !mode) return fail(PIC_ERR_BAD_ARG, "pic_sim_solver_mode: bad arguments");
    return pic_mg_effective_launch_mode(sim->s.mg, mode);
}

long long pic_sim_kernel_launches(pic_sim* sim) {
    if (!sim) return 0;
    SimImpl& S = sim->s;
    cudaDeviceSynchronize();
    // each solve runs its residual kernel plus `body` kernels per V-cycle
    return S.launches + S.solves * mg_fixed_launches(S.mg) + mg_total_cycles(S.mg) * mg_body_launches(S.mg);
}

int pic_sim_set_profiling(pic_sim* sim, int enable) {
    clear_error();
    if (!sim) return fail(PIC_ERR_BAD_ARG, "pic_sim_set_profiling: sim is NULL");
    SimImpl& S = sim->s;
    if (enable) {
        PIC_CUDA(cudaDeviceSynchronize());
        for (auto& m : S.marks) {
            S.event_pool.push_back(m.second.first);
            S.event_pool.push_back(m.second.second);
        }
        S.marks.clear();
        S.prof_cycles = mg_total_cycles(S.mg);
    }
    S.profiling = enable != 0;
    return PIC_OK;
}

int pic_sim_read_profile(pic_sim* sim, pic_sim_profile* out) {
    clear_error();
    if (!sim || !out) return fail(PIC_ERR_BAD_ARG, "pic_sim_read_profile: bad arguments");
    SimImpl& S = sim->s;
    PIC_CUDA(cudaDeviceSynchronize());
    *out = pic_sim_profile{};
    for (auto& m : S.marks) {
        float ms = 0.f;
        PIC_CUDA(cudaEventElapsedTime(&ms, m.second.first, m.second.second));
        out->ms[m.first] += ms;
        out->count[m.first] += 1;
    }
    out->mg_cycles = mg_total_cycles(S.mg) - S.prof_cycles;
    return PIC_OK;
}


int pic_ens_create(pic_sim* const* sims, int n, pic_ens** out) {
    clear_error();
    if (!out || !sims || n < 1) return fail(PIC_ERR_BAD_ARG, "pic_ens_create: bad arguments");
    for (int i = 0; i < n; ++i) {
        if (!sims[i]) return fail(PIC_ERR_BAD_ARG, "pic_ens_create: member %d is NULL", i);
        if (!sims[i]->s.d.use_graph || !mg_uses_graph(sims[i]->s.mg))
            return fail(PIC_ERR_BAD_ARG, "pic_ens_create: member %d must use graphs (use_graph and a graph multigrid)", i);
        for (int j = 0; j < i; ++j)
            if (sims[j] == sims[i]) return fail(PIC_ERR_BAD_ARG, "pic_ens_create: member %d appears twice", i);
    }
    pic_ens* e = new pic_ens;
    EnsImpl& E = e->e;
    auto bail = [&](int code) {
        ens_free(E);
        delete e;
        return code;
    };
    for (int i = 0; i < n; ++i) E.m.push_back(&sims[i]->s);
    E.branch.resize(n);
    E.side.resize(n + 1);
    E.ev.resize(n + 1);
    for (int i = 0; i < n; ++i)
        if (cudaStreamCreateWithFlags(&E.branch[i], cudaStreamNonBlocking) != cudaSuccess)
            return bail(fail(PIC_ERR_CUDA, "pic_ens_create: stream creation failed"));
    for (int i = 0; i <= n; ++i)
        if (cudaStreamCreateWithFlags(&E.side[i], cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&E.ev[i], cudaEventDisableTiming) != cudaSuccess)
            return bail(fail(PIC_ERR_CUDA, "pic_ens_create: stream creation failed"));
    if (cudaStreamCreateWithFlags(&E.cap, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMalloc(&E.d_steps, sizeof(long long) * n) != cudaSuccess ||
        cudaMalloc(&E.d_ctl, sizeof(EnsControl)) != cudaSuccess)
        return bail(fail(PIC_ERR_CUDA, "pic_ens_create: out of device memory"));
    const int rc = ens_setup_fused(E);
    if (rc != PIC_OK) return bail(rc);
    // a pass per member by default: a member's pass then overlaps the other
    // members' field solves (3.30 against 3.89 ms per step of the 64-member
    // ensemble with one pass over all members, which ends before any solve)
    E.fused = false;
    *out = e;
    return PIC_OK;
}

int pic_ens_set_fused_pass(pic_ens* e, int fused) {
    clear_error();
    if (!e) return fail(PIC_ERR_BAD_ARG, "pic_ens_set_fused_pass: e is NULL");
    EnsImpl& E = e->e;
    const bool want = fused != 0 && E.d_members != nullptr;
    if (want != E.fused && E.exec) {
        // the step graph holds the other structure: capture it again at the next step
        PIC_CUDA(cudaDeviceSynchronize());
        cudaGraphExecDestroy(E.exec);
        E.exec = nullptr;
    }
    E.fused = want;
    return PIC_OK;
}

int pic_ens_fused_pass(pic_ens* e, int* fused) {
    clear_error();
    if (!e || !fused) return fail(PIC_ERR_BAD_ARG, "pic_ens_fused_pass: bad arguments");
    *fused = e->e.fused ? 1 : 0;
    return PIC_OK;
}

int pic_ens_destroy(pic_ens* e) {
    clear_error();
    if (!e) return PIC_OK;
    cudaDeviceSynchronize();
    ens_free(e->e);
    delete e;
    return PIC_OK;
}

int pic_ens_step(pic_ens* e, int n_steps, void* stream) {
    clear_error();
    if (!e || n_steps < 0) return fail(PIC_ERR_BAD_ARG, "pic_ens_step: bad arguments");
    EnsImpl& E = e->e;
    if (n_steps == 0) return PIC_OK;
    cudaStream_t st = as_stream(stream);
    // A member fresh from pic_sim_init takes its first step without the kick,
    // which the graph does not hold: if any member is fresh, every member
    // takes one step eagerly and the graph runs the other n - 1.
    bool fresh = false;
    for (SimImpl* S : E.m) fresh = fresh || !S->kick_pending;
    if (fresh) {
        for (SimImpl* S : E.m) {
            const int k = S->kick_pending ? 1 : 0;
            if (S->prepared) {
                PIC_TRY(run_pass(*S, st, k, k, 1, 1, 1.0));
            } else {
                if (S->d.sort_interval > 0 && S->steps % S->d.sort_interval == 0) PIC_TRY(sort_all(*S, st));
                PIC_TRY(particle_pass(*S, st, k, k, 1, 1, 1.0, 1));
            }
            S->prepared = false;
            PIC_TRY(field_solve(*S, st, false));
            S->kick_pending = true;
            ++S->steps;
        }
        if (--n_steps == 0) return PIC_OK;
    }
    if (!E.exec) PIC_TRY(ens_capture(E));
    const int n = int(E.m.size());
    std::vector<long long> steps(n);
    for (int i = 0; i < n; ++i) steps[i] = E.m[i]->steps;
    const EnsControl ctl{n_steps};
    PIC_CUDA(cudaMemcpyAsync(E.d_steps, steps.data(), sizeof(long long) * n, cudaMemcpyHostToDevice, st));
    PIC_CUDA(cudaMemcpyAsync(E.d_ctl, &ctl, sizeof ctl, cudaMemcpyHostToDevice, st));
    PIC_CUDA(cudaStreamSynchronize(st));  // the host copies above read stack memory
    PIC_CUDA(cudaGraphLaunch(E.exec, st));
    // the ensemble's body prepares each pass itself
    for (SimImpl* S : E.m) S->prepared = false;
    for (SimImpl* S : E.m) {
        long long sorts = 0;
        if (S->d.sort_interval > 0)
            for (long long k = S->steps; k < S->steps + n_steps; ++k) sorts += (k % S->d.sort_interval == 0);
        // the step counter, the particle pass (items and the pass, plus the
        // collisions), the RHS and E; a fused ensemble's one pass (and its item
        // numbering) is counted with the first member
        const long long pass = E.fused ? (S == E.m[0] ? 3 : 1) : 2;
        S->launches += n_steps * (1LL + pass + (S->have_mcc ? 2 : 0) + 2) +
                       sorts * (1 + (long long)S->ns * (5 + 3 * S->sorter.passes));
        if (S->d.sort_interval > 0) S->launches += n_steps;  // the sort condition
        S->solves += n_steps;
        S->steps += n_steps;
    }
    return PIC_OK;
}

}  // extern "C"
