// Null-collision Monte-Carlo collisions, device side (replaces
// MCC.null_collision_method, src/MCC.py:308-415, which computes a collision
// mask and returns before scattering anything).
//
// Method (Vahedi & Surendra, Comput. Phys. Commun. 87 (1995) 179):
//   nu' = n_g * max_E sigma_T(E) v(E) over the table, P_null = 1 - exp(-nu' dt).
//   Candidates: independent Bernoulli(P_null) trials per particle, drawn as
//   geometric gaps (floor(log u / log(1 - P_null))) over fixed 256-slot
//   segments of the slot index, so that only ~P_null*N particles touch the
//   random stream and every segment is drawn by its own lane.
//   A candidate picks process k when u*nu' falls in the k-th slice of the
//   cumulative n_g*sigma_k(E)*v; past the last slice it is a null collision.
// Random numbers: Philox4x32-10 keyed by the run seed; counters
//   candidates: (segment, step, species, draw/4)
//   collision:  (slot, step, species | 0x100, call)
// All FP32 arithmetic uses explicit rounding intrinsics in the order of the
// CPU oracle (oracle/pic_oracle.c), so the process choice is reproducible.
#pragma once

#include "common.cuh"

namespace pic {

constexpr uint32_t kMccSegment = 256;  // slots per candidate segment (one lane draws one segment)

struct MccSpeciesDev {
    int nproc;
    int type[PIC_MAX_PROCESSES];
    float thr[PIC_MAX_PROCESSES];
    const float* sigma;   // nproc rows of ne values (m^2)
    float nu_max;         // nu' (1/s)
    double inv_log1m_p;   // 1/log(1 - P_null) = -1/(nu' dt)
    float half_m_over_q;  // eV per (m/s)^2
    float mass_ratio2;    // 2 m / M_gas
    float gas_vth;        // sqrt(k T / M_gas)
    int born_e, born_i;   // ionisation products (species indices)
};

struct MccDev {
    int ne;
    const float* energy;  // eV, log-spaced
    float e_lo, e_hi;     // energy[0] and energy[ne - 1]
    float log_e0, inv_log_ratio;
    float gas_density;
    MccSpeciesDev sp[PIC_MAX_SPECIES];
};

// Births from ionisation, appended through an atomic counter.
struct BirthDev {
    float *x, *y, *vx, *vy, *vz;
    int* species;
    int* count;
    int capacity;
};

// Where energy e falls on the shared log-spaced energy grid: below the first
// point (lo), past the last (hi), or in bin j at fraction t.  Every process's
// cross section is read at the same place, so a candidate locates it once.
struct MccBin {
    int j;
    float t;
    bool lo, hi;
};

__device__ __forceinline__ MccBin mcc_bin(const MccDev& M, float e) {
    const float* __restrict__ E = M.energy;
    const int ne = M.ne;
    MccBin b;
    b.j = 0;
    b.t = 0.0f;
    b.lo = e <= M.e_lo;
    b.hi = !b.lo && e >= M.e_hi;
    if (b.lo || b.hi) return b;
    // the bin from the log-spaced grid, corrected (rarely) by the grid
    // itself; both ends of the bin are loaded together
    int j = int(__fmul_rn(__fsub_rn(logf(e), M.log_e0), M.inv_log_ratio));
    j = max(0, min(j, ne - 2));
    float a = E[j], c = E[j + 1];
    while (j > 0 && e < a) {
        --j;
        c = a;
        a = E[j];
    }
    while (j < ne - 2 && e >= c) {
        ++j;
        a = c;
        c = E[j + 1];
    }
    b.j = j;
    b.t = __fdiv_rn(__fsub_rn(e, a), __fsub_rn(c, a));
    return b;
}

// Cross section S (one row of the table) at the located energy: clamped to the
// end values outside the grid, linear inside.
__device__ __forceinline__ float mcc_sigma(const MccDev& M, const float* __restrict__ S, const MccBin& b) {
    if (b.lo) return S[0];
    if (b.hi) return S[M.ne - 1];
    return __fmaf_rn(b.t, __fsub_rn(S[b.j + 1], S[b.j]), S[b.j]);
}

__device__ __forceinline__ void mcc_isotropic(float u_cos, float u_phi, float& dx, float& dy, float& dz) {
    const float c = __fsub_rn(1.0f, __fmul_rn(2.0f, u_cos));
    const float s = __fsqrt_rn(fmaxf(0.0f, __fsub_rn(1.0f, __fmul_rn(c, c))));
    const float ph = __fmul_rn(6.2831853071795864f, u_phi);
    dx = __fmul_rn(s, cosf(ph));
    dy = __fmul_rn(s, sinf(ph));
    dz = c;
}

__device__ __forceinline__ void mcc_maxwellian(uint4 r, float vth, float& vx, float& vy, float& vz) {
    const float a = __fsqrt_rn(__fmul_rn(-2.0f, logf(u01_float(r.x))));
    const float b = __fmul_rn(6.2831853071795864f, u01_float(r.y));
    const float c = __fsqrt_rn(__fmul_rn(-2.0f, logf(u01_float(r.z))));
    const float d = __fmul_rn(6.2831853071795864f, u01_float(r.w));
    vx = __fmul_rn(__fmul_rn(vth, a), cosf(b));
    vy = __fmul_rn(__fmul_rn(vth, a), sinf(b));
    vz = __fmul_rn(__fmul_rn(vth, c), cosf(d));
}

// Marks the candidates of segment g that fall in [b, e) in the bitmask bits
// (bit i-b); n = slots of the species (candidates at or past n are ignored).
__device__ __forceinline__ void mcc_mark_segment(const MccSpeciesDev& S, uint32_t species, long g, int n, int b, int e,
                                                 uint32_t step, uint2 key, unsigned* bits) {
    long pos = -1;
    uint32_t draw = 0;
    uint4 out = make_uint4(0, 0, 0, 0);
    for (uint32_t guard = 0; guard <= kMccSegment; ++guard) {
        if ((draw & 3u) == 0) out = philox4x32_10(make_uint4(uint32_t(g), step, species, draw >> 2), key);
        const uint32_t w = (draw & 3u) == 0 ? out.x : (draw & 3u) == 1 ? out.y : (draw & 3u) == 2 ? out.z : out.w;
        ++draw;
        const double f = floor(log(u01_double(w)) * S.inv_log1m_p);
        if (f > double(kMccSegment)) break;
        pos += 1 + long(f);
        if (pos >= long(kMccSegment)) break;
        const long i = g * long(kMccSegment) + pos;
        if (i >= n) break;
        if (i >= b && i < e) atomicOr(bits + ((i - b) >> 5), 1u << ((i - b) & 31));
    }
}

// Result of one candidate collision.
struct MccOutcome {
    int proc;        // process index, or -1 for a null collision
    bool born;       // ionisation: an electron and an ion were created
    float be[3];     // new electron velocity
    float bi[3];     // new ion velocity
    bool overflow;   // n_g sigma_T v exceeded nu' (probability under-sampled)
};

__device__ __forceinline__ MccOutcome mcc_collide(const MccDev& M, const MccSpeciesDev& S, uint32_t species,
                                                  uint32_t idx, uint32_t step, uint2 key, float& vx, float& vy,
                                                  float& vz) {
    MccOutcome o;
    o.proc = -1;
    o.born = false;
    o.overflow = false;
    uint4 ctr = make_uint4(idx, step, species | 0x100u, 0u);
    const uint4 r0 = philox4x32_10(ctr, key);
    const float v2 = __fadd_rn(__fadd_rn(__fmul_rn(vx, vx), __fmul_rn(vy, vy)), __fmul_rn(vz, vz));
    const float speed = __fsqrt_rn(v2);
    const float e = __fmul_rn(S.half_m_over_q, v2);
    const float target = __fmul_rn(u01_float(r0.x), S.nu_max);
    const MccBin bin = mcc_bin(M, e);
    // every process's cross section at once (independent loads), then the
    // cumulative test in process order
    float sigs[PIC_MAX_PROCESSES];
#pragma unroll
    for (int k = 0; k < PIC_MAX_PROCESSES; ++k)
        sigs[k] = k < S.nproc ? mcc_sigma(M, S.sigma + long(k) * M.ne, bin) : 0.0f;
    float acc = 0.0f;
    int proc = -1;
#pragma unroll
    for (int k = 0; k < PIC_MAX_PROCESSES; ++k) {
        if (k >= S.nproc) break;
        const float sig = sigs[k];
        acc = __fadd_rn(acc, __fmul_rn(__fmul_rn(M.gas_density, sig), speed));
        if (target < acc) {
            proc = k;
            break;
        }
    }
    if (proc < 0) {
        o.overflow = acc > S.nu_max;
        return o;
    }
    const int type = S.type[proc];
    float e_left = e;
    if (type == PIC_EXCITATION || type == PIC_IONIZATION) {
        e_left = __fsub_rn(e, S.thr[proc]);
        if (!(e_left > 0.0f)) return o;
    }
    o.proc = proc;
    if (type == PIC_CHARGE_EXCHANGE) {
        ctr.w = 2u;
        mcc_maxwellian(philox4x32_10(ctr, key), S.gas_vth, vx, vy, vz);
        return o;
    }
    float dx, dy, dz;
    mcc_isotropic(u01_float(r0.y), u01_float(r0.z), dx, dy, dz);
    float new_speed;
    if (type == PIC_ELASTIC) {
        const float inv = speed > 0.0f ? __fdiv_rn(1.0f, speed) : 0.0f;
        const float cosx =
            __fmul_rn(__fadd_rn(__fadd_rn(__fmul_rn(vx, dx), __fmul_rn(vy, dy)), __fmul_rn(vz, dz)), inv);
        new_speed = __fmul_rn(speed, __fsqrt_rn(fmaxf(0.0f, __fsub_rn(1.0f, __fmul_rn(S.mass_ratio2,
                                                                                       __fsub_rn(1.0f, cosx))))));
    } else if (type == PIC_EXCITATION) {
        new_speed = __fsqrt_rn(__fdiv_rn(e_left, S.half_m_over_q));
    } else {
        const float frac = __fadd_rn(0.2f, __fmul_rn(0.6f, u01_float(r0.w)));
        new_speed = __fsqrt_rn(__fdiv_rn(__fmul_rn(frac, e_left), S.half_m_over_q));
        const float sec = __fsqrt_rn(__fdiv_rn(__fmul_rn(__fsub_rn(1.0f, frac), e_left), S.half_m_over_q));
        ctr.w = 1u;
        const uint4 r1 = philox4x32_10(ctr, key);
        float sx, sy, sz;
        mcc_isotropic(u01_float(r1.x), u01_float(r1.y), sx, sy, sz);
        o.be[0] = __fmul_rn(sec, sx);
        o.be[1] = __fmul_rn(sec, sy);
        o.be[2] = __fmul_rn(sec, sz);
        ctr.w = 2u;
        mcc_maxwellian(philox4x32_10(ctr, key), S.gas_vth, o.bi[0], o.bi[1], o.bi[2]);
        o.born = true;
    }
    vx = __fmul_rn(new_speed, dx);
    vy = __fmul_rn(new_speed, dy);
    vz = __fmul_rn(new_speed, dz);
    return o;
}

// Appends one particle (x, y in grid units) to the birth buffer.
__device__ __forceinline__ bool birth_push(const BirthDev& B, int species, float x, float y, float vx, float vy,
                                          float vz) {
    const int slot = atomicAdd(B.count, 1);
    if (slot >= B.capacity) return false;
    B.x[slot] = x;
    B.y[slot] = y;
    B.vx[slot] = vx;
    B.vy[slot] = vy;
    B.vz[slot] = vz;
    B.species[slot] = species;
    return true;
}

// Counter layout (uint64): collisions[s][k] at s*4+k, candidates[s] at 16+s,
// dropped births at 20, nu overflow at 21, absorbed[s] at 22+s, born[s] at 26+s,
// candidates that did not fit the fused step's candidate list at 30, particles
// collected by internal electrodes[s] at 31+s.
constexpr int kCtrCollisions = 0, kCtrCandidates = 16, kCtrDropped = 20, kCtrOverflow = 21, kCtrAbsorbed = 22,
              kCtrBorn = 26, kCtrCandOverflow = 30, kCtrElectrode = 31, kCtrCount = 35;

}  // namespace pic
