// Host side of the null-collision MCC tables and the standalone MCC operator
// behind the drop-in MCC.null_collision_method (src/MCC.py:308-415).
#include <cmath>
#include <vector>

#include "mcc_host.cuh"

namespace pic {

int grid_blocks(long n, int threads);

int mcc_build(const pic_mcc_desc* d, int nspecies, const double* mass, double dt, MccHost* H) {
    constexpr double kQe = 1.6e-19;  // src/Consts.py:1
    constexpr double kKb = 1.380649e-23;
    if (!d || nspecies < 1 || nspecies > PIC_MAX_SPECIES || !mass || !(dt > 0))
        return fail(PIC_ERR_BAD_ARG, "mcc: bad arguments");
    if (d->ne < 2 || !d->h_energy || !(d->gas_density >= 0) || !(d->gas_mass > 0) || !(d->gas_temperature >= 0))
        return fail(PIC_ERR_BAD_ARG, "mcc: bad table or gas description");
    const int ne = d->ne;
    std::vector<float> energy(ne);
    for (int j = 0; j < ne; ++j) {
        energy[j] = float(d->h_energy[j]);
        if (!(energy[j] > 0) || (j && !(energy[j] > energy[j - 1])))
            return fail(PIC_ERR_BAD_ARG, "mcc: energies must be positive and increasing");
    }
    MccDev& M = H->dev;
    M = MccDev{};
    M.ne = ne;
    M.e_lo = energy[0];
    M.e_hi = energy[ne - 1];
    M.log_e0 = logf(energy[0]);
    M.inv_log_ratio = float(double(ne - 1) / std::log(double(energy[ne - 1]) / double(energy[0])));
    M.gas_density = float(d->gas_density);
    float* de = nullptr;
    PIC_CUDA(cudaMalloc(&de, sizeof(float) * ne));
    H->allocs.push_back(de);
    PIC_CUDA(cudaMemcpy(de, energy.data(), sizeof(float) * ne, cudaMemcpyHostToDevice));
    M.energy = de;
    for (int s = 0; s < nspecies; ++s) {
        const pic_mcc_species_desc& S = d->species[s];
        MccSpeciesDev& D = M.sp[s];
        D.nproc = S.nproc;
        H->nu_max[s] = 0.0;
        H->p_null[s] = 0.0;
        if (S.nproc <= 0) continue;
        if (S.nproc > PIC_MAX_PROCESSES) return fail(PIC_ERR_BAD_ARG, "mcc: species %d has too many processes", s);
        std::vector<float> sig(size_t(S.nproc) * ne);
        for (int k = 0; k < S.nproc; ++k) {
            if (!S.h_sigma[k]) return fail(PIC_ERR_BAD_ARG, "mcc: missing table %d of species %d", k, s);
            if (S.type[k] < PIC_ELASTIC || S.type[k] > PIC_CHARGE_EXCHANGE)
                return fail(PIC_ERR_BAD_ARG, "mcc: unknown process type %d", S.type[k]);
            D.type[k] = S.type[k];
            D.thr[k] = float(S.threshold[k]);
            for (int j = 0; j < ne; ++j) sig[size_t(k) * ne + j] = float(S.h_sigma[k][j]);
            if (S.type[k] == PIC_IONIZATION &&
                (S.born_electron_species < 0 || S.born_electron_species >= nspecies || S.born_ion_species < 0 ||
                 S.born_ion_species >= nspecies))
                return fail(PIC_ERR_BAD_ARG, "mcc: ionisation products of species %d out of range", s);
        }
        float* ds = nullptr;
        PIC_CUDA(cudaMalloc(&ds, sizeof(float) * sig.size()));
        H->allocs.push_back(ds);
        PIC_CUDA(cudaMemcpy(ds, sig.data(), sizeof(float) * sig.size(), cudaMemcpyHostToDevice));
        D.sigma = ds;
        D.half_m_over_q = float(0.5 * mass[s] / kQe);
        D.mass_ratio2 = float(2.0 * mass[s] / d->gas_mass);
        D.gas_vth = float(std::sqrt(kKb * d->gas_temperature / d->gas_mass));
        D.born_e = S.born_electron_species;
        D.born_i = S.born_ion_species;
        // nu' bounds n_g sigma_T(E) v(E) on every table interval (sigma is
        // linear in E there and v grows with E), from the float tables the
        // device interpolates.
        double numax = 0.0;
        for (int j = 0; j + 1 < ne; ++j) {
            double s0 = 0.0, s1 = 0.0;
            for (int k = 0; k < S.nproc; ++k) {
                s0 += sig[size_t(k) * ne + j];
                s1 += sig[size_t(k) * ne + j + 1];
            }
            const double v1 = std::sqrt(double(energy[j + 1]) / double(D.half_m_over_q));
            numax = std::max(numax, std::max(s0, s1) * v1);
        }
        numax *= double(d->gas_density) * (1.0 + 1e-5);
        D.nu_max = float(numax);
        if (D.nu_max > 0) {
            D.inv_log1m_p = -1.0 / (double(D.nu_max) * dt);
            H->p_null[s] = -std::expm1(-double(D.nu_max) * dt);
        } else {
            D.nproc = 0;
        }
        H->nu_max[s] = double(D.nu_max);
    }
    return PIC_OK;
}

void mcc_free(MccHost* H) {
    for (void* p : H->allocs) cudaFree(p);
    H->allocs.clear();
}

// One block per 4096 slots (16 candidate segments, one lane each).
constexpr int kMccBlockSlots = 4096;

__global__ void __launch_bounds__(256) k_mcc_apply(MccDev M, int s, const float* __restrict__ x,
                                                   const float* __restrict__ y, float* __restrict__ vx,
                                                   float* __restrict__ vy, float* __restrict__ vz, int n,
                                                   uint32_t step, uint2 key, BirthDev B,
                                                   unsigned long long* __restrict__ ctr) {
    __shared__ unsigned bits[kMccBlockSlots / 32];
    const MccSpeciesDev& S = M.sp[s];
    const int b = blockIdx.x * kMccBlockSlots, e = min(n, b + kMccBlockSlots);
    for (int q = threadIdx.x; q < kMccBlockSlots / 32; q += blockDim.x) bits[q] = 0;
    __syncthreads();
    constexpr int segs = kMccBlockSlots / int(kMccSegment);
    if (threadIdx.x < segs) {
        const long g = long(b) / kMccSegment + threadIdx.x;
        if (g * long(kMccSegment) < e) mcc_mark_segment(S, uint32_t(s), g, n, b, e, step, key, bits);
    }
    __syncthreads();
    for (int l = threadIdx.x; l < e - b; l += blockDim.x) {
        if (!(bits[l >> 5] & (1u << (l & 31)))) continue;
        const int p = b + l;
        const float px = x[p], py = y[p];
        if (!is_live(px)) continue;
        atomicAdd(ctr + kCtrCandidates + s, 1ull);
        float a = vx[p], c = vy[p], d = vz[p];
        const MccOutcome o = mcc_collide(M, S, uint32_t(s), uint32_t(p), step, key, a, c, d);
        if (o.overflow) atomicAdd(ctr + kCtrOverflow, 1ull);
        if (o.proc < 0) continue;
        atomicAdd(ctr + kCtrCollisions + s * PIC_MAX_PROCESSES + o.proc, 1ull);
        vx[p] = a;
        vy[p] = c;
        vz[p] = d;
        if (o.born) {
            const bool ok_e = birth_push(B, S.born_e, px, py, o.be[0], o.be[1], o.be[2]);
            const bool ok_i = birth_push(B, S.born_i, px, py, o.bi[0], o.bi[1], o.bi[2]);
            if (!ok_e || !ok_i) atomicAdd(ctr + kCtrDropped, 1ull);
        }
    }
}

}  // namespace pic

struct pic_mcc {
    pic::MccHost h;
    int nspecies = 0;
};

using namespace pic;

extern "C" {

int pic_mcc_create(const pic_mcc_desc* desc, int nspecies, const double* species_mass, double dt, pic_mcc** out) {
    clear_error();
    if (!out) return fail(PIC_ERR_BAD_ARG, "pic_mcc_create: out is NULL");
    pic_mcc* m = new pic_mcc;
    m->nspecies = nspecies;
    const int st = mcc_build(desc, nspecies, species_mass, dt, &m->h);
    if (st != PIC_OK) {
        mcc_free(&m->h);
        delete m;
        return st;
    }
    *out = m;
    return PIC_OK;
}

int pic_mcc_destroy(pic_mcc* m) {
    clear_error();
    if (!m) return PIC_OK;
    mcc_free(&m->h);
    delete m;
    return PIC_OK;
}

int pic_mcc_query(pic_mcc* m, int s, double* nu_max, double* p_null, double* inv_log1m_p) {
    clear_error();
    if (!m || s < 0 || s >= m->nspecies) return fail(PIC_ERR_BAD_ARG, "pic_mcc_query: bad arguments");
    if (nu_max) *nu_max = double(m->h.dev.sp[s].nu_max);
    if (p_null) *p_null = m->h.p_null[s];
    if (inv_log1m_p) *inv_log1m_p = m->h.dev.sp[s].inv_log1m_p;
    return PIC_OK;
}

int pic_mcc_apply(pic_mcc* m, int s, const float* d_x, const float* d_y, float* d_vx, float* d_vy, float* d_vz, int n,
                  unsigned long long seed, unsigned int step, const pic_birth_buffer* births,
                  unsigned long long* d_counters, void* stream) {
    clear_error();
    if (!m || s < 0 || s >= m->nspecies || n < 0 || !d_counters || !births || !births->count ||
        (n > 0 && (!d_x || !d_y || !d_vx || !d_vy || !d_vz)))
        return fail(PIC_ERR_BAD_ARG, "pic_mcc_apply: bad arguments");
    if (n == 0 || m->h.dev.sp[s].nproc == 0) return PIC_OK;
    BirthDev B{births->x, births->y, births->vx, births->vy, births->vz, births->species, births->count,
               births->capacity};
    const uint2 key = make_uint2(uint32_t(seed), uint32_t(seed >> 32));
    const int blocks = div_up(n, kMccBlockSlots);
    k_mcc_apply<<<blocks, 256, 0, as_stream(stream)>>>(m->h.dev, s, d_x, d_y, d_vx, d_vy, d_vz, n, step, key, B,
                                                       d_counters);
    PIC_LAUNCH_CHECK();
    return PIC_OK;
}

}  // extern "C"
