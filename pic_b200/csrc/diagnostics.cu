// Diagnostics of a simulation's device state (the reference computes them in
// src/simulation.py:116-345 with CuPy reductions and a float atomic kernel):
// kinetic energy and momentum per species, field energy, and Gauss's law
// (boundary flux of E against the enclosed charge, and the L2 norm of
// div E - rho/eps0).  FP64 accumulation; block partials are summed by one
// block in a fixed order, so the results do not depend on the schedule.
#include <cmath>

#include "common.cuh"

namespace pic {

int grid_blocks(long n, int threads);

constexpr int kDiagThreads = 256;
constexpr int kDiagBlocks = 296;
constexpr int kDiagParticleSums = 7;  // per species: live, vx^2+vy^2+vz^2, vx, vy, vz (scaled later), spare
constexpr int kDiagGridSums = 4;      // rho phi, boundary flux, charge, (div E - rho/eps0)^2

__device__ __forceinline__ double block_sum(double v, double* ws) {
    v = warp_sum(v);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) ws[w] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x == 0)
        for (int q = 0; q < int(blockDim.x >> 5); ++q) s += ws[q];
    return s;  // valid in thread 0
}

// partial[(s * kDiagParticleSums + k) * gridDim.x + block]
__global__ void __launch_bounds__(kDiagThreads) k_diag_particles(DiagSpecies sp, int s, double* __restrict__ partial) {
    __shared__ double ws[kDiagThreads / 32];
    double a[5] = {0, 0, 0, 0, 0};
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < sp.n; p += gridDim.x * blockDim.x) {
        if (!is_live(sp.x[p])) continue;
        const double vx = sp.vx[p], vy = sp.vy[p], vz = sp.vz ? double(sp.vz[p]) : 0.0;
        a[0] += 1.0;
        a[1] += vx * vx + vy * vy + vz * vz;
        a[2] += vx;
        a[3] += vy;
        a[4] += vz;
    }
    for (int k = 0; k < 5; ++k) {
        const double t = block_sum(a[k], ws);
        if (threadIdx.x == 0) partial[(s * kDiagParticleSums + k) * gridDim.x + blockIdx.x] = t;
    }
}

// Field energy, Gauss's law terms; partial[k * gridDim.x + block].  rowv
// (r-z geometry): per row V_j / (dx*dy), the node volume in units of dx*dy;
// null in Cartesian geometry (volume dx*dy per unit depth).
__global__ void __launch_bounds__(kDiagThreads) k_diag_grid(const double* __restrict__ phi, const float* __restrict__ rho,
                                                           const float* __restrict__ Ex, const float* __restrict__ Ey,
                                                           int nx, int ny, double dx, double dy, double inv_eps0,
                                                           const double* __restrict__ rowv,
                                                           double* __restrict__ partial) {
    __shared__ double ws[kDiagThreads / 32];
    double a[kDiagGridSums] = {0, 0, 0, 0};
    const long G = long(nx) * ny;
    const double two_pi = 6.283185307179586476925;
    for (long k = blockIdx.x * long(blockDim.x) + threadIdx.x; k < G; k += long(gridDim.x) * blockDim.x) {
        const int i = int(k % nx), j = int(k / nx);
        const double r = rho[k];
        const double w = rowv ? rowv[j] : 1.0;
        a[0] += r * phi[k] * w;
        a[2] += r * w;
        // outward flux through the domain boundary (node sums, as the reference);
        // r-z: the end disks (areas V_j / dx per node) and the outer cylinder
        if (i == nx - 1) a[1] += double(Ex[k]) * dy * w;
        if (i == 0) a[1] -= double(Ex[k]) * dy * w;
        if (j == ny - 1) a[1] += double(Ey[k]) * dx * (rowv ? two_pi * double(j) * dy : 1.0);
        if (j == 0 && !rowv) a[1] -= double(Ey[k]) * dx;
        // divergence of E with the stencil of the gradient (central inside, one-sided on the edges);
        // r-z: (1/r) d(r E_r)/dr, and 2 dE_r/dr on the axis
        double dex, dey;
        if (i > 0 && i < nx - 1) dex = (double(Ex[k + 1]) - double(Ex[k - 1])) / (2.0 * dx);
        else if (i == 0) dex = (double(Ex[k + 1]) - double(Ex[k])) / dx;
        else dex = (double(Ex[k]) - double(Ex[k - 1])) / dx;
        if (rowv) {
            if (j > 0 && j < ny - 1)
                dey = (double(j + 1) * double(Ey[k + nx]) - double(j - 1) * double(Ey[k - nx])) / (2.0 * double(j) * dy);
            else if (j == 0) dey = 2.0 * (double(Ey[k + nx]) - double(Ey[k])) / dy;
            else dey = (double(j) * double(Ey[k]) - double(j - 1) * double(Ey[k - nx])) / (double(j) * dy);
        } else if (j > 0 && j < ny - 1) dey = (double(Ey[k + nx]) - double(Ey[k - nx])) / (2.0 * dy);
        else if (j == 0) dey = (double(Ey[k + nx]) - double(Ey[k])) / dy;
        else dey = (double(Ey[k]) - double(Ey[k - nx])) / dy;
        const double e = dex + dey - r * inv_eps0;
        a[3] += e * e;
    }
    for (int q = 0; q < kDiagGridSums; ++q) {
        const double t = block_sum(a[q], ws);
        if (threadIdx.x == 0) partial[q * gridDim.x + blockIdx.x] = t;
    }
}

// out[c] = sum over blocks of partial[c * nb + b], one thread per column, in block order.
__global__ void k_diag_final(const double* __restrict__ partial, int ncols, int nb, double* __restrict__ out) {
    for (int c = threadIdx.x; c < ncols; c += blockDim.x) {
        double s = 0.0;
        for (int b = 0; b < nb; ++b) s += partial[long(c) * nb + b];
        out[c] = s;
    }
}

// The diagnostics of `ns` species and the fields; writes `out` (host).
int diagnostics(const DiagSpecies* sp, const double* mass, const double* np2c, int ns, const double* phi,
                const float* rho, const float* Ex, const float* Ey, int nx, int ny, double dx, double dy, double eps0,
                const double* rowv, double* scratch, pic_sim_diag* out, cudaStream_t st) {
    const int nb = kDiagBlocks;
    const int pcols = PIC_MAX_SPECIES * kDiagParticleSums;
    double* part = scratch;                        // [(pcols + kDiagGridSums) * nb]
    double* sums = scratch + size_t(pcols + kDiagGridSums) * nb;  // [pcols + kDiagGridSums]
    PIC_CUDA(cudaMemsetAsync(part, 0, sizeof(double) * size_t(pcols + kDiagGridSums) * nb, st));
    for (int s = 0; s < ns; ++s) k_diag_particles<<<nb, kDiagThreads, 0, st>>>(sp[s], s, part);
    k_diag_grid<<<nb, kDiagThreads, 0, st>>>(phi, rho, Ex, Ey, nx, ny, dx, dy, 1.0 / eps0, rowv,
                                             part + size_t(pcols) * nb);
    k_diag_final<<<1, 64, 0, st>>>(part, pcols + kDiagGridSums, nb, sums);
    PIC_LAUNCH_CHECK();
    double h[PIC_MAX_SPECIES * kDiagParticleSums + kDiagGridSums];
    PIC_CUDA(cudaMemcpyAsync(h, sums, sizeof h, cudaMemcpyDeviceToHost, st));
    PIC_CUDA(cudaStreamSynchronize(st));
    *out = pic_sim_diag{};
    for (int s = 0; s < ns; ++s) {
        const double* a = h + s * kDiagParticleSums;
        out->live[s] = (long long)(a[0] + 0.5);
        out->kinetic[s] = 0.5 * mass[s] * np2c[s] * a[1];
        for (int c = 0; c < 3; ++c) out->momentum[s][c] = mass[s] * np2c[s] * a[2 + c];
    }
    const double* g = h + pcols;
    out->field_energy = 0.5 * g[0] * dx * dy;
    out->gauss_flux = g[1];
    out->gauss_charge = g[2] * dx * dy / eps0;
    out->div_error_l2 = std::sqrt(g[3]);
    return PIC_OK;
}

size_t diagnostics_scratch_doubles() {
    return size_t(PIC_MAX_SPECIES * kDiagParticleSums + kDiagGridSums) * (kDiagBlocks + 1);
}

}  // namespace pic
