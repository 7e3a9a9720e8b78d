// Conjugate-gradient Poisson solve: the 'cg' and 'gmres' branches of the
// reference's Solver (src/Solvers.py:245-258, cupyx.scipy.sparse.linalg cg
// and gmres on the 5-point Laplacian with Dirichlet rows).  The system is
// symmetric, so conjugate gradients reach the solution GMRES would.
//
// lap(phi) = f on the free nodes, phi fixed on the Dirichlet nodes (the grid
// edges and the mask): with x = phi - phi_0 (zero on Dirichlet nodes), L x = r_0.
// Flexible preconditioned CG (Polak-Ribiere beta, which tolerates a
// preconditioner that is not exactly symmetric), preconditioned by one
// multigrid V-cycle from zero when a pic_mg is given.  Everything in FP64;
// the dot products are block partials summed on the host in a fixed order.
#include <cmath>
#include <vector>

#include "common.cuh"

namespace pic {

int mg_launch_graph(pic_mg* mg, double* phi, const double* f, double tol, int max_cycles, int min_cycles,
                    cudaStream_t st);
bool mg_is_rz(pic_mg* mg);

constexpr int kCgThreads = 256;

struct CgImpl {
    int nx = 0, ny = 0;
    long G = 0;
    double cx = 0, cy = 0;
    uint8_t* free_ = nullptr;  // 1 = unknown
    pic_mg* mg = nullptr;
    double *r = nullptr, *r_prev = nullptr, *z = nullptr, *p = nullptr, *q = nullptr, *x = nullptr;
    double* part = nullptr;  // [2][blocks]
    int blocks = 0;
    std::vector<void*> allocs;
};

// q = lap(v) on free nodes, 0 elsewhere (v is 0 on Dirichlet nodes or, for
// the first residual, holds their values).
__device__ __forceinline__ double lap_at(const double* __restrict__ v, long k, int nx, double cx, double cy) {
    const double c = v[k];
    return cx * ((v[k - 1] - c) + (v[k + 1] - c)) + cy * ((v[k - nx] - c) + (v[k + nx] - c));
}

// r = f - lap(phi) on free nodes, 0 elsewhere; x = 0.
__global__ void k_cg_init(const double* __restrict__ phi, const double* __restrict__ f,
                          const uint8_t* __restrict__ fr, int nx, long G, double cx, double cy, double* __restrict__ r,
                          double* __restrict__ x) {
    for (long k = blockIdx.x * long(blockDim.x) + threadIdx.x; k < G; k += long(gridDim.x) * blockDim.x) {
        r[k] = fr[k] ? f[k] - lap_at(phi, k, nx, cx, cy) : 0.0;
        x[k] = 0.0;
    }
}

// Block partials of a.b and c.d (c, d may be null) over the free nodes.
__global__ void __launch_bounds__(kCgThreads) k_cg_dot2(const double* __restrict__ a, const double* __restrict__ b,
                                                        const double* __restrict__ c, const double* __restrict__ d,
                                                        const uint8_t* __restrict__ fr, long G,
                                                        double* __restrict__ part) {
    __shared__ double ws[2][kCgThreads / 32];
    double s0 = 0.0, s1 = 0.0;
    for (long k = blockIdx.x * long(blockDim.x) + threadIdx.x; k < G; k += long(gridDim.x) * blockDim.x) {
        if (!fr[k]) continue;
        s0 += a[k] * b[k];
        if (c) s1 += c[k] * d[k];
    }
    s0 = warp_sum(s0);
    s1 = warp_sum(s1);
    if ((threadIdx.x & 31) == 0) {
        ws[0][threadIdx.x >> 5] = s0;
        ws[1][threadIdx.x >> 5] = s1;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double t0 = 0.0, t1 = 0.0;
        for (int w = 0; w < kCgThreads / 32; ++w) {
            t0 += ws[0][w];
            t1 += ws[1][w];
        }
        part[blockIdx.x] = t0;
        part[gridDim.x + blockIdx.x] = t1;
    }
}

// z = r on free nodes (no preconditioner), or z = 0 (before a V-cycle).
__global__ void k_cg_copy(double* __restrict__ z, const double* __restrict__ r, const uint8_t* __restrict__ fr, long G,
                          int zero) {
    for (long k = blockIdx.x * long(blockDim.x) + threadIdx.x; k < G; k += long(gridDim.x) * blockDim.x)
        z[k] = (zero || !fr[k]) ? 0.0 : r[k];
}

// p = z + beta p; q = lap(p) needs p complete, so it is a second kernel.
__global__ void k_cg_dir(double* __restrict__ p, const double* __restrict__ z, const uint8_t* __restrict__ fr, long G,
                         double beta) {
    for (long k = blockIdx.x * long(blockDim.x) + threadIdx.x; k < G; k += long(gridDim.x) * blockDim.x)
        p[k] = fr[k] ? z[k] + beta * p[k] : 0.0;
}

__global__ void k_cg_apply(const double* __restrict__ p, const uint8_t* __restrict__ fr, int nx, long G, double cx,
                           double cy, double* __restrict__ q) {
    for (long k = blockIdx.x * long(blockDim.x) + threadIdx.x; k < G; k += long(gridDim.x) * blockDim.x)
        q[k] = fr[k] ? lap_at(p, k, nx, cx, cy) : 0.0;
}

// x += alpha p; r_prev = r; r -= alpha q.
__global__ void k_cg_update(double* __restrict__ x, double* __restrict__ r, double* __restrict__ r_prev,
                            const double* __restrict__ p, const double* __restrict__ q, long G, double alpha) {
    for (long k = blockIdx.x * long(blockDim.x) + threadIdx.x; k < G; k += long(gridDim.x) * blockDim.x) {
        x[k] += alpha * p[k];
        r_prev[k] = r[k];
        r[k] -= alpha * q[k];
    }
}

__global__ void k_cg_finish(double* __restrict__ phi, const double* __restrict__ x, const uint8_t* __restrict__ fr,
                            long G) {
    for (long k = blockIdx.x * long(blockDim.x) + threadIdx.x; k < G; k += long(gridDim.x) * blockDim.x)
        if (fr[k]) phi[k] += x[k];
}

static int dots(CgImpl& C, const double* a, const double* b, const double* c, const double* d, double* s0, double* s1,
                cudaStream_t st) {
    k_cg_dot2<<<C.blocks, kCgThreads, 0, st>>>(a, b, c, d, C.free_, C.G, C.part);
    PIC_LAUNCH_CHECK();
    std::vector<double> h(size_t(2) * C.blocks);
    PIC_CUDA(cudaMemcpyAsync(h.data(), C.part, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, st));
    PIC_CUDA(cudaStreamSynchronize(st));
    double t0 = 0.0, t1 = 0.0;
    for (int b = 0; b < C.blocks; ++b) {
        t0 += h[b];
        t1 += h[C.blocks + b];
    }
    *s0 = t0;
    if (s1) *s1 = t1;
    return PIC_OK;
}

int grid_blocks(long n, int threads);

}  // namespace pic

struct pic_cg {
    pic::CgImpl c;
};

using namespace pic;

extern "C" {

int pic_cg_create(int nx, int ny, double dx, double dy, const uint8_t* h_dirichlet, pic_mg* precond, pic_cg** out) {
    clear_error();
    if (!out || !h_dirichlet || nx < 3 || ny < 3 || !(dx > 0) || !(dy > 0))
        return fail(PIC_ERR_BAD_ARG, "pic_cg_create: bad arguments");
    if (precond && mg_is_rz(precond))
        return fail(PIC_ERR_BAD_ARG, "pic_cg_create: the conjugate-gradient solve is Cartesian");
    pic_cg* h = new pic_cg;
    CgImpl& C = h->c;
    C.nx = nx;
    C.ny = ny;
    C.G = long(nx) * ny;
    C.cx = 1.0 / (dx * dx);
    C.cy = 1.0 / (dy * dy);
    C.mg = precond;
    C.blocks = 2 * num_sms();
    std::vector<uint8_t> fr(size_t(C.G));
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            const size_t k = size_t(j) * nx + i;
            fr[k] = (i > 0 && j > 0 && i < nx - 1 && j < ny - 1 && !h_dirichlet[k]) ? 1 : 0;
        }
    auto alloc = [&](void** p, size_t bytes) {
        if (cudaMalloc(p, bytes) != cudaSuccess) return false;
        C.allocs.push_back(*p);
        return cudaMemset(*p, 0, bytes) == cudaSuccess;
    };
    const size_t vb = sizeof(double) * size_t(C.G);
    bool ok = alloc(reinterpret_cast<void**>(&C.free_), size_t(C.G)) &&
              cudaMemcpy(C.free_, fr.data(), size_t(C.G), cudaMemcpyHostToDevice) == cudaSuccess;
    for (double** v : {&C.r, &C.r_prev, &C.z, &C.p, &C.q, &C.x})
        ok = ok && alloc(reinterpret_cast<void**>(v), vb);
    ok = ok && alloc(reinterpret_cast<void**>(&C.part), sizeof(double) * 2 * size_t(C.blocks));
    if (!ok) {
        for (void* a : C.allocs) cudaFree(a);
        delete h;
        return fail(PIC_ERR_CUDA, "pic_cg_create: out of device memory");
    }
    *out = h;
    return PIC_OK;
}

int pic_cg_destroy(pic_cg* h) {
    clear_error();
    if (!h) return PIC_OK;
    cudaDeviceSynchronize();
    for (void* a : h->c.allocs) cudaFree(a);
    delete h;
    return PIC_OK;
}

int pic_cg_solve(pic_cg* h, double* d_phi, const double* d_f, double tol, int max_iter, pic_mg_info* info,
                 void* stream) {
    clear_error();
    if (!h || !d_phi || !d_f || !(tol > 0) || max_iter < 1) return fail(PIC_ERR_BAD_ARG, "pic_cg_solve: bad arguments");
    CgImpl& C = h->c;
    cudaStream_t st = as_stream(stream);
    const int gb = grid_blocks(C.G, kCgThreads);
    k_cg_init<<<gb, kCgThreads, 0, st>>>(d_phi, d_f, C.free_, C.nx, C.G, C.cx, C.cy, C.r, C.x);
    PIC_LAUNCH_CHECK();
    double f2 = 0.0, r2 = 0.0;
    PIC_TRY(dots(C, d_f, d_f, C.r, C.r, &f2, &r2, st));
    const double ref = f2 > 0.0 ? f2 : 1.0;
    double rz_prev = 0.0;
    int it = 0;
    while (r2 >= tol * tol * ref && it < max_iter) {
        // z = M r: one V-cycle from zero, or z = r
        if (C.mg) {
            k_cg_copy<<<gb, kCgThreads, 0, st>>>(C.z, C.r, C.free_, C.G, 1);
            PIC_LAUNCH_CHECK();
            PIC_TRY(mg_launch_graph(C.mg, C.z, C.r, 1e-300, 1, 0, st));
        } else {
            k_cg_copy<<<gb, kCgThreads, 0, st>>>(C.z, C.r, C.free_, C.G, 0);
            PIC_LAUNCH_CHECK();
        }
        double rz = 0.0, rpz = 0.0;
        PIC_TRY(dots(C, C.r, C.z, it > 0 ? C.r_prev : nullptr, C.z, &rz, &rpz, st));
        // Polak-Ribiere: beta = z.(r - r_prev) / (z_prev . r_prev)
        const double beta = it > 0 && rz_prev != 0.0 ? (rz - rpz) / rz_prev : 0.0;
        k_cg_dir<<<gb, kCgThreads, 0, st>>>(C.p, C.z, C.free_, C.G, beta);
        k_cg_apply<<<gb, kCgThreads, 0, st>>>(C.p, C.free_, C.nx, C.G, C.cx, C.cy, C.q);
        PIC_LAUNCH_CHECK();
        double pq = 0.0;
        PIC_TRY(dots(C, C.p, C.q, nullptr, nullptr, &pq, nullptr, st));
        if (pq == 0.0 || !std::isfinite(pq)) break;
        const double alpha = rz / pq;
        k_cg_update<<<gb, kCgThreads, 0, st>>>(C.x, C.r, C.r_prev, C.p, C.q, C.G, alpha);
        PIC_LAUNCH_CHECK();
        rz_prev = rz;
        ++it;
        PIC_TRY(dots(C, C.r, C.r, nullptr, nullptr, &r2, nullptr, st));
    }
    k_cg_finish<<<gb, kCgThreads, 0, st>>>(d_phi, C.x, C.free_, C.G);
    PIC_LAUNCH_CHECK();
    PIC_CUDA(cudaStreamSynchronize(st));
    pic_mg_info loc{};
    loc.cycles = it;
    loc.rhs_norm = std::sqrt(f2);
    loc.rel_res = std::sqrt(r2 / ref);
    loc.converged = r2 < tol * tol * ref ? 1 : 0;
    if (info) *info = loc;
    if (!loc.converged)
        return fail(PIC_ERR_NOT_CONVERGED, "pic_cg_solve: relative residual %.3e after %d iterations (tol %.1e)",
                    loc.rel_res, it, tol);
    return PIC_OK;
}

}  // extern "C"
