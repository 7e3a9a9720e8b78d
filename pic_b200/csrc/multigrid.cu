// Geometric multigrid Poisson solver (replaces src/multigrid.py:277-455).
//
// Outer loop: FP64 iterative refinement on the fine grid
//     r = f - A phi   (FP64, 5-point operator, free nodes only)
//     solve A e = r approximately with one V-cycle from e = 0
//     phi += e        (FP64)
// until ||r|| / ||f|| < tol.  The V-cycle runs in FP32 (PIC_MG_MIXED) or FP64
// (PIC_MG_FP64); it is a correction scheme with red-black Gauss-Seidel
// smoothing, full-weighting restriction, bilinear prolongation and a dense
// FP64 direct solve on the coarsest level.  Dirichlet nodes (mask = 1, and
// the grid edges) carry a zero correction on every level; a coarse node is
// Dirichlet when its injected fine node is.
#include <cmath>
#include <vector>

#include "common.cuh"

namespace pic {

int grid_blocks(long n, int threads);

template <class T>
struct MgLevel {
    int nx, ny;
    T cx, cy;        // 1/dx^2, 1/dy^2 at this level
    uint8_t* mask;   // 1 = Dirichlet
    T* e;            // correction
    T* g;            // right-hand side of the correction equation
};

// ---- kernels ---------------------------------------------------------------------

template <class T>
__global__ void k_smooth(T* __restrict__ e, const T* __restrict__ g, const uint8_t* __restrict__ mask, int nx, int ny,
                         T cx, T cy, T omega, int color, const int* __restrict__ skip) {
    if (skip && *skip) return;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int i = 2 * (blockIdx.x * blockDim.x + threadIdx.x) + ((color + j) & 1);
    if (j >= ny - 1 || i < 1 || i >= nx - 1) return;
    const long k = long(j) * nx + i;
    if (mask[k]) return;
    const T inv_diag = T(1) / (T(2) * (cx + cy));
    const T s = cx * (e[k - 1] + e[k + 1]) + cy * (e[k - nx] + e[k + nx]);
    const T upd = (s - g[k]) * inv_diag;
    const T old = e[k];
    e[k] = old + omega * (upd - old);
}

template <class T>
__device__ __forceinline__ T fine_residual(const T* __restrict__ e, const T* __restrict__ g,
                                           const uint8_t* __restrict__ mask, long k, int nx, T cx, T cy) {
    if (mask[k]) return T(0);
    const T c = e[k];
    const T lap = cx * (e[k - 1] + e[k + 1] - T(2) * c) + cy * (e[k - nx] + e[k + nx] - T(2) * c);
    return g[k] - lap;
}

template <class T>
__global__ void k_resid_restrict(const T* __restrict__ e, const T* __restrict__ g, const uint8_t* __restrict__ mask,
                                 int nxf, T cx, T cy, T* __restrict__ gc, T* __restrict__ ec,
                                 const uint8_t* __restrict__ maskc, int nxc, int nyc, const int* __restrict__ skip) {
    if (skip && *skip) return;
    const int I = blockIdx.x * blockDim.x + threadIdx.x;
    const int J = blockIdx.y * blockDim.y + threadIdx.y;
    if (I >= nxc || J >= nyc) return;
    const long K = long(J) * nxc + I;
    ec[K] = T(0);
    if (I == 0 || J == 0 || I == nxc - 1 || J == nyc - 1 || maskc[K]) {
        gc[K] = T(0);
        return;
    }
    const long kc = long(2 * J) * nxf + 2 * I;
    T s = T(0.25) * fine_residual(e, g, mask, kc, nxf, cx, cy);
    s += T(0.125) * (fine_residual(e, g, mask, kc - 1, nxf, cx, cy) + fine_residual(e, g, mask, kc + 1, nxf, cx, cy) +
                     fine_residual(e, g, mask, kc - nxf, nxf, cx, cy) + fine_residual(e, g, mask, kc + nxf, nxf, cx, cy));
    s += T(0.0625) *
         (fine_residual(e, g, mask, kc - nxf - 1, nxf, cx, cy) + fine_residual(e, g, mask, kc - nxf + 1, nxf, cx, cy) +
          fine_residual(e, g, mask, kc + nxf - 1, nxf, cx, cy) + fine_residual(e, g, mask, kc + nxf + 1, nxf, cx, cy));
    gc[K] = s;
}

template <class T>
__global__ void k_prolong_add(T* __restrict__ ef, const uint8_t* __restrict__ maskf, int nxf, int nyf,
                              const T* __restrict__ ec, int nxc, const int* __restrict__ skip) {
    if (skip && *skip) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i < 1 || j < 1 || i >= nxf - 1 || j >= nyf - 1) return;
    const long k = long(j) * nxf + i;
    if (maskf[k]) return;
    const int I = i >> 1, J = j >> 1;
    const long K = long(J) * nxc + I;
    T v;
    if (!(i & 1) && !(j & 1)) v = ec[K];
    else if ((i & 1) && !(j & 1)) v = T(0.5) * (ec[K] + ec[K + 1]);
    else if (!(i & 1) && (j & 1)) v = T(0.5) * (ec[K] + ec[K + nxc]);
    else v = T(0.25) * (ec[K] + ec[K + 1] + ec[K + nxc] + ec[K + nxc + 1]);
    ef[k] += v;
}

template <class T>
__global__ void k_coarse_solve(T* __restrict__ e, const T* __restrict__ g, const double* __restrict__ ainv,
                               const int* __restrict__ idx, int nf, const int* __restrict__ skip) {
    if (skip && *skip) return;
    extern __shared__ double gs[];
    for (int b = threadIdx.x; b < nf; b += blockDim.x) gs[b] = double(g[idx[b]]);
    __syncthreads();
    for (int a = threadIdx.x; a < nf; a += blockDim.x) {
        const double* row = ainv + long(a) * nf;
        double s = 0.0;
        for (int b = 0; b < nf; ++b) s += row[b] * gs[b];
        e[idx[a]] = T(s);
    }
}

// Fine-grid FP64 residual; writes the correction equation's right-hand side
// g0 = r (in T), zeroes e0 and leaves one partial sum of r^2 per block.
template <class T>
__global__ void k_residual0(const double* __restrict__ phi, const double* __restrict__ f,
                            const uint8_t* __restrict__ mask, int nx, int ny, double cx, double cy, T* __restrict__ g0,
                            T* __restrict__ e0, double* __restrict__ partial, const int* __restrict__ skip) {
    if (skip && *skip) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    double r = 0.0;
    if (i < nx && j < ny) {
        const long k = long(j) * nx + i;
        if (i > 0 && j > 0 && i < nx - 1 && j < ny - 1 && !mask[k]) {
            const double c = phi[k];
            const double lap = cx * ((phi[k - 1] - c) + (phi[k + 1] - c)) + cy * ((phi[k - nx] - c) + (phi[k + nx] - c));
            r = f[k] - lap;
        }
        g0[k] = T(r);
        e0[k] = T(0);
    }
    __shared__ double ws[32];
    double s = warp_sum(r * r);
    const int t = threadIdx.y * blockDim.x + threadIdx.x;
    if ((t & 31) == 0) ws[t >> 5] = s;
    __syncthreads();
    if (t < 32) {
        const int nw = (blockDim.x * blockDim.y) >> 5;
        s = t < nw ? ws[t] : 0.0;
        s = warp_sum(s);
        if (t == 0) partial[blockIdx.y * gridDim.x + blockIdx.x] = s;
    }
}

template <class T>
__global__ void k_correct0(double* __restrict__ phi, const T* __restrict__ e0, long G, const int* __restrict__ skip) {
    if (skip && *skip) return;
    for (long k = blockIdx.x * long(blockDim.x) + threadIdx.x; k < G; k += long(gridDim.x) * blockDim.x)
        phi[k] += double(e0[k]);
}

__global__ void k_sumsq_free(const double* __restrict__ v, const uint8_t* __restrict__ mask, int nx, int ny,
                             double* __restrict__ partial) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    double x = 0.0;
    if (i > 0 && j > 0 && i < nx - 1 && j < ny - 1) {
        const long k = long(j) * nx + i;
        if (!mask[k]) x = v[k];
    }
    __shared__ double ws[32];
    double s = warp_sum(x * x);
    const int t = threadIdx.y * blockDim.x + threadIdx.x;
    if ((t & 31) == 0) ws[t >> 5] = s;
    __syncthreads();
    if (t < 32) {
        const int nw = (blockDim.x * blockDim.y) >> 5;
        s = t < nw ? ws[t] : 0.0;
        s = warp_sum(s);
        if (t == 0) partial[blockIdx.y * gridDim.x + blockIdx.x] = s;
    }
}

// Deterministic sum of the block partials.  mode 0: store ||f||^2 in norms[0];
// mode 1: store ||r||^2 in norms[1], count the cycle and raise *flag once
// ||r|| < tol ||f|| (||f|| = 0 falls back to the absolute residual).
__global__ void k_finalize(const double* __restrict__ partial, int np, double* __restrict__ norms, int mode,
                           double tol2, int* __restrict__ flag, int* __restrict__ cycles) {
    if (mode == 1 && flag && *flag) return;
    __shared__ double ws[32];
    double s = 0.0;
    for (int b = threadIdx.x; b < np; b += blockDim.x) s += partial[b];
    s = warp_sum(s);
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        s = threadIdx.x < (blockDim.x >> 5) ? ws[threadIdx.x] : 0.0;
        s = warp_sum(s);
        if (threadIdx.x == 0) {
            if (mode == 0) {
                norms[0] = s;
            } else {
                norms[1] = s;
                const double f2 = norms[0] > 0.0 ? norms[0] : 1.0;
                if (s < tol2 * f2) {
                    if (flag) *flag = 1;
                } else if (cycles) {
                    *cycles += 1;
                }
            }
        }
    }
}

__global__ void k_reset(int* flag, int* cycles) {
    *flag = 0;
    *cycles = 0;
}

// ---- host object ---------------------------------------------------------------

struct MgImpl {
    int precision = PIC_MG_MIXED;
    int nx = 0, ny = 0, L = 0;
    double dx = 0, dy = 0;
    pic_mg_options o{};
    std::vector<MgLevel<float>> lf;
    std::vector<MgLevel<double>> ld;
    std::vector<void*> allocs;
    double* ainv = nullptr;
    int* cidx = nullptr;
    int nfree_c = 0;
    double* partial = nullptr;
    int npartial = 0;
    double* norms = nullptr;  // [||f||^2, ||r||^2]
    int* flag = nullptr;      // converged
    int* cycles = nullptr;    // V-cycles run (device count)
    dim3 blk0{32, 8}, grd0;
    long long launches = 0;  // kernel launches issued (all calls)
};

}  // namespace pic

struct pic_mg {
    pic::MgImpl m;
};

namespace pic {

template <class T>
static int alloc_levels(MgImpl& M, std::vector<MgLevel<T>>& lv, const std::vector<std::vector<uint8_t>>& masks,
                        const std::vector<int>& nxs, const std::vector<int>& nys) {
    for (int l = 0; l < M.L; ++l) {
        MgLevel<T> v;
        v.nx = nxs[l];
        v.ny = nys[l];
        const double hx = M.dx * double(1 << l), hy = M.dy * double(1 << l);
        v.cx = T(1.0 / (hx * hx));
        v.cy = T(1.0 / (hy * hy));
        const size_t G = size_t(v.nx) * v.ny;
        PIC_CUDA(cudaMalloc(&v.mask, G));
        M.allocs.push_back(v.mask);
        PIC_CUDA(cudaMemcpy(v.mask, masks[l].data(), G, cudaMemcpyHostToDevice));
        PIC_CUDA(cudaMalloc(&v.e, G * sizeof(T)));
        M.allocs.push_back(v.e);
        PIC_CUDA(cudaMalloc(&v.g, G * sizeof(T)));
        M.allocs.push_back(v.g);
        PIC_CUDA(cudaMemset(v.e, 0, G * sizeof(T)));
        PIC_CUDA(cudaMemset(v.g, 0, G * sizeof(T)));
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

int mg_create(int nx, int ny, double dx, double dy, const uint8_t* h_mask, const pic_mg_options* opts,
              pic_mg** out) {
    if (!out || !h_mask || nx < 3 || ny < 3 || !(dx > 0) || !(dy > 0))
        return fail(PIC_ERR_BAD_ARG, "pic_mg_create: bad arguments");
    pic_mg* mg = new pic_mg;
    MgImpl& M = mg->m;
    M.o.precision = PIC_MG_MIXED;
    M.o.pre_sweeps = 2;
    M.o.post_sweeps = 2;
    M.o.omega = 1.0;
    M.o.coarsest_max = 9;
    if (opts) {
        M.o.precision = opts->precision;
        if (opts->pre_sweeps > 0) M.o.pre_sweeps = opts->pre_sweeps;
        if (opts->post_sweeps > 0) M.o.post_sweeps = opts->post_sweeps;
        if (opts->omega > 0) M.o.omega = opts->omega;
        if (opts->coarsest_max >= 3) M.o.coarsest_max = opts->coarsest_max;
    }
    if (M.o.precision != PIC_MG_MIXED && M.o.precision != PIC_MG_FP64) {
        delete mg;
        return fail(PIC_ERR_BAD_ARG, "pic_mg_create: unknown precision %d", M.o.precision);
    }
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
        std::vector<uint8_t> mc(size_t(cx) * cy);
        for (int J = 0; J < cy; ++J)
            for (int I = 0; I < cx; ++I) mc[size_t(J) * cx + I] = masks.back()[size_t(2 * J) * fx + 2 * I];
        nxs.push_back(cx);
        nys.push_back(cy);
        masks.push_back(std::move(mc));
    }
    M.L = int(nxs.size());
    const int ncx = nxs.back(), ncy = nys.back();
    // coarsest dense system over free interior nodes
    std::vector<int> idx;
    std::vector<int> where(size_t(ncx) * ncy, -1);
    for (int j = 1; j < ncy - 1; ++j)
        for (int i = 1; i < ncx - 1; ++i)
            if (!masks.back()[size_t(j) * ncx + i]) {
                where[size_t(j) * ncx + i] = int(idx.size());
                idx.push_back(j * ncx + i);
            }
    M.nfree_c = int(idx.size());
    if (M.nfree_c > 4096) {
        delete mg;
        return fail(PIC_ERR_BAD_ARG,
                    "pic_mg_create: coarsest level %dx%d has %d unknowns; node counts must be 2^k*c+1 with a small c",
                    ncx, ncy, M.nfree_c);
    }
    if (M.nfree_c > 0) {
        const double hx = dx * double(1 << (M.L - 1)), hy = dy * double(1 << (M.L - 1));
        const double ccx = 1.0 / (hx * hx), ccy = 1.0 / (hy * hy);
        const int n = M.nfree_c;
        std::vector<double> A(size_t(n) * n, 0.0);
        for (int a = 0; a < n; ++a) {
            const int k = idx[a];
            A[size_t(a) * n + a] = -2.0 * (ccx + ccy);
            const int nb[4] = {k - 1, k + 1, k - ncx, k + ncx};
            const double w[4] = {ccx, ccx, ccy, ccy};
            for (int q = 0; q < 4; ++q) {
                const int b = where[nb[q]];
                if (b >= 0) A[size_t(a) * n + b] += w[q];
            }
        }
        if (!invert(A, n)) {
            delete mg;
            return fail(PIC_ERR_NUMERIC, "pic_mg_create: singular coarsest system");
        }
        PIC_CUDA(cudaMalloc(&M.ainv, A.size() * sizeof(double)));
        M.allocs.push_back(M.ainv);
        PIC_CUDA(cudaMemcpy(M.ainv, A.data(), A.size() * sizeof(double), cudaMemcpyHostToDevice));
        PIC_CUDA(cudaMalloc(&M.cidx, idx.size() * sizeof(int)));
        M.allocs.push_back(M.cidx);
        PIC_CUDA(cudaMemcpy(M.cidx, idx.data(), idx.size() * sizeof(int), cudaMemcpyHostToDevice));
    }
    int st = M.precision == PIC_MG_MIXED ? alloc_levels(M, M.lf, masks, nxs, nys)
                                         : alloc_levels(M, M.ld, masks, nxs, nys);
    if (st != PIC_OK) {
        delete mg;
        return st;
    }
    M.grd0 = dim3(div_up(nx, M.blk0.x), div_up(ny, M.blk0.y));
    M.npartial = int(M.grd0.x * M.grd0.y);
    PIC_CUDA(cudaMalloc(&M.partial, sizeof(double) * M.npartial));
    M.allocs.push_back(M.partial);
    PIC_CUDA(cudaMalloc(&M.norms, sizeof(double) * 2));
    M.allocs.push_back(M.norms);
    PIC_CUDA(cudaMalloc(&M.flag, sizeof(int) * 2));
    M.allocs.push_back(M.flag);
    M.cycles = M.flag + 1;
    PIC_CUDA(cudaMemset(M.flag, 0, sizeof(int) * 2));
    PIC_CUDA(cudaMemset(M.norms, 0, sizeof(double) * 2));
    *out = mg;
    return PIC_OK;
}

template <class T>
static int vcycle(MgImpl& M, std::vector<MgLevel<T>>& lv, cudaStream_t st, const int* skip) {
    const dim3 b2(32, 8);
    M.launches += (long long)(M.L - 1) * (2 * M.o.pre_sweeps + 2 + 2 * M.o.post_sweeps) + (M.nfree_c > 0 ? 1 : 0);
    const T omega = T(M.o.omega);
    for (int l = 0; l < M.L - 1; ++l) {
        MgLevel<T>& f = lv[l];
        MgLevel<T>& c = lv[l + 1];
        const dim3 gs(div_up((f.nx + 1) / 2, b2.x), div_up(f.ny - 2, b2.y));
        for (int s = 0; s < M.o.pre_sweeps; ++s)
            for (int color = 0; color < 2; ++color)
                k_smooth<T><<<gs, b2, 0, st>>>(f.e, f.g, f.mask, f.nx, f.ny, f.cx, f.cy, omega, color, skip);
        const dim3 gc(div_up(c.nx, b2.x), div_up(c.ny, b2.y));
        k_resid_restrict<T><<<gc, b2, 0, st>>>(f.e, f.g, f.mask, f.nx, f.cx, f.cy, c.g, c.e, c.mask, c.nx, c.ny, skip);
    }
    MgLevel<T>& cl = lv[M.L - 1];
    if (M.nfree_c > 0) {
        const int thr = M.nfree_c < 1024 ? ((M.nfree_c + 31) / 32) * 32 : 1024;
        k_coarse_solve<T><<<1, thr, sizeof(double) * M.nfree_c, st>>>(cl.e, cl.g, M.ainv, M.cidx, M.nfree_c, skip);
    }
    for (int l = M.L - 2; l >= 0; --l) {
        MgLevel<T>& f = lv[l];
        MgLevel<T>& c = lv[l + 1];
        const dim3 gp(div_up(f.nx, b2.x), div_up(f.ny, b2.y));
        k_prolong_add<T><<<gp, b2, 0, st>>>(f.e, f.mask, f.nx, f.ny, c.e, c.nx, skip);
        const dim3 gs(div_up((f.nx + 1) / 2, b2.x), div_up(f.ny - 2, b2.y));
        for (int s = 0; s < M.o.post_sweeps; ++s)
            for (int color = 0; color < 2; ++color)
                k_smooth<T><<<gs, b2, 0, st>>>(f.e, f.g, f.mask, f.nx, f.ny, f.cx, f.cy, omega, color, skip);
    }
    PIC_LAUNCH_CHECK();
    return PIC_OK;
}

template <class T>
static int residual0(MgImpl& M, std::vector<MgLevel<T>>& lv, const double* phi, const double* f, cudaStream_t st,
                     const int* skip, double tol, bool count) {
    MgLevel<T>& l0 = lv[0];
    k_residual0<T><<<M.grd0, M.blk0, 0, st>>>(phi, f, l0.mask, M.nx, M.ny, 1.0 / (M.dx * M.dx),
                                              1.0 / (M.dy * M.dy), l0.g, l0.e, M.partial, skip);
    k_finalize<<<1, 1024, 0, st>>>(M.partial, M.npartial, M.norms, 1, tol * tol, M.flag, count ? M.cycles : nullptr);
    M.launches += 2;
    PIC_LAUNCH_CHECK();
    return PIC_OK;
}

template <class T>
static int correct0(MgImpl& M, std::vector<MgLevel<T>>& lv, double* phi, cudaStream_t st, const int* skip) {
    const long G = long(M.nx) * M.ny;
    k_correct0<T><<<grid_blocks(G, 256), 256, 0, st>>>(phi, lv[0].e, G, skip);
    M.launches += 1;
    PIC_LAUNCH_CHECK();
    return PIC_OK;
}

static int rhs_norm(MgImpl& M, const double* f, cudaStream_t st) {
    const uint8_t* mask0 = M.precision == PIC_MG_MIXED ? M.lf[0].mask : M.ld[0].mask;
    k_sumsq_free<<<M.grd0, M.blk0, 0, st>>>(f, mask0, M.nx, M.ny, M.partial);
    k_finalize<<<1, 1024, 0, st>>>(M.partial, M.npartial, M.norms, 0, 0.0, nullptr, nullptr);
    M.launches += 2;
    PIC_LAUNCH_CHECK();
    return PIC_OK;
}

int mg_residual_step(MgImpl& M, const double* phi, const double* f, cudaStream_t st, const int* skip, double tol,
                     bool count) {
    return M.precision == PIC_MG_MIXED ? residual0(M, M.lf, phi, f, st, skip, tol, count)
                                       : residual0(M, M.ld, phi, f, st, skip, tol, count);
}

int mg_cycle_and_correct(MgImpl& M, double* phi, cudaStream_t st, const int* skip) {
    if (M.precision == PIC_MG_MIXED) {
        PIC_TRY(vcycle(M, M.lf, st, skip));
        return correct0(M, M.lf, phi, st, skip);
    }
    PIC_TRY(vcycle(M, M.ld, st, skip));
    return correct0(M, M.ld, phi, st, skip);
}

int mg_solve_async(MgImpl& M, double* phi, const double* f, double tol, int cycles, cudaStream_t st) {
    k_reset<<<1, 1, 0, st>>>(M.flag, M.cycles);
    M.launches += 1;
    PIC_TRY(rhs_norm(M, f, st));
    for (int c = 0; c < cycles; ++c) {
        PIC_TRY(mg_residual_step(M, phi, f, st, M.flag, tol, true));
        PIC_TRY(mg_cycle_and_correct(M, phi, st, M.flag));
    }
    // final residual of the last correction
    PIC_TRY(mg_residual_step(M, phi, f, st, M.flag, tol, false));
    return PIC_OK;
}

int mg_read_info(MgImpl& M, double tol, pic_mg_info* info) {
    double norms[2];
    int fc[2];
    PIC_CUDA(cudaMemcpy(norms, M.norms, sizeof norms, cudaMemcpyDeviceToHost));
    PIC_CUDA(cudaMemcpy(fc, M.flag, sizeof fc, cudaMemcpyDeviceToHost));
    info->rhs_norm = std::sqrt(norms[0]);
    const double f = norms[0] > 0 ? std::sqrt(norms[0]) : 1.0;
    info->rel_res = std::sqrt(norms[1]) / f;
    info->cycles = fc[1];
    info->converged = fc[0] ? 1 : (info->rel_res < tol ? 1 : 0);
    return PIC_OK;
}

int mg_solve(MgImpl& M, double* phi, const double* f, double tol, int max_cycles, pic_mg_info* info,
             cudaStream_t st) {
    k_reset<<<1, 1, 0, st>>>(M.flag, M.cycles);
    M.launches += 1;
    PIC_TRY(rhs_norm(M, f, st));
    pic_mg_info loc{};
    int c = 0;
    for (;;) {
        PIC_TRY(mg_residual_step(M, phi, f, st, nullptr, tol, false));
        PIC_CUDA(cudaStreamSynchronize(st));
        PIC_TRY(mg_read_info(M, tol, &loc));
        loc.cycles = c;
        if (loc.converged || c >= max_cycles) break;
        PIC_TRY(mg_cycle_and_correct(M, phi, st, nullptr));
        ++c;
    }
    if (info) *info = loc;
    if (!loc.converged)
        return fail(PIC_ERR_NOT_CONVERGED, "multigrid: relative residual %.3e after %d cycles (tol %.1e)", loc.rel_res,
                    loc.cycles, tol);
    return PIC_OK;
}

long long mg_launches(pic_mg* mg) { return mg ? mg->m.launches : 0; }

}  // namespace pic

using namespace pic;

extern "C" {

int pic_mg_create(int nx, int ny, double dx, double dy, const uint8_t* h_dirichlet, const pic_mg_options* opts,
                  pic_mg** out) {
    clear_error();
    return mg_create(nx, ny, dx, dy, h_dirichlet, opts, out);
}

int pic_mg_destroy(pic_mg* mg) {
    clear_error();
    if (!mg) return PIC_OK;
    for (void* p : mg->m.allocs) cudaFree(p);
    delete mg;
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
    return mg_solve_async(mg->m, d_phi, d_f, tol, cycles, as_stream(stream));
}

int pic_mg_read_info(pic_mg* mg, double tol, pic_mg_info* info) {
    clear_error();
    if (!mg || !info) return fail(PIC_ERR_BAD_ARG, "pic_mg_read_info: bad arguments");
    return mg_read_info(mg->m, tol, info);
}

}  // extern "C"
