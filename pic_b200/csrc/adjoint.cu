// Hand-written adjoint of the collisionless step: CIC deposit -> multigrid
// Poisson solve -> E = -grad(phi) -> kick -> drift with wall absorption, in
// FP64, with gradients of a final-density loss with respect to the potentials
// of electrode segments and to the amplitude of an initial-velocity
// perturbation.
//
// Forward model (the reference's order, src/simulation.py:622-660):
//   init:  rho_0 = D(x_0), phi_0 = P(rho_0; V), E_0 = G phi_0,
//          u_0 = v_0 + A dv - (k/2) I(x_0; E_0)
//   step n = 0 .. N-1:
//          x_{n+1} = x_n + c u_n          (absorbed when outside the grid)
//          rho_{n+1} = D(x_{n+1}), phi_{n+1} = P(rho_{n+1}; V), E_{n+1} = G phi_{n+1}
//          u_{n+1} = u_n + k I(x_{n+1}; E_{n+1})
//   loss:  L = mean over nodes of (n_s(x_N) - n_target)^2 for one species s
// D is the CIC deposit (src/Grid.py:96-154), P the Poisson solve with
// Dirichlet values V on the electrode segments (f = -rho/eps0 on free nodes),
// G the gradient stencil of src/Grid.py:167-194 (one-sided on the edges), I
// the bilinear gather (src/Particles.py:117-180), k = q dt/m, c = dt/dx.
//
// Adjoint, per step n from N-1 down to 0 (absorption is a fixed mask: a
// particle dead at a state takes no part in it):
//   kick:    lambda_u_n += lambda_u_{n+1};  lambda_x_{n+1} += k (dI/dx)^T lambda_u_{n+1}
//            lambda_E_{n+1} = k I^T lambda_u_{n+1}              (a CIC scatter)
//   field:   lambda_phi = G^T lambda_E;  solve A mu = lambda_phi on free nodes
//            (A is symmetric, so the adjoint solve is one more multigrid solve
//            with zero boundary values); dL/dV_seg += sum over the segment's
//            nodes of lambda_phi_B - sum of the free neighbours' couplings * mu
//   deposit: lambda_x_{n+1} += (q np2c/(dx dy)) (dW/dx)^T (-mu/eps0)
//   drift:   lambda_u_n += c lambda_x_{n+1};  lambda_x_n = lambda_x_{n+1}
// and for the init half-kick and the perturbation:
//   dL/dA = sum_p lambda_u_0 . dv_p, plus the field terms of the init kick.
// The forward pass keeps a checkpoint (positions, velocities, phi) every C
// steps; the backward pass recomputes each segment of C steps from its
// checkpoint, keeping the segment's positions and fields, then walks it back.
#include <climits>
#include <vector>

#include "common.cuh"

namespace pic {

int grid_blocks(long n, int threads);
int mg_create(int nx, int ny, double dx, double dy, const uint8_t* h_mask, const pic_mg_options* opts, pic_mg** out);
int mg_launch_graph(pic_mg* mg, double* phi, const double* f, double tol, int max_cycles, int min_cycles,
                    cudaStream_t st);
const int* mg_device_converged(pic_mg* mg);

struct AdSpecies {
    double kq[PIC_MAX_SPECIES];      // q dt / m
    double charge[PIC_MAX_SPECIES];  // q np2c / (dx dy): charge density of one particle at weight 1
    double dens[PIC_MAX_SPECIES];    // np2c / (dx dy): number density of one particle at weight 1
};

// Cell of a live particle (grid units, inside [0, n-1]) and its offsets;
// x = n-1 falls in the last cell with weight 1 on its far node.
struct AdCell {
    int i, j;
    double fx, fy;
};

__device__ __forceinline__ AdCell ad_cell(double x, double y, int nx, int ny) {
    AdCell c;
    c.i = max(0, min(int(floor(x)), nx - 2));
    c.j = max(0, min(int(floor(y)), ny - 2));
    c.fx = x - double(c.i);
    c.fy = y - double(c.j);
    return c;
}

__device__ __forceinline__ double ad_interp(const double* __restrict__ F, const AdCell& c, int nx) {
    const long k = long(c.j) * nx + c.i;
    return (1.0 - c.fx) * (1.0 - c.fy) * F[k] + c.fx * (1.0 - c.fy) * F[k + 1] + (1.0 - c.fx) * c.fy * F[k + nx] +
           c.fx * c.fy * F[k + nx + 1];
}

// Gradient (per grid unit) of the bilinear interpolant of F at the particle.
__device__ __forceinline__ double2 ad_interp_grad(const double* __restrict__ F, const AdCell& c, int nx) {
    const long k = long(c.j) * nx + c.i;
    const double f00 = F[k], f10 = F[k + 1], f01 = F[k + nx], f11 = F[k + nx + 1];
    return make_double2((1.0 - c.fy) * (f10 - f00) + c.fy * (f11 - f01), (1.0 - c.fx) * (f01 - f00) + c.fx * (f11 - f10));
}

__device__ __forceinline__ void ad_scatter(double* __restrict__ F, const AdCell& c, int nx, double v) {
    const long k = long(c.j) * nx + c.i;
    atomicAdd(F + k, (1.0 - c.fx) * (1.0 - c.fy) * v);
    atomicAdd(F + k + 1, c.fx * (1.0 - c.fy) * v);
    atomicAdd(F + k + nx, (1.0 - c.fx) * c.fy * v);
    atomicAdd(F + k + nx + 1, c.fx * c.fy * v);
}

__device__ __forceinline__ bool alive(const int* __restrict__ death, int p, int state) { return death[p] > state; }

// ---- forward kernels --------------------------------------------------------------

// rho += charge (or number) density of the live particles; only species `only` if >= 0.
__global__ void k_ad_deposit(const double* __restrict__ x, const double* __restrict__ y,
                             const uint8_t* __restrict__ sp, const int* __restrict__ death, int state, int n, int nx,
                             int ny, AdSpecies S, int number, int only, double* __restrict__ rho) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        if (!alive(death, p, state)) continue;
        const int s = sp[p];
        if (only >= 0 && s != only) continue;
        ad_scatter(rho, ad_cell(x[p], y[p], nx, ny), nx, number ? S.dens[s] : S.charge[s]);
    }
}

// f = -rho/eps0 on free nodes, 0 on Dirichlet nodes; clears rho for the next deposit.
__global__ void k_ad_rhs(double* __restrict__ rho, const uint8_t* __restrict__ mask, double neg_inv_eps0,
                         double* __restrict__ f, long G) {
    for (long k = blockIdx.x * long(blockDim.x) + threadIdx.x; k < G; k += long(gridDim.x) * blockDim.x) {
        f[k] = mask[k] ? 0.0 : rho[k] * neg_inv_eps0;
        rho[k] = 0.0;
    }
}

// Dirichlet values: V[segment] on electrode nodes, the fixed value elsewhere.
__global__ void k_ad_bc(double* __restrict__ phi, const uint8_t* __restrict__ mask, const int* __restrict__ seg,
                        const double* __restrict__ fixed, const double* __restrict__ V, long G) {
    for (long k = blockIdx.x * long(blockDim.x) + threadIdx.x; k < G; k += long(gridDim.x) * blockDim.x)
        if (mask[k]) phi[k] = seg[k] >= 0 ? V[seg[k]] : fixed[k];
}

// E = -grad(phi) with the stencil of src/Grid.py:167-194.
__global__ void k_ad_efield(const double* __restrict__ phi, double* __restrict__ Ex, double* __restrict__ Ey, int nx,
                            int ny, double dx, double dy) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y;
    if (i >= nx) return;
    const long k = long(j) * nx + i;
    double ex, ey;
    if (i > 0 && i < nx - 1) ex = -(phi[k + 1] - phi[k - 1]) / (2.0 * dx);
    else if (i == 0) ex = -(phi[k + 1] - phi[k]) / dx;
    else ex = -(phi[k] - phi[k - 1]) / dx;
    if (j > 0 && j < ny - 1) ey = -(phi[k + nx] - phi[k - nx]) / (2.0 * dy);
    else if (j == 0) ey = -(phi[k + nx] - phi[k]) / dy;
    else ey = -(phi[k] - phi[k - nx]) / dy;
    Ex[k] = ex;
    Ey[k] = ey;
}

// u += factor k I(x; E) for particles alive at `state`.
__global__ void k_ad_kick(const double* __restrict__ x, const double* __restrict__ y, double* __restrict__ ux,
                          double* __restrict__ uy, const uint8_t* __restrict__ sp, const int* __restrict__ death,
                          int state, int n, int nx, int ny, const double* __restrict__ Ex,
                          const double* __restrict__ Ey, AdSpecies S, double factor) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        if (!alive(death, p, state)) continue;
        const AdCell c = ad_cell(x[p], y[p], nx, ny);
        const double k = factor * S.kq[sp[p]];
        ux[p] += k * ad_interp(Ex, c, nx);
        uy[p] += k * ad_interp(Ey, c, nx);
    }
}

// x += c u for particles alive at `state`; a particle that leaves [0, n-1]^2
// dies at state + 1 (unless the absorption steps are frozen).
__global__ void k_ad_drift(double* __restrict__ x, double* __restrict__ y, const double* __restrict__ ux,
                           const double* __restrict__ uy, int* __restrict__ death, int state, int n, int nx, int ny,
                           double cx, double cy, int frozen) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        if (!alive(death, p, state)) continue;
        const double a = x[p] + cx * ux[p], b = y[p] + cy * uy[p];
        x[p] = a;
        y[p] = b;
        if (!frozen && !(a >= 0.0 && a <= double(nx - 1) && b >= 0.0 && b <= double(ny - 1))) death[p] = state + 1;
    }
}

// v0 + A dv
__global__ void k_ad_perturb(double* __restrict__ ux, double* __restrict__ uy, const double* __restrict__ dvx,
                             const double* __restrict__ dvy, double A, int n) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        ux[p] += A * dvx[p];
        uy[p] += A * dvy[p];
    }
}

// loss = sum (dens - target)^2 / G, and g = dL/d dens = 2 (dens - target) / G.
__global__ void k_ad_loss(const double* __restrict__ dens, const double* __restrict__ target, double* __restrict__ g,
                          long G, double* __restrict__ loss) {
    double s = 0.0;
    for (long k = blockIdx.x * long(blockDim.x) + threadIdx.x; k < G; k += long(gridDim.x) * blockDim.x) {
        const double d = dens[k] - target[k];
        g[k] = 2.0 * d / double(G);
        s += d * d / double(G);
    }
    s = warp_sum(s);
    if ((threadIdx.x & 31) == 0) atomicAdd(loss, s);
}

// ---- adjoint kernels --------------------------------------------------------------

// Adjoint of u += factor k I(x; E) at `state`: lambda_x += factor k (dI/dx)^T
// lambda_u and lambda_E += factor k I^T lambda_u.
__global__ void k_ad_kick_adj(const double* __restrict__ x, const double* __restrict__ y,
                              const uint8_t* __restrict__ sp, const int* __restrict__ death, int state, int n, int nx,
                              int ny, const double* __restrict__ Ex, const double* __restrict__ Ey, AdSpecies S,
                              double factor, const double* __restrict__ lux, const double* __restrict__ luy,
                              double* __restrict__ lx, double* __restrict__ ly, double* __restrict__ lEx,
                              double* __restrict__ lEy) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        if (!alive(death, p, state)) continue;
        const double k = factor * S.kq[sp[p]];
        const double bx = k * lux[p], by = k * luy[p];
        if (bx == 0.0 && by == 0.0) continue;
        const AdCell c = ad_cell(x[p], y[p], nx, ny);
        const double2 gx = ad_interp_grad(Ex, c, nx), gy = ad_interp_grad(Ey, c, nx);
        lx[p] += bx * gx.x + by * gy.x;
        ly[p] += bx * gx.y + by * gy.y;
        ad_scatter(lEx, c, nx, bx);
        ad_scatter(lEy, c, nx, by);
    }
}

// lambda_phi = G^T lambda_E (transpose of k_ad_efield), and the right-hand
// side of the adjoint solve (lambda_phi on free nodes, 0 on Dirichlet nodes).
// Clears lambda_E.
__global__ void k_ad_gradT(double* __restrict__ lEx, double* __restrict__ lEy, const uint8_t* __restrict__ mask,
                           double* __restrict__ lphi, double* __restrict__ fa, int nx, int ny, double dx, double dy) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y;
    if (i >= nx) return;
    const long k = long(j) * nx + i;
    const double hx = 0.5 / dx, hy = 0.5 / dy;
    double v = 0.0;
    if (i + 1 >= 1 && i + 1 <= nx - 2) v += hx * lEx[k + 1];
    if (i - 1 >= 1 && i - 1 <= nx - 2) v -= hx * lEx[k - 1];
    if (i == 0) v += lEx[k] / dx;
    if (i == 1) v -= lEx[k - 1] / dx;
    if (i == nx - 1) v -= lEx[k] / dx;
    if (i == nx - 2) v += lEx[k + 1] / dx;
    if (j + 1 >= 1 && j + 1 <= ny - 2) v += hy * lEy[k + nx];
    if (j - 1 >= 1 && j - 1 <= ny - 2) v -= hy * lEy[k - nx];
    if (j == 0) v += lEy[k] / dy;
    if (j == 1) v -= lEy[k - nx] / dy;
    if (j == ny - 1) v -= lEy[k] / dy;
    if (j == ny - 2) v += lEy[k + nx] / dy;
    lphi[k] = v;
    fa[k] = mask[k] ? 0.0 : v;
}

__global__ void k_ad_zero2(double* __restrict__ a, double* __restrict__ b, long G) {
    for (long k = blockIdx.x * long(blockDim.x) + threadIdx.x; k < G; k += long(gridDim.x) * blockDim.x) {
        a[k] = 0.0;
        b[k] = 0.0;
    }
}

// dL/dV[seg] += lambda_phi_B - sum over free neighbours of the coupling * mu,
// over the Dirichlet nodes B of each electrode segment.
__global__ void k_ad_dV(const double* __restrict__ lphi, const double* __restrict__ mu,
                        const uint8_t* __restrict__ mask, const int* __restrict__ seg, int nx, int ny, double cx,
                        double cy, double* __restrict__ dV) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y;
    if (i >= nx) return;
    const long k = long(j) * nx + i;
    if (!mask[k] || seg[k] < 0) return;
    double v = lphi[k];
    auto free_node = [&](int a, int b) {
        return a > 0 && b > 0 && a < nx - 1 && b < ny - 1 && !mask[long(b) * nx + a];
    };
    if (free_node(i - 1, j)) v -= cx * mu[k - 1];
    if (free_node(i + 1, j)) v -= cx * mu[k + 1];
    if (free_node(i, j - 1)) v -= cy * mu[k - nx];
    if (free_node(i, j + 1)) v -= cy * mu[k + nx];
    atomicAdd(dV + seg[k], v);
}

// Deposit and drift adjoints at `state` (> 0): lambda_x += charge (dW/dx)^T
// (-mu/eps0) for particles alive at `state`, then lambda_u += c lambda_x for
// particles alive at state - 1 (the drift into `state`).
__global__ void k_ad_dep_drift_adj(const double* __restrict__ x, const double* __restrict__ y,
                                   const uint8_t* __restrict__ sp, const int* __restrict__ death, int state, int n,
                                   int nx, int ny, const double* __restrict__ mu, AdSpecies S, double neg_inv_eps0,
                                   double cx, double cy, double* __restrict__ lx, double* __restrict__ ly,
                                   double* __restrict__ lux, double* __restrict__ luy) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        if (!alive(death, p, state - 1)) continue;
        double ax = lx[p], ay = ly[p];
        if (alive(death, p, state)) {
            const double2 g = ad_interp_grad(mu, ad_cell(x[p], y[p], nx, ny), nx);
            const double s = S.charge[sp[p]] * neg_inv_eps0;
            ax += s * g.x;
            ay += s * g.y;
            lx[p] = ax;
            ly[p] = ay;
        }
        lux[p] += cx * ax;
        luy[p] += cy * ay;
    }
}

// lambda_x += dens (dW/dx)^T g for the loss species alive at the final state.
__global__ void k_ad_loss_adj(const double* __restrict__ x, const double* __restrict__ y,
                              const uint8_t* __restrict__ sp, const int* __restrict__ death, int state, int n, int nx,
                              int ny, const double* __restrict__ g, AdSpecies S, int only, double* __restrict__ lx,
                              double* __restrict__ ly) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        if (!alive(death, p, state) || sp[p] != only) continue;
        const double2 d = ad_interp_grad(g, ad_cell(x[p], y[p], nx, ny), nx);
        lx[p] += S.dens[sp[p]] * d.x;
        ly[p] += S.dens[sp[p]] * d.y;
    }
}

// dA = sum_p lambda_u . dv
__global__ void k_ad_dot(const double* __restrict__ lux, const double* __restrict__ luy,
                         const double* __restrict__ dvx, const double* __restrict__ dvy, int n,
                         double* __restrict__ out) {
    double s = 0.0;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x)
        s += lux[p] * dvx[p] + luy[p] * dvy[p];
    s = warp_sum(s);
    if ((threadIdx.x & 31) == 0) atomicAdd(out, s);
}

// Records a solve that did not converge.
__global__ void k_ad_track(const int* __restrict__ converged, int* __restrict__ failures) {
    if (!*converged) atomicAdd(failures, 1);
}

// ---- host object ------------------------------------------------------------------

struct AdjImpl {
    pic_adj_desc d{};
    int n = 0;  // particles of all species
    long G = 0;
    int first[PIC_MAX_SPECIES + 1]{};
    AdSpecies S{};
    pic_mg* mg = nullptr;   // forward solves
    pic_mg* mga = nullptr;  // adjoint solves
    std::vector<void*> allocs;
    // particles
    double *x0 = nullptr, *y0 = nullptr, *vx0 = nullptr, *vy0 = nullptr, *dvx = nullptr, *dvy = nullptr;
    uint8_t* sp = nullptr;
    double *x = nullptr, *y = nullptr, *ux = nullptr, *uy = nullptr;
    int* death = nullptr;
    double *lx = nullptr, *ly = nullptr, *lux = nullptr, *luy = nullptr;
    // checkpoints: x, y, ux, uy per particle and phi, every C steps (states 0, C, 2C, ...)
    int ncp = 0;
    double* cp = nullptr;
    double* cp_phi = nullptr;
    // one segment of positions and fields (states a+1 .. a+C)
    double *seg_xy = nullptr, *seg_E = nullptr;
    // grids
    uint8_t* mask = nullptr;
    int* segid = nullptr;
    double *fixed = nullptr, *V = nullptr, *rho = nullptr, *f = nullptr, *phi = nullptr, *Ex = nullptr, *Ey = nullptr;
    double *lEx = nullptr, *lEy = nullptr, *lphi = nullptr, *fa = nullptr, *mu = nullptr, *target = nullptr,
           *g = nullptr;
    double* red = nullptr;  // [0] loss, [1] dA, [2..] dV
    int* failures = nullptr;
    double A = 0.0;
    bool have_forward = false;
    bool frozen = false;  // reuse the absorption steps of the last forward pass
    double loss = 0.0;
};

template <class T>
static int adalloc(AdjImpl& J, T** p, size_t n) {
    PIC_CUDA(cudaMalloc(p, sizeof(T) * std::max<size_t>(n, 1)));
    J.allocs.push_back(*p);
    PIC_CUDA(cudaMemset(*p, 0, sizeof(T) * std::max<size_t>(n, 1)));
    return PIC_OK;
}

static void adj_free(AdjImpl& J) {
    if (J.mg) pic_mg_destroy(J.mg);
    if (J.mga) pic_mg_destroy(J.mga);
    J.mg = J.mga = nullptr;
    for (void* p : J.allocs) cudaFree(p);
    J.allocs.clear();
}

static int adj_create(const pic_adj_desc* d, AdjImpl& J) {
    if (!d || d->nx < 3 || d->ny < 3 || !(d->dx > 0) || !(d->dy > 0) || !(d->dt > 0) || !(d->eps0 > 0) ||
        d->nspecies < 1 || d->nspecies > PIC_MAX_SPECIES || !d->h_dirichlet || !d->h_segment || d->nseg < 0 ||
        d->nseg > PIC_ADJ_MAX_SEGMENTS || d->steps < 1 || d->checkpoint_every < 1 || d->loss_species < 0 ||
        d->loss_species >= d->nspecies || !(d->tol >= 0) || d->max_cycles < 1)
        return fail(PIC_ERR_BAD_ARG, "pic_adj_create: bad descriptor");
    J.d = *d;
    J.G = long(d->nx) * d->ny;
    J.n = 0;
    for (int s = 0; s < d->nspecies; ++s) {
        const pic_adj_species& q = d->species[s];
        if (q.n < 0 || !(q.mass > 0) || !(q.np2c > 0)) return fail(PIC_ERR_BAD_ARG, "pic_adj_create: species %d", s);
        J.first[s] = J.n;
        J.n += q.n;
        J.S.kq[s] = q.charge * d->dt / q.mass;
        J.S.charge[s] = q.charge * q.np2c / (d->dx * d->dy);
        J.S.dens[s] = q.np2c / (d->dx * d->dy);
    }
    J.first[d->nspecies] = J.n;
    std::vector<uint8_t> mask(d->h_dirichlet, d->h_dirichlet + J.G);
    for (long k = 0; k < J.G; ++k) {
        const int i = int(k % d->nx), j = int(k / d->nx);
        mask[k] = (mask[k] || i == 0 || j == 0 || i == d->nx - 1 || j == d->ny - 1) ? 1 : 0;
        if (d->h_segment[k] >= d->nseg) return fail(PIC_ERR_BAD_ARG, "pic_adj_create: segment index out of range");
    }
    pic_mg_options o{};
    o.precision = PIC_MG_FP64;
    o.pre_sweeps = o.post_sweeps = 2;
    o.omega = 1.0;
    o.coarsest_max = 9;
    o.launch_mode = PIC_MG_GRAPH_LOOP;
    PIC_TRY(mg_create(d->nx, d->ny, d->dx, d->dy, mask.data(), &o, &J.mg));
    PIC_TRY(mg_create(d->nx, d->ny, d->dx, d->dy, mask.data(), &o, &J.mga));
    const size_t n = size_t(std::max(J.n, 1)), G = size_t(J.G);
    for (double** p : {&J.x0, &J.y0, &J.vx0, &J.vy0, &J.dvx, &J.dvy, &J.x, &J.y, &J.ux, &J.uy, &J.lx, &J.ly, &J.lux,
                       &J.luy})
        PIC_TRY(adalloc(J, p, n));
    PIC_TRY(adalloc(J, &J.sp, n));
    PIC_TRY(adalloc(J, &J.death, n));
    J.ncp = (d->steps + d->checkpoint_every - 1) / d->checkpoint_every;  // states 0, C, ... < steps
    PIC_TRY(adalloc(J, &J.cp, size_t(J.ncp) * 4 * n));
    PIC_TRY(adalloc(J, &J.cp_phi, size_t(J.ncp) * G));
    const size_t C = size_t(std::min(d->checkpoint_every, d->steps));
    PIC_TRY(adalloc(J, &J.seg_xy, C * 2 * n));
    PIC_TRY(adalloc(J, &J.seg_E, C * 2 * G));
    PIC_TRY(adalloc(J, &J.mask, G));
    PIC_CUDA(cudaMemcpy(J.mask, mask.data(), G, cudaMemcpyHostToDevice));
    PIC_TRY(adalloc(J, &J.segid, G));
    PIC_CUDA(cudaMemcpy(J.segid, d->h_segment, sizeof(int) * G, cudaMemcpyHostToDevice));
    PIC_TRY(adalloc(J, &J.fixed, G));
    if (d->h_phi_fixed) PIC_CUDA(cudaMemcpy(J.fixed, d->h_phi_fixed, sizeof(double) * G, cudaMemcpyHostToDevice));
    for (double** p : {&J.rho, &J.f, &J.phi, &J.Ex, &J.Ey, &J.lEx, &J.lEy, &J.lphi, &J.fa, &J.mu, &J.target, &J.g})
        PIC_TRY(adalloc(J, p, G));
    PIC_TRY(adalloc(J, &J.V, size_t(PIC_ADJ_MAX_SEGMENTS)));
    PIC_TRY(adalloc(J, &J.red, size_t(2 + PIC_ADJ_MAX_SEGMENTS)));
    PIC_TRY(adalloc(J, &J.failures, 1));
    std::vector<uint8_t> spv(n, 0);
    for (int s = 0; s < d->nspecies; ++s)
        for (int p = J.first[s]; p < J.first[s + 1]; ++p) spv[p] = uint8_t(s);
    PIC_CUDA(cudaMemcpy(J.sp, spv.data(), n, cudaMemcpyHostToDevice));
    return PIC_OK;
}

static int grid2(const AdjImpl& J, dim3& g) {
    g = dim3(div_up(J.d.nx, 128), J.d.ny);
    return 128;
}

// rho -> phi -> E for the particles alive at `state` (phi keeps its previous
// value as the initial guess).
static int field_of(AdjImpl& J, int state, double* Ex, double* Ey, cudaStream_t st) {
    const int pb = grid_blocks(J.n, 256), gb = grid_blocks(J.G, 256);
    k_ad_deposit<<<pb, 256, 0, st>>>(J.x, J.y, J.sp, J.death, state, J.n, J.d.nx, J.d.ny, J.S, 0, -1, J.rho);
    k_ad_rhs<<<gb, 256, 0, st>>>(J.rho, J.mask, -1.0 / J.d.eps0, J.f, J.G);
    PIC_LAUNCH_CHECK();
    PIC_TRY(mg_launch_graph(J.mg, J.phi, J.f, J.d.tol, J.d.max_cycles, 0, st));
    if (J.d.tol > 0) k_ad_track<<<1, 1, 0, st>>>(mg_device_converged(J.mg), J.failures);
    dim3 g;
    const int t = grid2(J, g);
    k_ad_efield<<<g, t, 0, st>>>(J.phi, Ex, Ey, J.d.nx, J.d.ny, J.d.dx, J.d.dy);
    PIC_LAUNCH_CHECK();
    return PIC_OK;
}

// One step from `state` to state + 1; the new state's E goes to (Ex, Ey).
static int step_of(AdjImpl& J, int state, double* Ex, double* Ey, cudaStream_t st) {
    const int pb = grid_blocks(J.n, 256);
    k_ad_drift<<<pb, 256, 0, st>>>(J.x, J.y, J.ux, J.uy, J.death, state, J.n, J.d.nx, J.d.ny, J.d.dt / J.d.dx,
                                   J.d.dt / J.d.dy, J.frozen ? 1 : 0);
    PIC_TRY(field_of(J, state + 1, Ex, Ey, st));
    k_ad_kick<<<pb, 256, 0, st>>>(J.x, J.y, J.ux, J.uy, J.sp, J.death, state + 1, J.n, J.d.nx, J.d.ny, Ex, Ey, J.S,
                                  1.0);
    PIC_LAUNCH_CHECK();
    return PIC_OK;
}

static void save_checkpoint(AdjImpl& J, int c, cudaStream_t st) {
    const size_t n = size_t(J.n);
    double* b = J.cp + size_t(c) * 4 * n;
    cudaMemcpyAsync(b, J.x, sizeof(double) * n, cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(b + n, J.y, sizeof(double) * n, cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(b + 2 * n, J.ux, sizeof(double) * n, cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(b + 3 * n, J.uy, sizeof(double) * n, cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(J.cp_phi + size_t(c) * J.G, J.phi, sizeof(double) * J.G, cudaMemcpyDeviceToDevice, st);
}

static void load_checkpoint(AdjImpl& J, int c, cudaStream_t st) {
    const size_t n = size_t(J.n);
    const double* b = J.cp + size_t(c) * 4 * n;
    cudaMemcpyAsync(J.x, b, sizeof(double) * n, cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(J.y, b + n, sizeof(double) * n, cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(J.ux, b + 2 * n, sizeof(double) * n, cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(J.uy, b + 3 * n, sizeof(double) * n, cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(J.phi, J.cp_phi + size_t(c) * J.G, sizeof(double) * J.G, cudaMemcpyDeviceToDevice, st);
}

static int adj_forward(AdjImpl& J, const double* h_V, double A, double* loss, cudaStream_t st) {
    const int pb = grid_blocks(J.n, 256), gb = grid_blocks(J.G, 256);
    const size_t n = size_t(J.n);
    if (J.d.nseg > 0) PIC_CUDA(cudaMemcpyAsync(J.V, h_V, sizeof(double) * J.d.nseg, cudaMemcpyHostToDevice, st));
    PIC_CUDA(cudaMemsetAsync(J.failures, 0, sizeof(int), st));
    PIC_CUDA(cudaMemsetAsync(J.red, 0, sizeof(double) * (2 + PIC_ADJ_MAX_SEGMENTS), st));
    if (!(J.frozen && J.have_forward))
        PIC_CUDA(cudaMemsetAsync(J.death, 0x7f, sizeof(int) * n, st));  // alive at every state
    PIC_CUDA(cudaMemcpyAsync(J.x, J.x0, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
    PIC_CUDA(cudaMemcpyAsync(J.y, J.y0, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
    PIC_CUDA(cudaMemcpyAsync(J.ux, J.vx0, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
    PIC_CUDA(cudaMemcpyAsync(J.uy, J.vy0, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
    PIC_CUDA(cudaMemsetAsync(J.phi, 0, sizeof(double) * J.G, st));
    k_ad_bc<<<gb, 256, 0, st>>>(J.phi, J.mask, J.segid, J.fixed, J.V, J.G);
    k_ad_perturb<<<pb, 256, 0, st>>>(J.ux, J.uy, J.dvx, J.dvy, A, J.n);
    PIC_LAUNCH_CHECK();
    // init: E_0 and the backward half kick
    PIC_TRY(field_of(J, 0, J.Ex, J.Ey, st));
    k_ad_kick<<<pb, 256, 0, st>>>(J.x, J.y, J.ux, J.uy, J.sp, J.death, 0, J.n, J.d.nx, J.d.ny, J.Ex, J.Ey, J.S, -0.5);
    PIC_LAUNCH_CHECK();
    const int C = J.d.checkpoint_every;
    for (int s = 0; s < J.d.steps; ++s) {
        if (s % C == 0) save_checkpoint(J, s / C, st);
        PIC_TRY(step_of(J, s, J.Ex, J.Ey, st));
    }
    // loss on the final density of the loss species
    k_ad_deposit<<<pb, 256, 0, st>>>(J.x, J.y, J.sp, J.death, J.d.steps, J.n, J.d.nx, J.d.ny, J.S, 1,
                                     J.d.loss_species, J.rho);
    k_ad_loss<<<gb, 256, 0, st>>>(J.rho, J.target, J.g, J.G, J.red);
    PIC_CUDA(cudaMemsetAsync(J.rho, 0, sizeof(double) * J.G, st));
    PIC_LAUNCH_CHECK();
    int failures = 0;
    PIC_CUDA(cudaMemcpyAsync(&J.loss, J.red, sizeof(double), cudaMemcpyDeviceToHost, st));
    PIC_CUDA(cudaMemcpyAsync(&failures, J.failures, sizeof(int), cudaMemcpyDeviceToHost, st));
    PIC_CUDA(cudaStreamSynchronize(st));
    J.A = A;
    J.have_forward = true;
    if (loss) *loss = J.loss;
    if (failures) return fail(PIC_ERR_NOT_CONVERGED, "%d Poisson solves did not converge", failures);
    return PIC_OK;
}

// Field part of a kick adjoint already scattered into lambda_E: lambda_phi,
// the adjoint solve and the electrode-potential gradient.
static int field_adj(AdjImpl& J, cudaStream_t st) {
    dim3 g;
    const int t = grid2(J, g);
    k_ad_gradT<<<g, t, 0, st>>>(J.lEx, J.lEy, J.mask, J.lphi, J.fa, J.d.nx, J.d.ny, J.d.dx, J.d.dy);
    k_ad_zero2<<<grid_blocks(J.G, 256), 256, 0, st>>>(J.lEx, J.lEy, J.G);
    PIC_LAUNCH_CHECK();
    PIC_TRY(mg_launch_graph(J.mga, J.mu, J.fa, J.d.tol, J.d.max_cycles, 0, st));
    if (J.d.tol > 0) k_ad_track<<<1, 1, 0, st>>>(mg_device_converged(J.mga), J.failures);
    if (J.d.nseg > 0)
        k_ad_dV<<<g, t, 0, st>>>(J.lphi, J.mu, J.mask, J.segid, J.d.nx, J.d.ny, 1.0 / (J.d.dx * J.d.dx),
                                 1.0 / (J.d.dy * J.d.dy), J.red + 2);
    PIC_LAUNCH_CHECK();
    return PIC_OK;
}

static int adj_backward(AdjImpl& J, double* h_dV, double* h_dA, cudaStream_t st) {
    if (!J.have_forward) return fail(PIC_ERR_BAD_ARG, "pic_adj_backward: run pic_adj_forward first");
    const int pb = grid_blocks(J.n, 256);
    const size_t n = size_t(J.n), G = size_t(J.G);
    const int N = J.d.steps, C = J.d.checkpoint_every;
    PIC_CUDA(cudaMemsetAsync(J.failures, 0, sizeof(int), st));
    PIC_CUDA(cudaMemsetAsync(J.red + 1, 0, sizeof(double) * (1 + PIC_ADJ_MAX_SEGMENTS), st));
    for (double* p : {J.lx, J.ly, J.lux, J.luy}) PIC_CUDA(cudaMemsetAsync(p, 0, sizeof(double) * n, st));
    for (double* p : {J.lEx, J.lEy, J.mu}) PIC_CUDA(cudaMemsetAsync(p, 0, sizeof(double) * G, st));
    // the loss gradient at the final state (positions are those the forward pass ended with)
    k_ad_loss_adj<<<pb, 256, 0, st>>>(J.x, J.y, J.sp, J.death, N, J.n, J.d.nx, J.d.ny, J.g, J.S, J.d.loss_species,
                                      J.lx, J.ly);
    PIC_LAUNCH_CHECK();
    for (int c = J.ncp - 1; c >= 0; --c) {
        const int a = c * C, b = std::min(N, a + C);
        // recompute states a+1 .. b, keeping positions and fields
        load_checkpoint(J, c, st);
        for (int s = a; s < b; ++s) {
            double* E = J.seg_E + size_t(s - a) * 2 * G;
            PIC_TRY(step_of(J, s, E, E + G, st));
            double* xy = J.seg_xy + size_t(s - a) * 2 * n;
            PIC_CUDA(cudaMemcpyAsync(xy, J.x, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
            PIC_CUDA(cudaMemcpyAsync(xy + n, J.y, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
        }
        // walk the segment back: step s takes state s to s+1
        for (int s = b - 1; s >= a; --s) {
            const double* E = J.seg_E + size_t(s - a) * 2 * G;
            const double* xy = J.seg_xy + size_t(s - a) * 2 * n;
            k_ad_kick_adj<<<pb, 256, 0, st>>>(xy, xy + n, J.sp, J.death, s + 1, J.n, J.d.nx, J.d.ny, E, E + G, J.S,
                                              1.0, J.lux, J.luy, J.lx, J.ly, J.lEx, J.lEy);
            PIC_LAUNCH_CHECK();
            PIC_TRY(field_adj(J, st));
            k_ad_dep_drift_adj<<<pb, 256, 0, st>>>(xy, xy + n, J.sp, J.death, s + 1, J.n, J.d.nx, J.d.ny, J.mu, J.S,
                                                   -1.0 / J.d.eps0, J.d.dt / J.d.dx, J.d.dt / J.d.dy, J.lx, J.ly,
                                                   J.lux, J.luy);
            PIC_LAUNCH_CHECK();
        }
    }
    // the init half kick at state 0 (positions x_0; its E_0 recomputed with the
    // forward's initial guess) and the perturbation amplitude
    PIC_CUDA(cudaMemcpyAsync(J.x, J.x0, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
    PIC_CUDA(cudaMemcpyAsync(J.y, J.y0, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
    load_checkpoint(J, 0, st);  // phi_0 (the positions of state 0 match x_0)
    PIC_TRY(field_of(J, 0, J.Ex, J.Ey, st));
    k_ad_kick_adj<<<pb, 256, 0, st>>>(J.x, J.y, J.sp, J.death, 0, J.n, J.d.nx, J.d.ny, J.Ex, J.Ey, J.S, -0.5, J.lux,
                                      J.luy, J.lx, J.ly, J.lEx, J.lEy);
    PIC_LAUNCH_CHECK();
    PIC_TRY(field_adj(J, st));
    k_ad_dot<<<pb, 256, 0, st>>>(J.lux, J.luy, J.dvx, J.dvy, J.n, J.red + 1);
    PIC_LAUNCH_CHECK();
    double out[2 + PIC_ADJ_MAX_SEGMENTS];
    int failures = 0;
    PIC_CUDA(cudaMemcpyAsync(out, J.red, sizeof out, cudaMemcpyDeviceToHost, st));
    PIC_CUDA(cudaMemcpyAsync(&failures, J.failures, sizeof(int), cudaMemcpyDeviceToHost, st));
    PIC_CUDA(cudaStreamSynchronize(st));
    if (h_dA) *h_dA = out[1];
    if (h_dV)
        for (int q = 0; q < J.d.nseg; ++q) h_dV[q] = out[2 + q];
    if (failures) return fail(PIC_ERR_NOT_CONVERGED, "%d Poisson solves did not converge", failures);
    return PIC_OK;
}

}  // namespace pic

struct pic_adj {
    pic::AdjImpl j;
};

using namespace pic;

extern "C" {

int pic_adj_create(const pic_adj_desc* desc, pic_adj** out) {
    clear_error();
    if (!out) return fail(PIC_ERR_BAD_ARG, "pic_adj_create: out is NULL");
    pic_adj* a = new pic_adj;
    const int st = adj_create(desc, a->j);
    if (st != PIC_OK) {
        adj_free(a->j);
        delete a;
        return st;
    }
    *out = a;
    return PIC_OK;
}

int pic_adj_destroy(pic_adj* a) {
    clear_error();
    if (!a) return PIC_OK;
    cudaDeviceSynchronize();
    adj_free(a->j);
    delete a;
    return PIC_OK;
}

int pic_adj_set_particles(pic_adj* a, int s, const double* d_x, const double* d_y, const double* d_vx,
                          const double* d_vy, const double* d_dvx, const double* d_dvy, void* stream) {
    clear_error();
    if (!a || s < 0 || s >= a->j.d.nspecies || !d_x || !d_y || !d_vx || !d_vy)
        return fail(PIC_ERR_BAD_ARG, "pic_adj_set_particles: bad arguments");
    AdjImpl& J = a->j;
    cudaStream_t st = as_stream(stream);
    const int b = J.first[s], n = J.first[s + 1] - b;
    if (n == 0) return PIC_OK;
    const double* src[6] = {d_x, d_y, d_vx, d_vy, d_dvx, d_dvy};
    double* dst[6] = {J.x0, J.y0, J.vx0, J.vy0, J.dvx, J.dvy};
    for (int q = 0; q < 6; ++q) {
        if (src[q]) PIC_CUDA(cudaMemcpyAsync(dst[q] + b, src[q], sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
        else PIC_CUDA(cudaMemsetAsync(dst[q] + b, 0, sizeof(double) * n, st));
    }
    J.have_forward = false;
    return PIC_OK;
}

int pic_adj_set_target(pic_adj* a, const double* d_target, void* stream) {
    clear_error();
    if (!a || !d_target) return fail(PIC_ERR_BAD_ARG, "pic_adj_set_target: bad arguments");
    PIC_CUDA(cudaMemcpyAsync(a->j.target, d_target, sizeof(double) * a->j.G, cudaMemcpyDeviceToDevice,
                             as_stream(stream)));
    a->j.have_forward = false;
    return PIC_OK;
}

int pic_adj_forward(pic_adj* a, const double* h_V, double A, double* loss, void* stream) {
    clear_error();
    if (!a || (a->j.d.nseg > 0 && !h_V)) return fail(PIC_ERR_BAD_ARG, "pic_adj_forward: bad arguments");
    return adj_forward(a->j, h_V, A, loss, as_stream(stream));
}

int pic_adj_backward(pic_adj* a, double* h_dV, double* h_dA, void* stream) {
    clear_error();
    if (!a) return fail(PIC_ERR_BAD_ARG, "pic_adj_backward: bad arguments");
    return adj_backward(a->j, h_dV, h_dA, as_stream(stream));
}

int pic_adj_freeze_absorption(pic_adj* a, int on) {
    clear_error();
    if (!a) return fail(PIC_ERR_BAD_ARG, "pic_adj_freeze_absorption: bad arguments");
    if (on && !a->j.have_forward) return fail(PIC_ERR_BAD_ARG, "pic_adj_freeze_absorption: run a forward pass first");
    a->j.frozen = on != 0;
    return PIC_OK;
}

int pic_adj_state(pic_adj* a, double** x, double** y, double** ux, double** uy, int** death, double** phi) {
    clear_error();
    if (!a) return fail(PIC_ERR_BAD_ARG, "pic_adj_state: bad arguments");
    AdjImpl& J = a->j;
    if (x) *x = J.x;
    if (y) *y = J.y;
    if (ux) *ux = J.ux;
    if (uy) *uy = J.uy;
    if (death) *death = J.death;
    if (phi) *phi = J.phi;
    return PIC_OK;
}

}  // extern "C"
