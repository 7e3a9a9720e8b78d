/*
 * Test infrastructure (oracle only): host driver for the reference's own
 * RawKernel sources.  ref_build.py extracts the kernel strings from the
 * reference's Python files, prepends cuda_shim.h and appends this file, and
 * compiles the result into oracle/_ref/libpicref.so.  Nothing here is part
 * of the shipped library: the tests use it to produce golden vectors and the
 * benchmark times it as the CPU baseline of the reference's time step.
 *
 * Every wrapper launches one reference kernel over the same 1-D / 2-D launch
 * shape the reference uses (block 256, or 16x16 for the 2-D kernels):
 *   K1  update_density_direct_cartesian   src/Grid.py:96-154, host part :246-294
 *   K3  update_E                          src/Grid.py:157-196
 *   K4  update_particle_velocity_direct   src/Particles.py:117-180
 *   K6  update_r_kernel                   src/Particles.py:251-264
 *   K7  update_particle_axis              src/Particles.py:267-280
 *   K9  sort_particles_sparse             src/Particles.py:595-617
 *   K10 gauss_seidel_red_black            src/multigrid.py:13-49
 *   K11 residual_kernel                   src/multigrid.py:52-81
 *   K12 restriction_kernel                src/multigrid.py:84-134
 *   K13 prolong_kernel                    src/multigrid.py:138-196
 *   K15 coarsen_bc_mask                   src/multigrid.py:235-274
 *   K22 compute_speeds_and_energies       src/MCC.py:7-30
 *   K23 interpolate_cross_sections        src/MCC.py:32-83
 * K11 and K13 read the mask array past its end for the tail threads of the
 * last block (src/multigrid.py:77,155); the wrappers hand them a copy padded
 * with one block of zeros so the emulation stays in bounds.
 */
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>
#include <omp.h>

thread_local ref_dim3 blockIdx;
thread_local ref_dim3 threadIdx;
thread_local ref_dim3 blockDim;
thread_local ref_dim3 gridDim;
int g_ref_parallel = 0;

namespace {

template <class F>
void launch_1d(long total, int block, F&& body) {
    const long grid = (total + block - 1) / block;
    auto run_block = [&](long b) {
        blockIdx = {unsigned(b), 0, 0};
        blockDim = {unsigned(block), 1, 1};
        gridDim = {unsigned(grid), 1, 1};
        for (int t = 0; t < block; ++t) {
            threadIdx = {unsigned(t), 0, 0};
            body();
        }
    };
    if (g_ref_parallel) {
#pragma omp parallel for schedule(static)
        for (long b = 0; b < grid; ++b) run_block(b);
    } else {
        for (long b = 0; b < grid; ++b) run_block(b);
    }
}

template <class F>
void launch_2d(int nx, int ny, int bx, int by, F&& body) {
    const int gx = (nx + bx - 1) / bx, gy = (ny + by - 1) / by;
    auto run_block = [&](long b) {
        blockIdx = {unsigned(b % gx), unsigned(b / gx), 0};
        blockDim = {unsigned(bx), unsigned(by), 1};
        gridDim = {unsigned(gx), unsigned(gy), 1};
        for (int ty = 0; ty < by; ++ty)
            for (int tx = 0; tx < bx; ++tx) {
                threadIdx = {unsigned(tx), unsigned(ty), 0};
                body();
            }
    };
    const long nb = long(gx) * gy;
    if (g_ref_parallel) {
#pragma omp parallel for schedule(static)
        for (long b = 0; b < nb; ++b) run_block(b);
    } else {
        for (long b = 0; b < nb; ++b) run_block(b);
    }
}

std::vector<int> padded_mask(const int* mask, long n) {
    std::vector<int> m(n + 256, 0);
    std::memcpy(m.data(), mask, sizeof(int) * n);
    return m;
}

double sum_sq(const double* v, long n) {
    double s = 0.0;
    if (g_ref_parallel) {
#pragma omp parallel for reduction(+ : s) schedule(static)
        for (long i = 0; i < n; ++i) s += v[i] * v[i];
    } else {
        for (long i = 0; i < n; ++i) s += v[i] * v[i];
    }
    return s;
}

inline double ref_uniform(unsigned long long seed, unsigned long long i) {
    /* splitmix64 of (seed, index): stands in for CuPy's unseeded cp.random.random */
    unsigned long long z = seed + (i + 1) * 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return double(z >> 11) * (1.0 / 9007199254740992.0);
}

/* Runs body(i) for i in [0, n), over OpenMP threads when the baseline is parallel. */
template <class F>
void ref_for(long n, F&& body) {
    if (g_ref_parallel) {
#pragma omp parallel for schedule(static)
        for (long i = 0; i < n; ++i) body(i);
    } else {
        for (long i = 0; i < n; ++i) body(i);
    }
}

}  // namespace

extern "C" {

void ref_set_parallel(int on, int threads) {
    g_ref_parallel = on;
    if (threads > 0) omp_set_num_threads(threads);
}

int ref_max_threads(void) { return omp_get_max_threads(); }

/* Grid2D.update_density, Cartesian branch (src/Grid.py:246-294). */
void ref_update_density(double* rho, const double* R, const int* part_type, const double* q_type,
                        double np2c, double dx, double dy, int m, int n, int last_alive) {
    std::memset(rho, 0, sizeof(double) * long(m) * n);
    launch_1d(last_alive, 256, [&] {
        update_density_direct_cartesian(rho, R, part_type, q_type, np2c, dx, dy, m, n, last_alive);
    });
    const double inv = dx * dy;
    for (long i = 0; i < long(m) * n; ++i) rho[i] /= inv;
}

/* Grid2D.update_E (src/Grid.py:232-243). */
void ref_update_E(const double* phi, double* E, int nx, int ny, double dx, double dy) {
    launch_1d(long(nx) * ny, 256, [&] { update_E(phi, E, nx, ny, dx, dy); });
}

/* Particles2D.update_V, Cartesian branch (src/Particles.py:378-410). */
void ref_update_V(double* V, const double* R, const double* Ex, const double* Ey, const int* part_type,
                  const double* q_type, const double* m_type_inv, double dt, double dx, double dy, int m,
                  int n, int last_alive) {
    launch_1d(last_alive, 256, [&] {
        update_particle_velocity_direct(V, R, Ex, Ey, part_type, q_type, m_type_inv, dt, dx, dy, m, n,
                                        last_alive);
    });
}

/* Particles2D.update_R (src/Particles.py:359-367). */
void ref_update_R(double* R_old, double* R, double* V, double dt, int last_alive) {
    launch_1d(last_alive, 256, [&] { update_r_kernel(R_old, R, V, dt, last_alive); });
}

/* Particles2D.update_axis (src/Particles.py:369-376). */
void ref_update_axis(double* R, double* V, int last_alive) {
    launch_1d(last_alive, 256, [&] { update_particle_axis(R, V, last_alive); });
}

/* The scatter step of Particles2D.sort_particles_sparse (src/Particles.py:595-617). */
void ref_sort_scatter(const int* cell_indices, const int* cell_to_active_map, const int* cell_positions,
                      int* temp_positions, int* sorted_indices, int num_particles) {
    launch_1d(num_particles, 256, [&] {
        sort_particles_sparse(cell_indices, cell_to_active_map, cell_positions, temp_positions,
                              sorted_indices, num_particles);
    });
}

/* MultigridSolver.smooth, one colour (src/multigrid.py:314-333). */
void ref_gauss_seidel(double* phi, const double* rho, const int* bc_mask, double h2, double omega, int nx,
                      int ny, int is_red) {
    launch_1d(long(nx) * ny, 256,
              [&] { gauss_seidel_red_black(phi, rho, bc_mask, h2, omega, nx, ny, is_red); });
}

/* MultigridSolver.residual (src/multigrid.py:337-345). */
void ref_residual(const double* phi, const double* rho, double* res, const int* bc_mask, double inv_h2,
                  int nx, int ny) {
    std::vector<int> mask = padded_mask(bc_mask, long(nx) * ny);
    launch_1d(long(nx) * ny, 256, [&] { residual_kernel(phi, rho, res, mask.data(), inv_h2, nx, ny); });
}

/* MultigridSolver.restrict (src/multigrid.py:348-362). */
void ref_restrict(const double* fine, double* coarse, const int* bc_mask, int nx, int ny) {
    const int nxc = (nx + 1) / 2, nyc = (ny + 1) / 2;
    launch_2d(nxc, nyc, 16, 16, [&] { restriction_kernel(fine, coarse, bc_mask, nx, ny, nxc, nyc); });
}

/* MultigridSolver.prolong (src/multigrid.py:365-374). */
void ref_prolong(double* fine, const double* coarse, const int* bc_mask_fine, int nxc, int nyc) {
    const int nxf = 2 * (nxc - 1) + 1, nyf = 2 * (nyc - 1) + 1;
    std::vector<int> mask = padded_mask(bc_mask_fine, long(nxf) * nyf);
    launch_1d(long(nxf) * nyf, 256, [&] { prolong_kernel(fine, coarse, mask.data(), nxc, nyc, nxf); });
}

/* MultigridSolver._coarsen_bc_mask (src/multigrid.py:432-443). */
void ref_coarsen_bc_mask(const int* fine, int* coarse, int nxf, int nyf, int nxc, int nyc) {
    launch_2d(nxc, nyc, 16, 16, [&] { coarsen_bc_mask(fine, coarse, nxf, nyf, nxc, nyc); });
}

/* MCC.compute_speeds_and_energies kernel (src/MCC.py:7-30, called at :118-121). */
void ref_speeds_energies(const double* vx, const double* vy, const double* vz, double* speeds,
                         double* energies, const int* type, const double* me, int N) {
    launch_1d(N, 256, [&] { compute_speeds_and_energies(vx, vy, vz, speeds, energies, type, me, N); });
}

/* MCC.interp_table kernel (src/MCC.py:32-83, called at :150-170). */
void ref_interp_cross_sections(const double* energies, const double* xs_energy, const double* xs_values,
                               const bool* mcc_mask, double* output, int xs_len, int N) {
    launch_1d(N, 256, [&] {
        interpolate_cross_sections(energies, xs_energy, xs_values, mcc_mask, output, xs_len, N);
    });
}

/* ------------------------------------------------------------------------
 * The reference's multigrid solve driven through its own kernels
 * (src/multigrid.py:378-455), with the two fixes without which it cannot
 * converge: the right-hand side carries no extra dx^2 (the kernels apply h^2
 * themselves) and every level uses the mask meaning each kernel expects
 * (K10/K11: 1 = Dirichlet; K13/K15: 1 = free node).
 * ---------------------------------------------------------------------- */
struct ref_mg {
    int n, levels;
    double h, omega;
    std::vector<std::vector<double>> phi, rhs, res;
    std::vector<std::vector<int>> bc, freem;
    std::vector<double> res0;
};

ref_mg* ref_mg_create(const int* bc_lookup, int n, double h, int levels, double omega) {
    ref_mg* mg = new ref_mg;
    mg->n = n;
    mg->levels = levels;
    mg->h = h;
    mg->omega = omega;
    mg->res0.assign(long(n) * n, 0.0);
    for (int l = 0; l < levels; ++l) {
        const int nl = (n + (1 << l) - 1) >> l;
        mg->phi.emplace_back(long(nl) * nl, 0.0);
        mg->rhs.emplace_back(long(nl) * nl, 0.0);
        mg->res.emplace_back(long(nl) * nl, 0.0);
        mg->bc.emplace_back(long(nl) * nl, 0);
        mg->freem.emplace_back(long(nl) * nl, 0);
    }
    for (long i = 0; i < long(n) * n; ++i) {
        mg->bc[0][i] = bc_lookup[i] ? 1 : 0;
        mg->freem[0][i] = 1 - mg->bc[0][i];
    }
    for (int l = 1; l < levels; ++l) {
        const int nf = (n + (1 << (l - 1)) - 1) >> (l - 1), nc = (n + (1 << l) - 1) >> l;
        ref_coarsen_bc_mask(mg->freem[l - 1].data(), mg->freem[l].data(), nf, nf, nc, nc);
        for (long i = 0; i < long(nc) * nc; ++i) mg->bc[l][i] = 1 - mg->freem[l][i];
    }
    return mg;
}

void ref_mg_destroy(ref_mg* mg) { delete mg; }

static void ref_mg_smooth(ref_mg* mg, double* phi, const double* rhs, const int* bc, int n, double h,
                          int iters) {
    for (int it = 0; it < iters; ++it) {
        ref_gauss_seidel(phi, rhs, bc, h * h, mg->omega, n, n, 1);
        ref_gauss_seidel(phi, rhs, bc, h * h, mg->omega, n, n, 0);
    }
}

static void ref_mg_vcycle(ref_mg* mg, double* phi, const double* rhs, int smooth_iter, int solve_iter) {
    const int L = mg->levels;
    int n = mg->n;
    double h = mg->h;
    std::vector<double*> P(L), F(L);
    P[0] = phi;
    F[0] = const_cast<double*>(rhs);
    for (int l = 1; l < L; ++l) {
        P[l] = mg->phi[l].data();
        F[l] = mg->rhs[l].data();
    }
    for (int l = 0; l < L - 1; ++l) {
        ref_mg_smooth(mg, P[l], F[l], mg->bc[l].data(), n, h, smooth_iter);
        ref_residual(P[l], F[l], mg->res[l].data(), mg->bc[l].data(), 1.0 / (h * h), n, n);
        ref_restrict(mg->res[l].data(), F[l + 1], mg->bc[l].data(), n, n);
        std::fill(mg->phi[l + 1].begin(), mg->phi[l + 1].end(), 0.0);
        n = (n + 1) / 2;
        h *= 2;
    }
    ref_mg_smooth(mg, P[L - 1], F[L - 1], mg->bc[L - 1].data(), n, h, solve_iter);
    for (int l = L - 2; l >= 0; --l) {
        const int nc = n;
        n = 2 * n - 1;
        h /= 2;
        ref_prolong(P[l], P[l + 1], mg->freem[l].data(), nc, nc);
        ref_mg_smooth(mg, P[l], F[l], mg->bc[l].data(), n, h, smooth_iter);
    }
}

/* Returns the number of cycles run; *rel_res receives the last relative residual. */
int ref_mg_solve(ref_mg* mg, double* phi, const double* rhs, double tol, int smooth_iter, int solve_iter,
                 int max_cycles, double* rel_res) {
    const long N = long(mg->n) * mg->n;
    const double rhs_norm = std::sqrt(sum_sq(rhs, N));
    int it = 0;
    double rel = 0.0;
    for (it = 0; it < max_cycles; ++it) {
        ref_residual(phi, rhs, mg->res0.data(), mg->bc[0].data(), 1.0 / (mg->h * mg->h), mg->n, mg->n);
        rel = std::sqrt(sum_sq(mg->res0.data(), N)) / rhs_norm;
        if (rel < tol) break;
        ref_mg_vcycle(mg, phi, rhs, smooth_iter, solve_iter);
    }
    if (rel_res) *rel_res = rel;
    return it;
}

/* ------------------------------------------------------------------------
 * One time step of the reference (SimulationManager._step,
 * src/simulation.py:640-660) on the reference's AoS FP64 arrays:
 * update_R, update_axis, update_density, Solver.solve (multigrid branch,
 * src/Solvers.py:269-299 with the RHS scaling fix), update_E, update_V and
 * the part of MCC.null_collision_method that runs before its early return
 * (src/MCC.py:328-394, elastic table only).
 * ---------------------------------------------------------------------- */
struct ref_state {
    int m, n, last_alive;
    double dx, dy, dt, np2c, eps0;
    double *R, *R_old, *V;
    int* part_type;
    const double *q_type, *m_type, *m_type_inv;
    double *rho, *b, *phi, *E;
    const int* bc_idx;
    const double* bc_val;
    int n_bc;
    ref_mg* mg;
    double tol;
    int smooth_iter, solve_iter, max_cycles;
    /* MCC */
    int do_mcc;
    double gas_density;
    const double *xs_energy, *xs_sigma;
    int xs_len;
    int mcc_species;
    double *speeds, *energies, *sigma, *rand_buf;
    unsigned char* mcc_mask; /* bool */
    unsigned long long rng;
    /* outputs */
    int last_cycles;
    double last_rel;
    long long collided;
};

void ref_step(ref_state* s) {
    const long G = long(s->m) * s->n;
    ref_update_R(s->R_old, s->R, s->V, s->dt, s->last_alive);
    ref_update_axis(s->R, s->V, s->last_alive);
    ref_update_density(s->rho, s->R, s->part_type, s->q_type, s->np2c, s->dx, s->dy, s->m, s->n,
                       s->last_alive);
    const double eps0_1 = 1.0 / s->eps0;
    ref_for(G, [&](long i) { s->b[i] = -s->rho[i] * eps0_1; });
    for (int k = 0; k < s->n_bc; ++k) s->b[s->bc_idx[k]] = s->bc_val[k];
    double rel = 0.0;
    s->last_cycles = ref_mg_solve(s->mg, s->phi, s->b, s->tol, s->smooth_iter, s->solve_iter,
                                  s->max_cycles, &rel);
    s->last_rel = rel;
    ref_update_E(s->phi, s->E, s->m, s->n, s->dx, s->dy);
    ref_update_V(s->V, s->R, s->E, s->E + G, s->part_type, s->q_type, s->m_type_inv, s->dt, s->dx, s->dy,
                 s->m, s->n, s->last_alive);
    if (!s->do_mcc) return;
    const int N = s->last_alive;
    /* compute_speeds_and_energies passes V[0], V[1], V[2] (rows of the (N,3) array) */
    ref_speeds_energies(s->V, s->V + 3, s->V + 6, s->speeds, s->energies, s->part_type, s->m_type, N);
    ref_for(N, [&](long i) { s->mcc_mask[i] = (s->part_type[i] == s->mcc_species); });
    ref_interp_cross_sections(s->energies, s->xs_energy, s->xs_sigma, reinterpret_cast<bool*>(s->mcc_mask),
                              s->sigma, s->xs_len, N);
    ref_for(N, [&](long i) {
        s->sigma[i] = s->gas_density * s->sigma[i] * s->speeds[i] * (s->mcc_mask[i] ? 1.0 : 0.0);
    });
    double nu_max = 0.0;
    for (int i = 0; i < N; ++i) nu_max = s->sigma[i] > nu_max ? s->sigma[i] : nu_max;
    long long hits = 0;
    const unsigned long long seed = s->rng++;
    if (g_ref_parallel) {
#pragma omp parallel for reduction(+ : hits) schedule(static)
        for (long i = 0; i < N; ++i) hits += (ref_uniform(seed, i) < s->sigma[i] / nu_max) && s->mcc_mask[i];
    } else {
        for (long i = 0; i < N; ++i) hits += (ref_uniform(seed, i) < s->sigma[i] / nu_max) && s->mcc_mask[i];
    }
    s->collided = hits;
}

}  // extern "C"
