// Stateless particle and grid operators: the drop-in kernels behind
// Particles2D.update_R / update_V, Grid2D.update_density / update_E and the
// Poisson right-hand side.  Positions are float32 grid units, velocities m/s.
#include <cstring>
#include <string>

#include "common.cuh"

namespace pic {

static thread_local std::string g_last_error;

int fail(int code, const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

void clear_error() { g_last_error.clear(); }

int num_sms() {
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (sms <= 0) sms = 148;
    }
    return sms;
}

int raise_smem_limit(const void* kernel, size_t bytes) {
    cudaFuncAttributes a{};
    PIC_CUDA(cudaFuncGetAttributes(&a, kernel));
    if (size_t(a.maxDynamicSharedSizeBytes) < bytes)
        PIC_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes)));
    return PIC_OK;
}

// ---- kernels -------------------------------------------------------------------

__global__ void k_update_R(float* __restrict__ x, float* __restrict__ y, const float* __restrict__ vx,
                           const float* __restrict__ vy, int n, float dtdx, float dtdy, float* __restrict__ x_old,
                           float* __restrict__ y_old) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        const float px = x[p], py = y[p];
        if (x_old) x_old[p] = px;
        if (y_old) y_old[p] = py;
        if (!is_live(px)) continue;
        x[p] = __fmaf_rn(vx[p], dtdx, px);
        y[p] = __fmaf_rn(vy[p], dtdy, py);
    }
}

__global__ void k_absorb(float* __restrict__ x, float* __restrict__ y, int n, float X, float Y,
                         unsigned long long* __restrict__ absorbed) {
    __shared__ unsigned int block_count;
    if (threadIdx.x == 0) block_count = 0;
    __syncthreads();
    unsigned int mine = 0;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        const float px = x[p], py = y[p];
        if (!is_live(px)) continue;
        if (!(px >= 0.0f && px <= X && py >= 0.0f && py <= Y)) {
            x[p] = __int_as_float(0x7fc00000);
            y[p] = __int_as_float(0x7fc00000);
            ++mine;
        }
    }
    mine = __reduce_add_sync(0xffffffffu, mine);
    if ((threadIdx.x & 31) == 0 && mine) atomicAdd(&block_count, mine);
    __syncthreads();
    if (threadIdx.x == 0 && block_count && absorbed) atomicAdd(absorbed, (unsigned long long)block_count);
}

__global__ void k_update_V(const float* __restrict__ x, const float* __restrict__ y, float* __restrict__ vx,
                           float* __restrict__ vy, int n, const float* __restrict__ Ex,
                           const float* __restrict__ Ey, int nx, int ny, float kq) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        const float px = x[p];
        if (!is_live(px)) continue;
        const Cic c = cic_weights(px, y[p], nx, ny);
        const int k00 = c.j0 * nx + c.i0, k10 = c.j0 * nx + c.i1, k01 = c.j1 * nx + c.i0, k11 = c.j1 * nx + c.i1;
        const float ex = cic_interp(c, __ldg(Ex + k00), __ldg(Ex + k10), __ldg(Ex + k01), __ldg(Ex + k11));
        const float ey = cic_interp(c, __ldg(Ey + k00), __ldg(Ey + k10), __ldg(Ey + k01), __ldg(Ey + k11));
        vx[p] = __fmaf_rn(kq, ex, vx[p]);
        vy[p] = __fmaf_rn(kq, ey, vy[p]);
    }
}

__global__ void k_deposit(const float* __restrict__ x, const float* __restrict__ y, int n, float scale,
                          float* __restrict__ rho, int nx, int ny) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        const float px = x[p];
        if (!is_live(px)) continue;
        const Cic c = cic_weights(px, y[p], nx, ny);
        atomicAdd(rho + c.j0 * nx + c.i0, __fmul_rn(scale, c.w00));
        atomicAdd(rho + c.j0 * nx + c.i1, __fmul_rn(scale, c.w10));
        atomicAdd(rho + c.j1 * nx + c.i0, __fmul_rn(scale, c.w01));
        atomicAdd(rho + c.j1 * nx + c.i1, __fmul_rn(scale, c.w11));
    }
}

// E = -grad(phi) (src/Grid.py:167-194), FP64 arithmetic, rounded once to float.
// axis: r-z geometry, where row 0 is the axis and E_r vanishes there by symmetry.
__device__ __forceinline__ double2 grad_node(const double* __restrict__ phi, int i, int j, int nx, int ny,
                                             double dx, double dy, bool axis) {
    const long k = long(j) * nx + i;
    double ex, ey;
    if (i > 0 && i < nx - 1) ex = -(phi[k + 1] - phi[k - 1]) / (2.0 * dx);
    else if (i == 0) ex = -(phi[k + 1] - phi[k]) / dx;
    else ex = -(phi[k] - phi[k - 1]) / dx;
    if (j > 0 && j < ny - 1) ey = -(phi[k + nx] - phi[k - nx]) / (2.0 * dy);
    else if (j == 0) ey = axis ? 0.0 : -(phi[k + nx] - phi[k]) / dy;
    else ey = -(phi[k] - phi[k - nx]) / dy;
    return make_double2(ex, ey);
}

// E2 (when given) is the interleaved (Ex, Ey) copy the particle pass
// gathers from, with rows `ep` nodes apart.
__global__ void k_update_E(const double* __restrict__ phi, float* __restrict__ Ex, float* __restrict__ Ey,
                           float2* __restrict__ E2, int ep, int nx, int ny, double dx, double dy, int axis) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (i >= nx) return;
    const double2 e = grad_node(phi, i, j, nx, ny, dx, dy, axis != 0);
    const long k = long(j) * nx + i;
    const float fx = float(e.x), fy = float(e.y);
    if (Ex) Ex[k] = fx;
    if (Ey) Ey[k] = fy;
    if (E2) E2[long(j) * ep + i] = make_float2(fx, fy);
}

// rho -> f = -rho/eps0 on free nodes.  With phi_prev given, also replaces the
// initial guess by its linear extrapolation in time, phi <- 2 phi - phi_prev,
// on free nodes and keeps the old phi in phi_prev.  With rowf (r-z geometry),
// the deposited charge of row j (per dx*dy) becomes a charge density first:
// rho *= rowf[j] = dx*dy / V_j; the snapshot holds the density.
__global__ void k_form_rhs(const float* __restrict__ rho, const uint8_t* __restrict__ dirichlet, double neg_inv_eps0,
                           double* __restrict__ f, float* __restrict__ rho_snapshot, float* __restrict__ rho_zero,
                           double* __restrict__ phi, double* __restrict__ phi_prev, long G,
                           const double* __restrict__ rowf, int nx) {
    for (long k = blockIdx.x * long(blockDim.x) + threadIdx.x; k < G; k += long(gridDim.x) * blockDim.x) {
        float r = rho[k];
        double rd = double(r);
        if (rowf) {
            rd *= rowf[int(k) / nx];
            r = float(rd);
        }
        const bool dir = dirichlet[k] != 0;
        f[k] = dir ? 0.0 : rd * neg_inv_eps0;
        if (rho_snapshot) rho_snapshot[k] = r;
        if (rho_zero) rho_zero[k] = 0.0f;
        if (phi_prev && !dir) {
            const double p = phi[k];
            phi[k] = 2.0 * p - phi_prev[k];
            phi_prev[k] = p;
        }
    }
}

// Deposited charge (per dx*dy) -> r-z charge density, rho_j *= dx*dy / V_j.
__global__ void k_rz_density(float* __restrict__ rho, int nx, int ny, double dy, long G) {
    for (long k = blockIdx.x * long(blockDim.x) + threadIdx.x; k < G; k += long(gridDim.x) * blockDim.x)
        rho[k] = float(double(rho[k]) * (1.0 / rz_row_volume(int(k / nx), ny, dy)));
}

// The r-z drift of every live particle (drift_rz); dead slots are skipped.
__global__ void k_update_R_rz(float* __restrict__ x, float* __restrict__ y, const float* __restrict__ vx,
                              float* __restrict__ vy, float* __restrict__ vz, int n, float dtdx, float dtdy) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        float px = x[p], py = y[p];
        if (!is_live(px)) continue;
        float v1 = vy[p], v2 = vz[p];
        drift_rz(px, py, vx[p], v1, v2, dtdx, dtdy);
        x[p] = px;
        y[p] = py;
        vy[p] = v1;
        vz[p] = v2;
    }
}

int grid_blocks(long n, int threads) {
    long b = (n + threads - 1) / threads;
    const long cap = long(num_sms()) * 16;
    if (b > cap) b = cap;
    if (b < 1) b = 1;
    return int(b);
}

int launch_update_E(const double* phi, float* Ex, float* Ey, float2* E2, int ep, int nx, int ny, double dx,
                    double dy, cudaStream_t st, bool axis) {
    dim3 grid(div_up(nx, 128), ny);
    k_update_E<<<grid, 128, 0, st>>>(phi, Ex, Ey, E2, ep, nx, ny, dx, dy, axis ? 1 : 0);
    PIC_LAUNCH_CHECK();
    return PIC_OK;
}

int launch_form_rhs(const float* rho, const uint8_t* dirichlet, double eps0, double* f, float* snapshot,
                    float* zero, double* phi, double* phi_prev, long G, cudaStream_t st, const double* rowf, int nx) {
    k_form_rhs<<<grid_blocks(G, 256), 256, 0, st>>>(rho, dirichlet, -1.0 / eps0, f, snapshot, zero, phi, phi_prev, G,
                                                    rowf, nx);
    PIC_LAUNCH_CHECK();
    return PIC_OK;
}

}  // namespace pic

using namespace pic;

extern "C" {

int pic_abi_version(void) { return PIC_ABI_VERSION; }

const char* pic_last_error(void) { return g_last_error.c_str(); }

int pic_update_R(float* d_x, float* d_y, const float* d_vx, const float* d_vy, int n, float dtdx, float dtdy,
                 float* d_x_old, float* d_y_old, void* stream) {
    clear_error();
    if (n < 0 || (n > 0 && (!d_x || !d_y || !d_vx || !d_vy))) return fail(PIC_ERR_BAD_ARG, "pic_update_R: bad arguments");
    if (n == 0) return PIC_OK;
    k_update_R<<<grid_blocks(n, 256), 256, 0, as_stream(stream)>>>(d_x, d_y, d_vx, d_vy, n, dtdx, dtdy, d_x_old,
                                                                  d_y_old);
    PIC_LAUNCH_CHECK();
    return PIC_OK;
}

int pic_absorb(float* d_x, float* d_y, int n, int nx, int ny, unsigned long long* d_absorbed, void* stream) {
    clear_error();
    if (n < 0 || nx < 2 || ny < 2 || (n > 0 && (!d_x || !d_y))) return fail(PIC_ERR_BAD_ARG, "pic_absorb: bad arguments");
    if (n == 0) return PIC_OK;
    k_absorb<<<grid_blocks(n, 256), 256, 0, as_stream(stream)>>>(d_x, d_y, n, float(nx - 1), float(ny - 1),
                                                                d_absorbed);
    PIC_LAUNCH_CHECK();
    return PIC_OK;
}

int pic_update_V(const float* d_x, const float* d_y, float* d_vx, float* d_vy, int n, const float* d_Ex,
                 const float* d_Ey, int nx, int ny, float kq, void* stream) {
    clear_error();
    if (n < 0 || nx < 2 || ny < 2 || (n > 0 && (!d_x || !d_y || !d_vx || !d_vy || !d_Ex || !d_Ey)))
        return fail(PIC_ERR_BAD_ARG, "pic_update_V: bad arguments");
    if (n == 0) return PIC_OK;
    k_update_V<<<grid_blocks(n, 256), 256, 0, as_stream(stream)>>>(d_x, d_y, d_vx, d_vy, n, d_Ex, d_Ey, nx, ny, kq);
    PIC_LAUNCH_CHECK();
    return PIC_OK;
}

int pic_deposit(const float* d_x, const float* d_y, int n, float scale, float* d_rho, int nx, int ny, void* stream) {
    clear_error();
    if (n < 0 || nx < 2 || ny < 2 || !d_rho || (n > 0 && (!d_x || !d_y)))
        return fail(PIC_ERR_BAD_ARG, "pic_deposit: bad arguments");
    if (n == 0) return PIC_OK;
    k_deposit<<<grid_blocks(n, 256), 256, 0, as_stream(stream)>>>(d_x, d_y, n, scale, d_rho, nx, ny);
    PIC_LAUNCH_CHECK();
    return PIC_OK;
}

int pic_update_E(const double* d_phi, float* d_Ex, float* d_Ey, int nx, int ny, double dx, double dy,
                 void* stream) {
    clear_error();
    if (!d_phi || !d_Ex || !d_Ey || nx < 2 || ny < 2 || !(dx > 0) || !(dy > 0))
        return fail(PIC_ERR_BAD_ARG, "pic_update_E: bad arguments");
    return launch_update_E(d_phi, d_Ex, d_Ey, nullptr, nx, nx, ny, dx, dy, as_stream(stream), false);
}

int pic_update_E_rz(const double* d_phi, float* d_Ex, float* d_Ey, int nx, int ny, double dx, double dy,
                    void* stream) {
    clear_error();
    if (!d_phi || !d_Ex || !d_Ey || nx < 2 || ny < 2 || !(dx > 0) || !(dy > 0))
        return fail(PIC_ERR_BAD_ARG, "pic_update_E_rz: bad arguments");
    return launch_update_E(d_phi, d_Ex, d_Ey, nullptr, nx, nx, ny, dx, dy, as_stream(stream), true);
}

int pic_rz_density(float* d_rho, int nx, int ny, double dy, void* stream) {
    clear_error();
    if (!d_rho || nx < 2 || ny < 2 || !(dy > 0)) return fail(PIC_ERR_BAD_ARG, "pic_rz_density: bad arguments");
    const long G = long(nx) * ny;
    k_rz_density<<<grid_blocks(G, 256), 256, 0, as_stream(stream)>>>(d_rho, nx, ny, dy, G);
    PIC_LAUNCH_CHECK();
    return PIC_OK;
}

int pic_update_R_rz(float* d_x, float* d_y, const float* d_vx, float* d_vy, float* d_vz, int n, float dtdx,
                    float dtdy, void* stream) {
    clear_error();
    if (n < 0 || (n > 0 && (!d_x || !d_y || !d_vx || !d_vy || !d_vz)))
        return fail(PIC_ERR_BAD_ARG, "pic_update_R_rz: bad arguments");
    if (n == 0) return PIC_OK;
    k_update_R_rz<<<grid_blocks(n, 256), 256, 0, as_stream(stream)>>>(d_x, d_y, d_vx, d_vy, d_vz, n, dtdx, dtdy);
    PIC_LAUNCH_CHECK();
    return PIC_OK;
}

int pic_form_rhs(const float* d_rho, const uint8_t* d_dirichlet, double eps0, double* d_f, int nx, int ny,
                 void* stream) {
    clear_error();
    if (!d_rho || !d_dirichlet || !d_f || nx < 2 || ny < 2 || !(eps0 > 0))
        return fail(PIC_ERR_BAD_ARG, "pic_form_rhs: bad arguments");
    return launch_form_rhs(d_rho, d_dirichlet, eps0, d_f, nullptr, nullptr, nullptr, nullptr, long(nx) * ny,
                           as_stream(stream), nullptr, 0);
}

}  // extern "C"
