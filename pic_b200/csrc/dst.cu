// Fast Poisson solve by discrete sine transforms, for grids whose Dirichlet
// nodes are exactly the four edges (the reference's poisson_fft_dirichlet,
// src/FFT.py:10-64, and poisson_solver_dirichlet_2d, :102-121).
//
// lap(phi) = f with the 5-point operator and phi given on the edges: the edge
// values move to the right-hand side of the interior nodes next to them
// (f - lap(phi_edges)), the interior is diagonalised by DST-I in x and y,
// divided by the operator's eigenvalues, and transformed back:
//
//   phi = (2/Mx)(2/My) Sx Sy [ (Sy Sx f') / lambda ],   Mx = nx - 1, My = ny - 1,
//   lambda(k, l) = -cx 4 sin^2(pi k / 2Mx) - cy 4 sin^2(pi l / 2My).
//
// A DST-I of length N = M - 1 is read off the FFT of the odd extension of
// length 2M, which is purely imaginary: FFT(y)_k = -2i X_k.  Two rows share
// one complex FFT (the first as the real part, the second as the imaginary
// part): Z_k = -2i A_k + 2 B_k, so A_k = -Im Z_k / 2 and B_k = Re Z_k / 2.
// M must be a power of two (grids of 2^q + 1 nodes, as the multigrid's).
//
// Three kernels, each one complex FFT of 2M points per CTA in shared memory
// (radix-2, bit-reversed load, FP64):
//   k_dst_rows:  interior rows, forward along x, stored transposed, T[k][j];
//   k_dst_cols:  rows of T, forward along y, divide, inverse along y, in place;
//   k_dst_back:  columns of T, inverse along x, written to the interior of phi.
#include <cmath>
#include <vector>

#include "common.cuh"

namespace pic {

constexpr int kDstThreads = 256;

struct DstDev {
    int nx, ny;    // nodes
    int Nx, Ny;    // interior nodes per direction
    int Mx, My;    // Nx + 1, Ny + 1 (powers of two)
    int px, py;    // log2(2 Mx), log2(2 My)
    double cx, cy;
    const double2* twx;  // e^{-2 pi i m / (2 Mx)}, m < Mx
    const double2* twy;
    const double* lamx;  // 4 cx sin^2(pi k / 2Mx), k = 0..Mx
    const double* lamy;
    double* T;           // Nx * Ny, T[(k-1) * Ny + (j-1)]
};

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

__device__ __forceinline__ unsigned bitrev(unsigned n, int p) { return __brev(n) >> (32 - p); }

// In-place radix-2 decimation-in-time FFT of L = 2^p points in shared memory
// (input in bit-reversed order, output in natural order); tw[m] = e^{-2 pi i m / L}.
__device__ void fft_smem(double2* s, int p, const double2* tw) {
    const int L = 1 << p;
    for (int h = 1, st = L >> 1; h < L; h <<= 1, st >>= 1) {
        for (int b = threadIdx.x; b < (L >> 1); b += blockDim.x) {
            const int pos = b & (h - 1);
            const int i0 = ((b - pos) << 1) + pos, i1 = i0 + h;
            const double2 w = tw[pos * st];
            const double2 a = s[i0], t = cmul(w, s[i1]);
            s[i0] = make_double2(a.x + t.x, a.y + t.y);
            s[i1] = make_double2(a.x - t.x, a.y - t.y);
        }
        __syncthreads();
    }
}

// Writes the odd extension of two real rows a[1..N], b[1..N] (M = N + 1) into
// s in bit-reversed order: z_n = a_n + i b_n, z_0 = z_M = 0, z_{2M-n} = -z_n.
template <class A, class B>
__device__ void load_odd_pair(double2* s, int p, int M, A a, B b) {
    const int L = 2 * M;
    for (int n = threadIdx.x; n <= M; n += blockDim.x) {
        double2 v = make_double2(0.0, 0.0);
        if (n > 0 && n < M) v = make_double2(a(n), b(n));
        s[bitrev(unsigned(n), p)] = v;
        if (n > 0 && n < M) s[bitrev(unsigned(L - n), p)] = make_double2(-v.x, -v.y);
    }
}

// Copies the twiddles e^{-2 pi i m / L}, m < L/2, to shared memory.
__device__ void load_twiddles(double2* tw_s, const double2* tw, int p) {
    for (int m = threadIdx.x; m < (1 << (p - 1)); m += blockDim.x) tw_s[m] = tw[m];
}

// Interior rows (j_a, j_b) = (1 + 2 blockIdx.x, 2 + 2 blockIdx.x): forward DST
// along x of f minus the edge terms, stored transposed in T.
__global__ void __launch_bounds__(kDstThreads) k_dst_rows(DstDev D, const double* __restrict__ phi,
                                                          const double* __restrict__ f) {
    extern __shared__ __align__(16) unsigned char smem[];
    double2* s = reinterpret_cast<double2*>(smem);
    double2* tw = s + (1 << D.px);
    load_twiddles(tw, D.twx, D.px);
    const int ja = 1 + 2 * int(blockIdx.x), jb = ja + 1;
    const int nx = D.nx;
    // f' = f - lap(phi on the edges), on the interior nodes next to an edge
    auto fmod = [&](int i, int j) {
        if (j > D.Ny) return 0.0;
        const long k = long(j) * nx + i;
        double v = f[k];
        if (i == 1) v -= D.cx * phi[k - 1];
        if (i == D.Nx) v -= D.cx * phi[k + 1];
        if (j == 1) v -= D.cy * phi[k - nx];
        if (j == D.Ny) v -= D.cy * phi[k + nx];
        return v;
    };
    load_odd_pair(s, D.px, D.Mx, [&](int n) { return fmod(n, ja); }, [&](int n) { return fmod(n, jb); });
    __syncthreads();
    fft_smem(s, D.px, tw);
    for (int k = 1 + threadIdx.x; k < D.Mx; k += blockDim.x) {
        const double2 z = s[k];
        double* t = D.T + long(k - 1) * D.Ny + (ja - 1);
        t[0] = -0.5 * z.y;
        if (jb <= D.Ny) t[1] = 0.5 * z.x;
    }
}

// Rows (k_a, k_b) of T: forward DST along y, divide by the eigenvalues (and
// the normalisation 4 / (Mx My)), inverse DST along y, in place.
__global__ void __launch_bounds__(kDstThreads) k_dst_cols(DstDev D) {
    extern __shared__ __align__(16) unsigned char smem[];
    double2* s = reinterpret_cast<double2*>(smem);
    double2* tw = s + (1 << D.py);
    double* u = reinterpret_cast<double*>(tw + (1 << (D.py - 1)));  // [2][My]
    load_twiddles(tw, D.twy, D.py);
    const int ka = 1 + 2 * int(blockIdx.x), kb = ka + 1;
    const double* ra = D.T + long(ka - 1) * D.Ny;
    const double* rb = D.T + long(kb - 1) * D.Ny;
    const bool hb = kb <= D.Nx;
    load_odd_pair(s, D.py, D.My, [&](int n) { return ra[n - 1]; }, [&](int n) { return hb ? rb[n - 1] : 0.0; });
    __syncthreads();
    fft_smem(s, D.py, tw);
    const double norm = 4.0 / (double(D.Mx) * double(D.My));
    for (int l = 1 + threadIdx.x; l < D.My; l += blockDim.x) {
        const double2 z = s[l];
        u[l] = (-0.5 * z.y) * norm / -(D.lamx[ka] + D.lamy[l]);
        u[D.My + l] = hb ? (0.5 * z.x) * norm / -(D.lamx[kb] + D.lamy[l]) : 0.0;
    }
    __syncthreads();
    load_odd_pair(s, D.py, D.My, [&](int n) { return u[n]; }, [&](int n) { return u[D.My + n]; });
    __syncthreads();
    fft_smem(s, D.py, tw);
    double* wa = D.T + long(ka - 1) * D.Ny;
    double* wb = D.T + long(kb - 1) * D.Ny;
    for (int l = 1 + threadIdx.x; l < D.My; l += blockDim.x) {
        const double2 z = s[l];
        wa[l - 1] = -0.5 * z.y;
        if (hb) wb[l - 1] = 0.5 * z.x;
    }
}

// Interior rows (j_a, j_b): inverse DST along x of the columns of T, written
// to the interior of phi (the edges keep their values).
__global__ void __launch_bounds__(kDstThreads) k_dst_back(DstDev D, double* __restrict__ phi) {
    extern __shared__ __align__(16) unsigned char smem[];
    double2* s = reinterpret_cast<double2*>(smem);
    double2* tw = s + (1 << D.px);
    load_twiddles(tw, D.twx, D.px);
    const int ja = 1 + 2 * int(blockIdx.x), jb = ja + 1;
    const bool hb = jb <= D.Ny;
    load_odd_pair(
        s, D.px, D.Mx, [&](int n) { return D.T[long(n - 1) * D.Ny + (ja - 1)]; },
        [&](int n) { return hb ? D.T[long(n - 1) * D.Ny + (jb - 1)] : 0.0; });
    __syncthreads();
    fft_smem(s, D.px, tw);
    for (int i = 1 + threadIdx.x; i < D.Mx; i += blockDim.x) {
        const double2 z = s[i];
        phi[long(ja) * D.nx + i] = -0.5 * z.y;
        if (hb) phi[long(jb) * D.nx + i] = 0.5 * z.x;
    }
}

// ---- host plan ------------------------------------------------------------------------

struct DstPlan {
    DstDev d{};
    std::vector<void*> allocs;
    size_t smem_rows = 0, smem_cols = 0;
};

static int log2_exact(int v) {
    int p = 0;
    while ((1 << p) < v) ++p;
    return (1 << p) == v ? p : -1;
}

void dst_destroy(DstPlan* P) {
    if (!P) return;
    for (void* a : P->allocs) cudaFree(a);
    delete P;
}

// nx - 1 and ny - 1 powers of two, 4..2048.
int dst_create(int nx, int ny, double dx, double dy, DstPlan** out) {
    const int qx = log2_exact(nx - 1), qy = log2_exact(ny - 1);
    if (qx < 2 || qy < 2 || qx > 11 || qy > 11)
        return fail(PIC_ERR_BAD_ARG, "DST solver: node counts must be 2^q + 1 with 2 <= q <= 11 (got %dx%d)", nx, ny);
    DstPlan* P = new DstPlan;
    DstDev& D = P->d;
    D.nx = nx;
    D.ny = ny;
    D.Mx = nx - 1;
    D.My = ny - 1;
    D.Nx = nx - 2;
    D.Ny = ny - 2;
    D.px = qx + 1;
    D.py = qy + 1;
    D.cx = 1.0 / (dx * dx);
    D.cy = 1.0 / (dy * dy);
    const double pi = 3.14159265358979323846;
    auto upload = [&](const void* h, size_t bytes, void** d) {
        if (cudaMalloc(d, bytes) != cudaSuccess) return false;
        P->allocs.push_back(*d);
        return cudaMemcpy(*d, h, bytes, cudaMemcpyHostToDevice) == cudaSuccess;
    };
    bool ok = true;
    for (int a = 0; a < 2 && ok; ++a) {
        const int M = a ? D.My : D.Mx;
        const double c = a ? D.cy : D.cx;
        std::vector<double2> tw(static_cast<size_t>(M));
        for (int m = 0; m < M; ++m) tw[m] = make_double2(std::cos(pi * m / M), -std::sin(pi * m / M));
        std::vector<double> lam(static_cast<size_t>(M) + 1);
        for (int k = 0; k <= M; ++k) {
            const double sn = std::sin(pi * k / (2.0 * M));
            lam[k] = 4.0 * c * sn * sn;
        }
        void *dt = nullptr, *dl = nullptr;
        ok = upload(tw.data(), tw.size() * sizeof(double2), &dt) && upload(lam.data(), lam.size() * sizeof(double), &dl);
        if (a) {
            D.twy = static_cast<const double2*>(dt);
            D.lamy = static_cast<const double*>(dl);
        } else {
            D.twx = static_cast<const double2*>(dt);
            D.lamx = static_cast<const double*>(dl);
        }
    }
    if (ok) {
        void* t = nullptr;
        ok = cudaMalloc(&t, sizeof(double) * size_t(D.Nx) * D.Ny) == cudaSuccess;
        if (ok) {
            P->allocs.push_back(t);
            D.T = static_cast<double*>(t);
        }
    }
    if (!ok) {
        dst_destroy(P);
        return fail(PIC_ERR_CUDA, "DST solver: out of device memory");
    }
    // shared memory: the FFT (2M complex), its twiddles (M complex), and for the
    // column kernel the divided spectrum of two rows (2M doubles)
    P->smem_rows = sizeof(double2) * (size_t(2 * D.Mx) + D.Mx);
    P->smem_cols = sizeof(double2) * (size_t(2 * D.My) + D.My) + sizeof(double) * 2 * size_t(D.My);
    int rc = raise_smem_limit(reinterpret_cast<const void*>(k_dst_rows), P->smem_rows);
    if (rc == PIC_OK) rc = raise_smem_limit(reinterpret_cast<const void*>(k_dst_back), P->smem_rows);
    if (rc == PIC_OK) rc = raise_smem_limit(reinterpret_cast<const void*>(k_dst_cols), P->smem_cols);
    if (rc != PIC_OK) {
        dst_destroy(P);
        return rc;
    }
    *out = P;
    return PIC_OK;
}

// phi: FP64 nx*ny with the edge values set (kept); f: FP64 right-hand side.
int dst_launch(DstPlan* P, double* phi, const double* f, cudaStream_t st) {
    const DstDev& D = P->d;
    k_dst_rows<<<(D.Ny + 1) / 2, kDstThreads, P->smem_rows, st>>>(D, phi, f);
    k_dst_cols<<<(D.Nx + 1) / 2, kDstThreads, P->smem_cols, st>>>(D);
    k_dst_back<<<(D.Ny + 1) / 2, kDstThreads, P->smem_rows, st>>>(D, phi);
    PIC_LAUNCH_CHECK();
    return PIC_OK;
}

}  // namespace pic
