/*
 * pic_oracle.c -- CPU restatement of the reference's electrostatic PIC time
 * step.  TEST INFRASTRUCTURE ONLY: the tests, smoke() and the benchmark's CPU
 * baseline call it as the checker; the shipped library never links it.
 *
 * Two arithmetics are restated:
 *   *_f64  the reference's own FP64 arithmetic, operation for operation, on
 *          per-species SoA arrays in metres (pinned bit-exact against the
 *          reference's kernels compiled by ref_build.py, through the golden
 *          vectors in tests/golden/).  `floorf_quirk` reproduces the
 *          reference's `int(floorf(double))`, which rounds to float first
 *          (src/Grid.py:120-121, src/Particles.py:145-146).
 *   *_f32  the FP32 arithmetic the CUDA build uses, with the same operation
 *          order (explicit fmaf where the kernels use an FMA, no contraction
 *          elsewhere: compile with -ffp-contract=off).  Positions are in grid
 *          units (x/dx), velocities in m/s.  A dead (absorbed) particle holds
 *          NaN in its position.
 * Every function names the reference lines it follows.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------ */
/* FP64, reference arithmetic                                          */
/* ------------------------------------------------------------------ */

static inline int floor_ref(double v, int quirk) { return quirk ? (int)floorf((float)v) : (int)floor(v); }

static inline double clamp_ref(double v, int hi) {
    /* max(0.0f, min(v, double(hi))) with CUDA's fmin/fmax semantics */
    return fmax(0.0, fmin(v, (double)hi));
}

/* Cartesian CIC deposit of one species: src/Grid.py:108-152 (kernel body).
 * Accumulates charge*w into rho; the caller zeroes rho and divides by dx*dy
 * (src/Grid.py:250,294). */
void or_deposit_f64(double* rho, const double* x, const double* y, long n, double charge, double dx,
                    double dy, int m, int nn, int floorf_quirk) {
    for (long p = 0; p < n; ++p) {
        double gx = x[p] / dx, gy = y[p] / dy;
        gx = clamp_ref(gx, m - 1);
        gy = clamp_ref(gy, nn - 1);
        int x0 = floor_ref(gx, floorf_quirk), y0 = floor_ref(gy, floorf_quirk);
        int x1 = x0 + 1 < m - 1 ? x0 + 1 : m - 1;
        int y1 = y0 + 1 < nn - 1 ? y0 + 1 : nn - 1;
        double wx = gx - (double)x0, wy = gy - (double)y0;
        double wx1 = 1.0 - wx, wy1 = 1.0 - wy;
        rho[(long)y0 * m + x0] += charge * (wx1 * wy1);
        rho[(long)y0 * m + x1] += charge * (wx * wy1);
        rho[(long)y1 * m + x0] += charge * (wx1 * wy);
        rho[(long)y1 * m + x1] += charge * (wx * wy);
    }
}

/* E = -grad(phi): src/Grid.py:167-194. */
void or_update_E_f64(const double* phi, double* Ex, double* Ey, int nx, int ny, double dx, double dy) {
    for (int iy = 0; iy < ny; ++iy)
        for (int ix = 0; ix < nx; ++ix) {
            long i = (long)iy * nx + ix;
            double ex = 0.0, ey = 0.0;
            if (ix > 0 && ix < nx - 1) ex = -(phi[i + 1] - phi[i - 1]) / (2.0 * dx);
            else if (ix == 0) ex = -(phi[i + 1] - phi[i]) / dx;
            else ex = -(phi[i] - phi[i - 1]) / dx;
            if (iy > 0 && iy < ny - 1) ey = -(phi[i + nx] - phi[i - nx]) / (2.0 * dy);
            else if (iy == 0) ey = -(phi[i + nx] - phi[i]) / dy;
            else ey = -(phi[i] - phi[i - nx]) / dy;
            Ex[i] = ex;
            Ey[i] = ey;
        }
}

/* Gather + kick of one species: src/Particles.py:128-179.  k = dt*q/m. */
void or_update_V_f64(const double* x, const double* y, double* vx, double* vy, long n, const double* Ex,
                     const double* Ey, double k, double dx, double dy, int m, int nn, int floorf_quirk) {
    for (long p = 0; p < n; ++p) {
        double gx = x[p] / dx, gy = y[p] / dy;
        if (!isfinite(gx)) gx = 0.0;
        if (!isfinite(gy)) gy = 0.0;
        gx = clamp_ref(gx, m - 1);
        gy = clamp_ref(gy, nn - 1);
        int x0 = floor_ref(gx, floorf_quirk), y0 = floor_ref(gy, floorf_quirk);
        int x1 = x0 + 1 < m - 1 ? x0 + 1 : m - 1;
        int y1 = y0 + 1 < nn - 1 ? y0 + 1 : nn - 1;
        double wx = gx - (double)x0, wy = gy - (double)y0;
        double wx1 = 1.0 - wx, wy1 = 1.0 - wy;
        double w0 = wx1 * wy1, w1 = wx * wy1, w2 = wx1 * wy, w3 = wx * wy;
        long i0 = (long)y0 * m + x0, i1 = (long)y0 * m + x1, i2 = (long)y1 * m + x0, i3 = (long)y1 * m + x1;
        double epx = w0 * Ex[i0] + w1 * Ex[i1] + w2 * Ex[i2] + w3 * Ex[i3];
        double epy = w0 * Ey[i0] + w1 * Ey[i1] + w2 * Ey[i2] + w3 * Ey[i3];
        vx[p] += k * epx;
        vy[p] += k * epy;
    }
}

/* Drift: src/Particles.py:257-262 (R_old is the caller's copy). */
void or_update_R_f64(double* x, double* y, const double* vx, const double* vy, long n, double dt) {
    for (long p = 0; p < n; ++p) {
        x[p] += vx[p] * dt;
        y[p] += vy[p] * dt;
    }
}

/* Absorbing walls: the out-of-bounds predicate of src/collisions.py:193-194
 * applied to all four walls.  Returns the number absorbed; absorbed entries
 * get NaN positions. */
long or_absorb_f64(double* x, double* y, long n, double X, double Y) {
    long a = 0;
    for (long p = 0; p < n; ++p) {
        if (x[p] != x[p]) continue;
        if (x[p] < 0.0 || x[p] > X || y[p] < 0.0 || y[p] > Y) {
            x[p] = NAN;
            y[p] = NAN;
            ++a;
        }
    }
    return a;
}

/* Five-point residual r = f - A phi on free nodes (0 on Dirichlet and edge
 * nodes): the operator of src/multigrid.py:68-75 with the mask meaning of
 * src/Boundaries.py:9-10 (1 = Dirichlet).  Returns sum r^2. */
double or_residual_f64(const double* phi, const double* f, const unsigned char* dirichlet, double* r, int nx,
                       int ny, double dx, double dy) {
    const double cx = 1.0 / (dx * dx), cy = 1.0 / (dy * dy);
    double s = 0.0;
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            long k = (long)j * nx + i;
            double v = 0.0;
            if (i > 0 && i < nx - 1 && j > 0 && j < ny - 1 && !dirichlet[k]) {
                double lap = cx * (phi[k - 1] + phi[k + 1]) + cy * (phi[k - nx] + phi[k + nx]) -
                             2.0 * (cx + cy) * phi[k];
                v = f[k] - lap;
            }
            if (r) r[k] = v;
            s += v * v;
        }
    return s;
}

/* ------------------------------------------------------------------ */
/* FP32, the build's arithmetic (grid units, NaN = dead)               */
/* ------------------------------------------------------------------ */

typedef struct {
    int i0, j0, i1, j1;
    float w00, w10, w01, w11;
} or_cic;

/* Node indices and bilinear weights; same clamp/floor/neighbour rule as
 * src/Grid.py:116-137 in FP32. */
static inline or_cic or_weights(float gx, float gy, int m, int n) {
    or_cic c;
    float cx = fminf(fmaxf(gx, 0.0f), (float)(m - 1));
    float cy = fminf(fmaxf(gy, 0.0f), (float)(n - 1));
    c.i0 = (int)floorf(cx);
    c.j0 = (int)floorf(cy);
    c.i1 = c.i0 + 1 < m - 1 ? c.i0 + 1 : m - 1;
    c.j1 = c.j0 + 1 < n - 1 ? c.j0 + 1 : n - 1;
    float wx = cx - (float)c.i0, wy = cy - (float)c.j0;
    float ux = 1.0f - wx, uy = 1.0f - wy;
    c.w00 = ux * uy;
    c.w10 = wx * uy;
    c.w01 = ux * wy;
    c.w11 = wx * wy;
    return c;
}

/* E node values in FP32 from FP64 phi: or_update_E_f64 rounded once. */
void or_update_E_f32(const double* phi, float* Ex, float* Ey, int nx, int ny, double dx, double dy) {
    long G = (long)nx * ny;
    double* ex = (double*)malloc(sizeof(double) * G);
    double* ey = (double*)malloc(sizeof(double) * G);
    or_update_E_f64(phi, ex, ey, nx, ny, dx, dy);
    for (long i = 0; i < G; ++i) {
        Ex[i] = (float)ex[i];
        Ey[i] = (float)ey[i];
    }
    free(ex);
    free(ey);
}

/* CIC deposit of one species (FP32 contributions accumulated in FP64 so the
 * comparison is against the exact sum of the contributions).  `scale` is
 * q*np2c/(dx*dy) rounded to float.  abs_sum (optional) receives sum |c|. */
void or_deposit_f32(double* rho, double* abs_sum, const float* gx, const float* gy, long n, float scale, int m,
                    int nn) {
    for (long p = 0; p < n; ++p) {
        if (gx[p] != gx[p]) continue;
        or_cic c = or_weights(gx[p], gy[p], m, nn);
        float v00 = scale * c.w00, v10 = scale * c.w10, v01 = scale * c.w01, v11 = scale * c.w11;
        long k00 = (long)c.j0 * m + c.i0, k10 = (long)c.j0 * m + c.i1;
        long k01 = (long)c.j1 * m + c.i0, k11 = (long)c.j1 * m + c.i1;
        rho[k00] += v00;
        rho[k10] += v10;
        rho[k01] += v01;
        rho[k11] += v11;
        if (abs_sum) {
            abs_sum[k00] += fabsf(v00);
            abs_sum[k10] += fabsf(v10);
            abs_sum[k01] += fabsf(v01);
            abs_sum[k11] += fabsf(v11);
        }
    }
}

/* Gather + kick (src/Particles.py:128-179 in FP32): kq = q/m*dt as float. */
void or_kick_f32(const float* gx, const float* gy, float* vx, float* vy, long n, const float* Ex,
                 const float* Ey, float kq, int m, int nn) {
    for (long p = 0; p < n; ++p) {
        if (gx[p] != gx[p]) continue;
        or_cic c = or_weights(gx[p], gy[p], m, nn);
        long k00 = (long)c.j0 * m + c.i0, k10 = (long)c.j0 * m + c.i1;
        long k01 = (long)c.j1 * m + c.i0, k11 = (long)c.j1 * m + c.i1;
        float ex = c.w00 * Ex[k00];
        ex = fmaf(c.w10, Ex[k10], ex);
        ex = fmaf(c.w01, Ex[k01], ex);
        ex = fmaf(c.w11, Ex[k11], ex);
        float ey = c.w00 * Ey[k00];
        ey = fmaf(c.w10, Ey[k10], ey);
        ey = fmaf(c.w01, Ey[k01], ey);
        ey = fmaf(c.w11, Ey[k11], ey);
        vx[p] = fmaf(kq, ex, vx[p]);
        vy[p] = fmaf(kq, ey, vy[p]);
    }
}

/* Drift (src/Particles.py:257-262 in grid units) followed by absorption at
 * all four walls.  Returns the number absorbed. */
long or_drift_absorb_f32(float* gx, float* gy, const float* vx, const float* vy, long n, float dtdx, float dtdy,
                         int m, int nn) {
    long a = 0;
    const float X = (float)(m - 1), Y = (float)(nn - 1);
    for (long p = 0; p < n; ++p) {
        if (gx[p] != gx[p]) continue;
        float x = fmaf(vx[p], dtdx, gx[p]);
        float y = fmaf(vy[p], dtdy, gy[p]);
        if (x >= 0.0f && x <= X && y >= 0.0f && y <= Y) {
            gx[p] = x;
            gy[p] = y;
        } else {
            gx[p] = NAN;
            gy[p] = NAN;
            ++a;
        }
    }
    return a;
}

/* Internal electrodes (the build's collection of particles by internal
 * equipotentials; the reference's tracing in src/collisions.py:73-175 is
 * unused).  Vertical edge (X, j): x = X, j < y < j + 1, bit X*(ny-1)+j of vb;
 * horizontal edge (i, Y): y = Y, i < x < i + 1, bit Y*(nx-1)+i of hb.  A line
 * is crossed when the drift ends on it or passes it, not when it starts on
 * it; each crossing is intersected in FP32 (x - x0) / dx, fmaf(t, dy, y0). */
static int edge_bit(const uint32_t* b, long k) { return (int)((b[k >> 5] >> (k & 31)) & 1u); }

int or_hits_electrode(float x0, float y0, float x1, float y1, int nx, int ny, const uint32_t* vb,
                      const uint32_t* hb) {
    const float ddx = x1 - x0, ddy = y1 - y0;
    if (ddx != 0.0f) {
        int a = ddx > 0.0f ? (int)floorf(x0) + 1 : (int)ceilf(x1);
        int b = ddx > 0.0f ? (int)floorf(x1) : (int)ceilf(x0) - 1;
        if (a < 1) a = 1;
        if (b > nx - 2) b = nx - 2;
        for (int X = a; X <= b; ++X) {
            const float t = ((float)X - x0) / ddx;
            const int j = (int)floorf(fmaf(t, ddy, y0));
            if (j >= 0 && j < ny - 1 && edge_bit(vb, (long)X * (ny - 1) + j)) return 1;
        }
    }
    if (ddy != 0.0f) {
        int a = ddy > 0.0f ? (int)floorf(y0) + 1 : (int)ceilf(y1);
        int b = ddy > 0.0f ? (int)floorf(y1) : (int)ceilf(y0) - 1;
        if (a < 1) a = 1;
        if (b > ny - 2) b = ny - 2;
        for (int Y = a; Y <= b; ++Y) {
            const float t = ((float)Y - y0) / ddy;
            const int i = (int)floorf(fmaf(t, ddx, x0));
            if (i >= 0 && i < nx - 1 && edge_bit(hb, (long)Y * (nx - 1) + i)) return 1;
        }
    }
    return 0;
}

/* or_drift_absorb_f32 plus collection by internal electrodes; *collected
 * receives the particles the electrodes took, the return value the wall count. */
long or_drift_absorb_electrodes_f32(float* gx, float* gy, const float* vx, const float* vy, long n, float dtdx,
                                    float dtdy, int m, int nn, const uint32_t* vb, const uint32_t* hb,
                                    long* collected) {
    long a = 0, c = 0;
    const float X = (float)(m - 1), Y = (float)(nn - 1);
    for (long p = 0; p < n; ++p) {
        if (gx[p] != gx[p]) continue;
        const float x0 = gx[p], y0 = gy[p];
        float x = fmaf(vx[p], dtdx, x0);
        float y = fmaf(vy[p], dtdy, y0);
        if (!(x >= 0.0f && x <= X && y >= 0.0f && y <= Y)) {
            gx[p] = NAN;
            gy[p] = NAN;
            ++a;
        } else if (or_hits_electrode(x0, y0, x, y, m, nn, vb, hb)) {
            gx[p] = NAN;
            gy[p] = NAN;
            ++c;
        } else {
            gx[p] = x;
            gy[p] = y;
        }
    }
    *collected = c;
    return a;
}

/* r-z (axisymmetric) drift, the build's replacement of the planar drift and
 * axis reflection the reference uses in cylindrical mode too
 * (src/Particles.py:359-376, kernels K6/K7 at :251-280).  x axial, y radial
 * (grid units), vx axial, vy radial, vz azimuthal.  The particle moves on a
 * straight line in 3D; in the plane normal to the axis it goes from (y, 0)
 * to (y + vy dtdy, vz dtdy), its new radius is the length of that vector and
 * (vy, vz) are turned by its angle (Birdsall and Langdon sec. 14-12).  The
 * operation order is the CUDA build's (drift_rz); sqrtf and / are correctly
 * rounded, as there. */
static void drift_rz1(float* x, float* y, float vx, float* vy, float* vz, float dtdx, float dtdy) {
    *x = fmaf(vx, dtdx, *x);
    const float yr = fmaf(*vy, dtdy, *y);
    const float yt = *vz * dtdy;
    const float r = sqrtf(fmaf(yr, yr, yt * yt));
    if (r > 0.0f) {
        const float c = yr / r, s = yt / r;
        const float vr = fmaf(c, *vy, s * *vz);
        const float vt = fmaf(c, *vz, -(s * *vy));
        *vy = vr;
        *vz = vt;
    }
    *y = r;
}

/* r-z drift of every live particle with wall absorption (x outside [0, m-1]
 * or r > n-1) and, with vb/hb not NULL, collection by internal electrodes;
 * returns the wall count, *collected the electrode count. */
long or_drift_rz_absorb_f32(float* gx, float* gy, const float* vx, float* vy, float* vz, long n, float dtdx,
                            float dtdy, int m, int nn, const uint32_t* vb, const uint32_t* hb, long* collected) {
    long a = 0, c = 0;
    const float X = (float)(m - 1), Y = (float)(nn - 1);
    for (long p = 0; p < n; ++p) {
        if (gx[p] != gx[p]) continue;
        const float x0 = gx[p], y0 = gy[p];
        float x = x0, y = y0, v1 = vy[p], v2 = vz[p];
        drift_rz1(&x, &y, vx[p], &v1, &v2, dtdx, dtdy);
        vy[p] = v1;
        vz[p] = v2;
        if (!(x >= 0.0f && x <= X && y >= 0.0f && y <= Y)) {
            gx[p] = NAN;
            gy[p] = NAN;
            ++a;
        } else if (vb && hb && or_hits_electrode(x0, y0, x, y, m, nn, vb, hb)) {
            gx[p] = NAN;
            gy[p] = NAN;
            ++c;
        } else {
            gx[p] = x;
            gy[p] = y;
        }
    }
    if (collected) *collected = c;
    return a;
}

/* ------------------------------------------------------------------ */
/* Cell sort (the deterministic replacement of src/Particles.py:550-632) */
/* ------------------------------------------------------------------ */

/* Tile-major cell key: cells are grouped in ts x ts tiles, tiles in row-major
 * order, cells row-major inside a tile.  Dead particles get key = ncells. */
void or_sort_keys(const float* gx, const float* gy, long n, int m, int nn, int ts, uint32_t* keys) {
    const int cx_n = m - 1, cy_n = nn - 1;
    const int tiles_x = (cx_n + ts - 1) / ts;
    const uint32_t ncells = (uint32_t)((long)tiles_x * ((cy_n + ts - 1) / ts) * ts * ts);
    for (long p = 0; p < n; ++p) {
        if (gx[p] != gx[p]) {
            keys[p] = ncells;
            continue;
        }
        int cx = (int)gx[p], cy = (int)gy[p];
        if (cx > cx_n - 1) cx = cx_n - 1;
        if (cy > cy_n - 1) cy = cy_n - 1;
        int tx = cx / ts, ty = cy / ts;
        keys[p] = (uint32_t)(((long)ty * tiles_x + tx) * ts * ts + (cy - ty * ts) * ts + (cx - tx * ts));
    }
}

/* Stable counting sort of keys in [0, nkeys]: perm[k] = source index of the
 * k-th element of the sorted order. */
void or_counting_sort(const uint32_t* keys, long n, uint32_t nkeys, uint32_t* perm) {
    long* start = (long*)calloc((size_t)nkeys + 2, sizeof(long));
    for (long p = 0; p < n; ++p) start[keys[p] + 1]++;
    for (uint32_t k = 0; k <= nkeys; ++k) start[k + 1] += start[k];
    for (long p = 0; p < n; ++p) perm[start[keys[p]]++] = (uint32_t)p;
    free(start);
}

/* ------------------------------------------------------------------ */
/* Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11)                    */
/* ------------------------------------------------------------------ */

void or_philox4x32_10(const uint32_t ctr_in[4], const uint32_t key_in[2], uint32_t out[4]) {
    uint32_t c0 = ctr_in[0], c1 = ctr_in[1], c2 = ctr_in[2], c3 = ctr_in[3];
    uint32_t k0 = key_in[0], k1 = key_in[1];
    for (int r = 0; r < 10; ++r) {
        if (r) {
            k0 += 0x9E3779B9u;
            k1 += 0xBB67AE85u;
        }
        uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
        c0 = n0;
        c1 = lo1;
        c2 = n2;
        c3 = lo0;
    }
    out[0] = c0;
    out[1] = c1;
    out[2] = c2;
    out[3] = c3;
}

/* ------------------------------------------------------------------ */
/* Null-collision MCC (Vahedi & Surendra, CPC 87 (1995) 179)           */
/* ------------------------------------------------------------------ */

enum { OR_ELASTIC = 0, OR_EXCITATION = 1, OR_IONIZATION = 2, OR_CHARGE_EXCHANGE = 3 };

typedef struct {
    int nproc;
    int type[4];
    float threshold[4];
    const float* sigma[4]; /* each ne values on the shared energy grid */
    int ne;
    const float* energy;   /* ne log-spaced energies, eV */
    float inv_log_ratio;   /* 1/log(E[1]/E[0]) */
    float log_e0;          /* log(E[0]) */
    float gas_density;     /* m^-3 */
    float half_m_over_q;   /* 0.5*m/qe: eV per (m/s)^2 */
    float mass_ratio2;     /* 2*m/M_gas for elastic recoil */
    float gas_vth;         /* sqrt(kT/M_gas), m/s */
    float nu_max;          /* nu' = max over the table of n_g*sigma_T(E)*v(E), 1/s */
    double inv_log1m_p;    /* 1/log(1-P_null) */
    uint32_t species;      /* stream id */
    uint32_t seg;          /* particles per candidate segment */
} or_mcc_species;

/* The uniform in (0,1] made from one 32-bit Philox output, as a double and as a float. */
static inline double or_u64(uint32_t x) { return ((double)x + 1.0) * (1.0 / 4294967296.0); }
static inline float or_u32(uint32_t x) { return (float)(x >> 8) * (1.0f / 16777216.0f) + (0.5f / 16777216.0f); }

/* Candidates of segment g: geometric gaps between successes of independent
 * Bernoulli(P_null) trials.  Sets mark[i] for candidates i in [0, n). */
void or_mcc_candidates(const or_mcc_species* s, long n, uint32_t step, uint32_t seed_lo, uint32_t seed_hi,
                       unsigned char* mark) {
    const uint32_t key[2] = {seed_lo, seed_hi};
    const long nseg = (n + s->seg - 1) / s->seg;
    for (long g = 0; g < nseg; ++g) {
        long pos = -1;
        uint32_t draw = 0, out[4];
        for (;;) {
            if ((draw & 3u) == 0) {
                uint32_t ctr[4] = {(uint32_t)g, step, s->species, draw >> 2};
                or_philox4x32_10(ctr, key, out);
            }
            double u = or_u64(out[draw & 3u]);
            ++draw;
            double f = floor(log(u) * s->inv_log1m_p);
            if (f > (double)s->seg) break;
            pos += 1 + (long)f;
            if (pos >= (long)s->seg) break;
            long i = g * (long)s->seg + pos;
            if (i >= n) break;
            mark[i] = 1;
        }
    }
}

/* Linear interpolation of a process table at energy e (eV); clamps at the
 * table ends like src/MCC.py:54-60 and interpolates linearly in E inside. */
static inline float or_sigma(const or_mcc_species* s, int k, float e) {
    const float* E = s->energy;
    const float* S = s->sigma[k];
    if (e <= E[0]) return S[0];
    if (e >= E[s->ne - 1]) return S[s->ne - 1];
    int j = (int)((logf(e) - s->log_e0) * s->inv_log_ratio);
    if (j < 0) j = 0;
    if (j > s->ne - 2) j = s->ne - 2;
    while (j > 0 && e < E[j]) --j;
    while (j < s->ne - 2 && e >= E[j + 1]) ++j;
    float t = (e - E[j]) / (E[j + 1] - E[j]);
    return fmaf(t, S[j + 1] - S[j], S[j]);
}

static inline void or_isotropic(float u_cos, float u_phi, float* dx, float* dy, float* dz) {
    float c = 1.0f - 2.0f * u_cos;
    float s = sqrtf(fmaxf(0.0f, 1.0f - c * c));
    float ph = 6.2831853071795864f * u_phi;
    *dx = s * cosf(ph);
    *dy = s * sinf(ph);
    *dz = c;
}

/* One candidate collision.  Returns the process index that fired, or -1
 * (null collision).  Births (ionisation) are written to born_e / born_i
 * (x, y, vx, vy, vz) when not NULL. */
int or_mcc_collide(const or_mcc_species* s, uint32_t idx, uint32_t step, uint32_t seed_lo, uint32_t seed_hi,
                   float* vx, float* vy, float* vz, float born_e[3], float born_i[3]) {
    const uint32_t key[2] = {seed_lo, seed_hi};
    uint32_t r0[4], r1[4], r2[4];
    uint32_t ctr[4] = {idx, step, s->species | 0x100u, 0};
    or_philox4x32_10(ctr, key, r0);
    float v2 = (*vx) * (*vx) + (*vy) * (*vy) + (*vz) * (*vz);
    float speed = sqrtf(v2);
    float e = s->half_m_over_q * v2;
    float target = or_u32(r0[0]) * s->nu_max;
    float acc = 0.0f;
    int proc = -1;
    for (int k = 0; k < s->nproc; ++k) {
        acc += s->gas_density * or_sigma(s, k, e) * speed;
        if (target < acc) {
            proc = k;
            break;
        }
    }
    if (proc < 0) return -1;
    const int type = s->type[proc];
    float e_left = e;
    if (type == OR_EXCITATION || type == OR_IONIZATION) {
        e_left = e - s->threshold[proc];
        if (!(e_left > 0.0f)) return -1;
    }
    if (type == OR_CHARGE_EXCHANGE) {
        ctr[3] = 2;
        or_philox4x32_10(ctr, key, r2);
        float a = sqrtf(-2.0f * logf(or_u32(r2[0]))), b = 6.2831853071795864f * or_u32(r2[1]);
        float c = sqrtf(-2.0f * logf(or_u32(r2[2]))), d = 6.2831853071795864f * or_u32(r2[3]);
        *vx = s->gas_vth * a * cosf(b);
        *vy = s->gas_vth * a * sinf(b);
        *vz = s->gas_vth * c * cosf(d);
        return proc;
    }
    float dx, dy, dz;
    or_isotropic(or_u32(r0[1]), or_u32(r0[2]), &dx, &dy, &dz);
    float new_speed;
    if (type == OR_ELASTIC) {
        float inv = speed > 0.0f ? 1.0f / speed : 0.0f;
        float cosx = ((*vx) * dx + (*vy) * dy + (*vz) * dz) * inv;
        new_speed = speed * sqrtf(fmaxf(0.0f, 1.0f - s->mass_ratio2 * (1.0f - cosx)));
    } else if (type == OR_EXCITATION) {
        new_speed = sqrtf(e_left / s->half_m_over_q);
    } else { /* ionisation: energy split U(0.2,0.8) as src/MCC.py:272-287 */
        float frac = 0.2f + 0.6f * or_u32(r0[3]);
        new_speed = sqrtf(frac * e_left / s->half_m_over_q);
        float sec_speed = sqrtf((1.0f - frac) * e_left / s->half_m_over_q);
        ctr[3] = 1;
        or_philox4x32_10(ctr, key, r1);
        float sx, sy, sz;
        or_isotropic(or_u32(r1[0]), or_u32(r1[1]), &sx, &sy, &sz);
        if (born_e) {
            born_e[0] = sec_speed * sx;
            born_e[1] = sec_speed * sy;
            born_e[2] = sec_speed * sz;
        }
        ctr[3] = 2;
        or_philox4x32_10(ctr, key, r2);
        float a = sqrtf(-2.0f * logf(or_u32(r2[0]))), b = 6.2831853071795864f * or_u32(r2[1]);
        float c = sqrtf(-2.0f * logf(or_u32(r2[2]))), d = 6.2831853071795864f * or_u32(r2[3]);
        if (born_i) {
            born_i[0] = s->gas_vth * a * cosf(b);
            born_i[1] = s->gas_vth * a * sinf(b);
            born_i[2] = s->gas_vth * c * cosf(d);
        }
    }
    *vx = new_speed * dx;
    *vy = new_speed * dy;
    *vz = new_speed * dz;
    return proc;
}
