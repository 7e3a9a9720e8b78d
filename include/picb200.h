/*
 * picb200.h -- C ABI of libpicb200.so, the B200 (sm_100a) implementation of
 * the electrostatic PIC time step of dimad285/PIC: CIC charge deposition,
 * the multigrid Poisson solve, field gather fused with the leapfrog push and
 * wall absorption, cell sorting, and null-collision Monte-Carlo collisions.
 *
 * The reference has no C interface: its operator API is the set of Python
 * classes that src/simulation.py calls (Particles2D, Grid2D, Solver,
 * MultigridSolver, Boundaries, MCC).  Each entry point below names the
 * reference function it replaces; the Python shims in pic_b200/ bind these
 * symbols with ctypes and keep the reference's call signatures.
 *
 * Conventions
 *  - Every function returns a pic_status; 0 is success.  pic_last_error()
 *    returns a message for the last failing call on the calling thread.
 *  - Pointers named d_* are device pointers; h_* are host pointers.
 *  - Grid arrays are flat row-major, index = j*nx + i, nx = number of nodes
 *    in x (src/Grid.py:140-143).  Grids are given in NODES (Grid2D(m, n, ...)).
 *  - Particle arrays are SoA float32.  Positions are in grid units
 *    (x/dx, y/dy); velocities in m/s.  A dead (absorbed) slot holds NaN in x.
 *  - `stream` is a cudaStream_t passed as void*; NULL is the legacy stream.
 *    All calls are asynchronous on that stream unless they say otherwise.
 *  - Objects (pic_mg, pic_sorter, pic_sim) are not thread-safe; use one per
 *    host thread or serialise calls.
 */
#ifndef PICB200_H
#define PICB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PIC_ABI_VERSION 4
#define PIC_MAX_SPECIES 4
#define PIC_MAX_PROCESSES 4

typedef enum pic_status {
    PIC_OK = 0,
    PIC_ERR_BAD_ARG = 1,
    PIC_ERR_CUDA = 2,
    PIC_ERR_NOT_CONVERGED = 3,
    PIC_ERR_TIMEOUT = 4,
    PIC_ERR_OUT_OF_CAPACITY = 5,
    PIC_ERR_NUMERIC = 6
} pic_status;

int pic_abi_version(void);
/* Message of the last failing call on this host thread ("" if none). */
const char* pic_last_error(void);

/* ------------------------------------------------------------------ */
/* Stateless particle and grid operators                               */
/* ------------------------------------------------------------------ */

/* Particles2D.update_R (src/Particles.py:359-367, kernel :251-264):
 * x += vx*dtdx, y += vy*dtdy for live slots [0, n).  dtdx = dt/dx.
 * d_x_old/d_y_old (optional, may be NULL) receive the positions before the move. */
int pic_update_R(float* d_x, float* d_y, const float* d_vx, const float* d_vy, int n, float dtdx, float dtdy,
                 float* d_x_old, float* d_y_old, void* stream);

/* Wall absorption, the predicate of collisions.remove_out_of_bounds
 * (src/collisions.py:177-215) on all four walls: a live particle outside
 * [0, nx-1] x [0, ny-1] (grid units) is marked dead.  Replaces
 * Particles2D.update_axis (src/Particles.py:369-376), which reflects at y < 0.
 * *d_absorbed (device, uint64) is incremented by the number absorbed. */
int pic_absorb(float* d_x, float* d_y, int n, int nx, int ny, unsigned long long* d_absorbed, void* stream);

/* Particles2D.update_V (src/Particles.py:378-410, kernel :117-180): bilinear
 * gather of (Ex, Ey) at each live particle, v += kq*E with kq = dt*q/m. */
int pic_update_V(const float* d_x, const float* d_y, float* d_vx, float* d_vy, int n, const float* d_Ex,
                 const float* d_Ey, int nx, int ny, float kq, void* stream);

/* Grid2D.update_density, Cartesian (src/Grid.py:246-294, kernel :96-154):
 * adds scale*w (scale = q*np2c/(dx*dy)) of each live particle to the four
 * surrounding nodes of d_rho (float32, nx*ny).  The caller zeroes d_rho
 * once before depositing all species. */
int pic_deposit(const float* d_x, const float* d_y, int n, float scale, float* d_rho, int nx, int ny,
                void* stream);

/* Grid2D.update_E (src/Grid.py:232-243, kernel :157-196): E = -grad(phi),
 * central differences inside, one-sided at the edges, computed in FP64 and
 * stored as float32 planes d_Ex, d_Ey (nx*ny each). */
int pic_update_E(const double* d_phi, float* d_Ex, float* d_Ey, int nx, int ny, double dx, double dy,
                 void* stream);

/* Solver.solve right-hand side (src/Solvers.py:271-276): d_f = -rho/eps0 on
 * free nodes, d_f = 0 on Dirichlet nodes (d_dirichlet: uint8, 1 = Dirichlet).
 * The reference's extra dx^2 factor is not applied: the multigrid applies h^2. */
int pic_form_rhs(const float* d_rho, const uint8_t* d_dirichlet, double eps0, double* d_f, int nx, int ny,
                 void* stream);

/* r-z (axisymmetric) variants of the operators above, for Grid2D /
 * Particles2D with cylindrical=True (the reference's cylindrical kernels,
 * src/Grid.py:5-93 and src/Particles.py:183-248, with the corrections listed
 * in the design notes).  Coordinates: x axial, y radial (grid units), row 0
 * the axis.
 *
 * pic_update_E_rz: pic_update_E with E_r = 0 on the axis row (symmetry).
 * pic_rz_density: turns a charge deposited by pic_deposit (per dx*dy) into
 *   the charge density, rho_j *= dx*dy / V_j, with V_j the node volumes of
 *   the linear weighting (2 pi r_j dr dz inside; pi dr^2 dz / 3 on the axis;
 *   pi dr dz (r_top - dr/3) on the outer row), so a uniform load gives a
 *   uniform density.
 * pic_update_R_rz: the drift in 3D with the radial and azimuthal velocities
 *   (d_vy, d_vz) turned into the new local frame (Birdsall and Langdon,
 *   sec. 14-12), for live slots [0, n). */
int pic_update_E_rz(const double* d_phi, float* d_Ex, float* d_Ey, int nx, int ny, double dx, double dy,
                    void* stream);
int pic_rz_density(float* d_rho, int nx, int ny, double dy, void* stream);
int pic_update_R_rz(float* d_x, float* d_y, const float* d_vx, float* d_vy, float* d_vz, int n, float dtdx,
                    float dtdy, void* stream);

/* ------------------------------------------------------------------ */
/* Multigrid Poisson solver (src/multigrid.py:277-455, src/Solvers.py:258-299) */
/* ------------------------------------------------------------------ */

typedef struct pic_mg pic_mg;

typedef enum pic_mg_precision {
    PIC_MG_MIXED = 0, /* FP32 V-cycles inside an FP64 iterative-refinement loop */
    PIC_MG_FP64 = 1   /* the same V-cycle in FP64 throughout                    */
} pic_mg_precision;

typedef enum pic_mg_launch_mode {
    PIC_MG_PERSISTENT = 0, /* one cooperative kernel per solve; phases separated by grid barriers */
    PIC_MG_HOST_LOOP = 1,  /* one launch per kernel, convergence tested on the host each cycle */
    PIC_MG_GRAPH_LOOP = 2, /* one launch per kernel inside a CUDA-graph conditional WHILE node */
    PIC_MG_CLUSTER = 3,    /* one launch of a single thread-block cluster per solve (FP32 levels whose
                              row bands fit in shared memory; otherwise the graph loop) */
    PIC_MG_DST = 4,        /* no V-cycles: the direct solve by sine transforms of src/FFT.py:10-64
                              (FP64, three kernels, then the FP64 residual for pic_mg_info), for
                              Cartesian grids of 2^q + 1 nodes (q <= 11) whose Dirichlet nodes are
                              exactly the four edges; otherwise the graph loop */
    PIC_MG_HYBRID = 5      /* the graph loop with the levels of at most 129^2 nodes of each V-cycle
                              in one thread-block-cluster launch (FP32 Cartesian levels, grids
                              larger than 129^2; otherwise the graph loop) */
} pic_mg_launch_mode;

/* Geometry of the grid.  PIC_GEOM_RZ is axisymmetric r-z (the reference's
 * Grid.Cylindrical = 1, src/Grid.py:5-93, src/Solvers.py:100-166): x is the
 * axial coordinate z (nodes i, spacing dx), y the radius r (rows j, r = j*dy),
 * row 0 is the axis.  The axis row is not a boundary: its nodes are free
 * unless the mask marks them, and the operator there is the symmetric limit
 * 2 d2phi/dr2.  In a simulation, vx is the axial, vy the radial and vz the
 * azimuthal velocity, and particle counts (np2c) are real particles, not
 * particles per unit depth. */
typedef enum pic_geometry {
    PIC_GEOM_CARTESIAN = 0,
    PIC_GEOM_RZ = 1
} pic_geometry;

typedef struct pic_mg_options {
    int precision;    /* pic_mg_precision */
    int pre_sweeps;   /* red-black Gauss-Seidel sweeps before restriction (default 2) */
    int post_sweeps;  /* sweeps after prolongation (default 2) */
    double omega;     /* over-relaxation of the red-black smoother (default, when <= 0: 1.15) */
    int coarsest_max; /* coarsen while both node counts exceed this (default 9) */
    int launch_mode;  /* pic_mg_launch_mode (r-z solves use the graph or host loop) */
    int geometry;     /* pic_geometry (default 0: Cartesian) */
    int coarse_fp32;  /* PIC_MG_MIXED: 1 keeps the direct solve of the first level of at most 33^2
                         nodes (its inverse and products) in FP32; 0 (default) runs it in FP64 */
} pic_mg_options;

typedef struct pic_mg_info {
    int cycles;        /* V-cycles run */
    double rel_res;    /* final ||f - A phi|| / ||f|| over free nodes (FP64) */
    double rhs_norm;   /* ||f|| */
    int converged;     /* 1 if rel_res < tol */
} pic_mg_info;

/* MultigridSolver.__init__ (src/multigrid.py:278-309).  h_dirichlet: host
 * uint8 mask nx*ny (1 = Dirichlet: the bc_lookup of src/Boundaries.py:9-10).
 * Grid spacings dx, dy; (nx-1) and (ny-1) must be divisible by 2 down to
 * the coarsest level (nodes 2^k*c+1, as the reference requires).  opts may
 * be NULL for defaults.  Allocates device memory. */
int pic_mg_create(int nx, int ny, double dx, double dy, const uint8_t* h_dirichlet, const pic_mg_options* opts,
                  pic_mg** out);
int pic_mg_destroy(pic_mg* mg);

/* MultigridSolver.solve (src/multigrid.py:445-455): iterate V-cycles until
 * ||f - A phi||/||f|| < tol or max_cycles.  d_phi (FP64, nx*ny) holds the
 * initial guess and the Dirichlet values on Dirichlet nodes (never changed);
 * d_f (FP64) is the right-hand side (-rho/eps0).  Synchronises `stream` once
 * per cycle to test convergence.  Returns PIC_ERR_NOT_CONVERGED (with *info
 * filled) if max_cycles is reached first. */
int pic_mg_solve(pic_mg* mg, double* d_phi, const double* d_f, double tol, int max_cycles, pic_mg_info* info,
                 void* stream);

/* Device-resident solve for graph capture: runs exactly `cycles` V-cycles
 * with no host synchronisation; each cycle after convergence is skipped on
 * the device (the kernels test a device flag).  Read the outcome with
 * pic_mg_read_info after synchronising the stream. */
int pic_mg_solve_async(pic_mg* mg, double* d_phi, const double* d_f, double tol, int cycles, void* stream);
int pic_mg_read_info(pic_mg* mg, double tol, pic_mg_info* info);
/* The launch mode solves actually use (PIC_MG_CLUSTER falls back to
 * PIC_MG_GRAPH_LOOP where the cluster solve does not apply). */
int pic_mg_effective_launch_mode(pic_mg* mg, int* mode);
/* Failure detection of the persistent solve (PIC_MG_PERSISTENT; the
 * reference's host loop, src/multigrid.py:445-455, has no device wait to
 * bound): polls a grid barrier makes before the solve gives up, sets a device
 * error flag and returns, and the solve returns PIC_ERR_TIMEOUT (the flag is
 * then cleared and the solver stays usable).  polls < 0 restores the default
 * (2^24 polls, about a second). */
int pic_mg_set_wait_limit(pic_mg* mg, long long polls);
/* The shared-memory tile geometry the multigrid's tile kernels use for
 * `sweeps` red-black sweeps (1..8), in nodes, as PIC_MG_GEOMETRY_VALUES ints:
 * tile side; down phase halo and width; up phase halo, width and coarse
 * window width; the same for the finest up phase with the residual; the
 * two-level down launch's coarse halo and width and fine halo and width; the
 * two-level up launch's fine halo, width and coarse window width, and its
 * coarse width and coarse window width.  No counterpart in the reference (its
 * kernels work on whole levels); the tests emulate the tiles with these. */
#define PIC_MG_GEOMETRY_VALUES 18
int pic_mg_tile_geometry(int sweeps, int* out);

/* Solver(solver_type='cg' | 'gmres') (src/Solvers.py:245-258: cupyx cg and
 * gmres on the 5-point Laplacian with Dirichlet rows): flexible
 * preconditioned conjugate gradients for lap(phi) = f in FP64, Cartesian.
 * The system is symmetric, so the solution is the one GMRES converges to.
 * h_dirichlet: nx*ny, 1 = Dirichlet (the grid edges always are); precond: a
 * pic_mg of the same grid and mask whose one V-cycle from zero
 * preconditions each iteration (NULL: none).  pic_cg_solve keeps phi on the
 * Dirichlet nodes, iterates until ||f - lap(phi)|| / ||f|| < tol over the free
 * nodes or max_iter (info->cycles = iterations), synchronises `stream` once
 * per dot product, and returns PIC_ERR_NOT_CONVERGED if tol is not reached. */
typedef struct pic_cg pic_cg;
int pic_cg_create(int nx, int ny, double dx, double dy, const uint8_t* h_dirichlet, pic_mg* precond, pic_cg** out);
int pic_cg_solve(pic_cg* cg, double* d_phi, const double* d_f, double tol, int max_iter, pic_mg_info* info,
                 void* stream);
int pic_cg_destroy(pic_cg* cg);

/* ------------------------------------------------------------------ */
/* Cell sort (replaces Particles2D.sort_particles_sparse, src/Particles.py:550-632) */
/* ------------------------------------------------------------------ */

typedef struct pic_sorter pic_sorter;

/* Scratch for sorting up to `capacity` particles on an nx*ny-node grid whose
 * cells are grouped in tile x tile tiles (tile-major cell keys). */
int pic_sorter_create(int capacity, int nx, int ny, int tile, pic_sorter** out);
int pic_sorter_destroy(pic_sorter* s);

/* Stable counting sort by tile-major cell key.  Dead slots sort last and are
 * dropped.  Writes d_perm[k] = source slot of the k-th live particle in key
 * order (bit-identical to a stable argsort of the keys), gathers the five
 * arrays into the *_out arrays, writes the live count to *d_count_out
 * (device int) and, if d_tile_start is not NULL, the first sorted slot of
 * each tile (ntiles+1 ints).  d_perm and the *_out arrays need room for n
 * entries: only the first (live count) are written.  d_x_out may be NULL to
 * get the permutation alone.  Deterministic. */
int pic_sort(pic_sorter* s, const float* d_x, const float* d_y, const float* d_vx, const float* d_vy,
             const float* d_vz, int n, float* d_x_out, float* d_y_out, float* d_vx_out, float* d_vy_out,
             float* d_vz_out, uint32_t* d_perm, int* d_count_out, int* d_tile_start, void* stream);

/* The cell sort of pic_sort without allocation.  No counterpart in the
 * reference: it serves callers that must not allocate device memory.  Its
 * scratch is a fixed device array sized for PIC_SORT_STATIC_MAX particles
 * (about 17 MiB, held by every GPU that loads the library until the process
 * exits); n above that is rejected with PIC_ERR_BAD_ARG.  nx, ny and tile
 * are the arguments of pic_sorter_create; the rest, and the results, are
 * those of pic_sort.  Every call shares the array, which keeps the last
 * call's contents, so calls that overlap on the GPU race.  The first call on
 * a device (with that device current) looks up the array's address; make it
 * before any stream capture. */
#define PIC_SORT_STATIC_MAX (1 << 20)
int pic_sort_static(const float* d_x, const float* d_y, const float* d_vx, const float* d_vy, const float* d_vz,
                    int n, int nx, int ny, int tile, float* d_x_out, float* d_y_out, float* d_vx_out,
                    float* d_vy_out, float* d_vz_out, uint32_t* d_perm, int* d_count_out, int* d_tile_start,
                    void* stream);

/* ------------------------------------------------------------------ */
/* Null-collision Monte-Carlo collisions (src/MCC.py:308-415)          */
/* ------------------------------------------------------------------ */

typedef enum pic_process_type {
    PIC_ELASTIC = 0,        /* isotropic, with the 2m/M recoil loss           */
    PIC_EXCITATION = 1,     /* isotropic, loses the threshold energy          */
    PIC_IONIZATION = 2,     /* loses the threshold, splits the rest U(0.2,0.8) with a new electron, adds an ion */
    PIC_CHARGE_EXCHANGE = 3 /* ion takes a neutral Maxwellian velocity        */
} pic_process_type;

/* Cross-section tables of one species on a shared log-spaced energy grid
 * (h_energy[0..ne-1], eV, geometric); h_sigma[k] has ne values (m^2). */
typedef struct pic_mcc_species_desc {
    int nproc;
    int type[PIC_MAX_PROCESSES];
    double threshold[PIC_MAX_PROCESSES]; /* eV */
    const double* h_sigma[PIC_MAX_PROCESSES];
    int born_electron_species;           /* ionisation: species index of the new electron */
    int born_ion_species;                /* ionisation: species index of the new ion */
} pic_mcc_species_desc;

typedef struct pic_mcc_desc {
    int ne;
    const double* h_energy;              /* eV, log-spaced */
    double gas_density;                  /* m^-3 */
    double gas_temperature;              /* K */
    double gas_mass;                     /* kg */
    pic_mcc_species_desc species[PIC_MAX_SPECIES]; /* nproc = 0: no collisions */
} pic_mcc_desc;

/* Birth buffer for ionisation products: positions (grid units) and
 * velocities of new particles with their species; *count (device int) is
 * advanced atomically and may exceed capacity (the excess is dropped and
 * counted). */
typedef struct pic_birth_buffer {
    float *x, *y, *vx, *vy, *vz;
    int* species;
    int* count;
    int capacity;
} pic_birth_buffer;

typedef struct pic_mcc pic_mcc;

/* Uploads the tables; species_mass[s] in kg (m_type), dt in s.  Computes the
 * null-collision frequency nu' = n_g max_E sigma_T(E) v(E) per species. */
int pic_mcc_create(const pic_mcc_desc* desc, int nspecies, const double* species_mass, double dt, pic_mcc** out);
int pic_mcc_destroy(pic_mcc* m);
/* nu' (1/s), P_null = 1 - exp(-nu' dt) and 1/log(1 - P_null) of species s. */
int pic_mcc_query(pic_mcc* m, int s, double* nu_max, double* p_null, double* inv_log1m_p);

/* MCC.null_collision_method (src/MCC.py:308-415) on the n slots of species s,
 * after their kick: selects null-collision candidates from the Philox stream
 * (seed, step) and scatters them; ionisation products go to *births.
 * d_counters: 30 uint64 counters, see pic_sim_counters for the meaning;
 * index s*4+k = collisions of process k, 16+s = candidates, 20 = dropped
 * births, 21 = nu' overflow. */
int pic_mcc_apply(pic_mcc* m, int s, const float* d_x, const float* d_y, float* d_vx, float* d_vy, float* d_vz, int n,
                  unsigned long long seed, unsigned int step, const pic_birth_buffer* births,
                  unsigned long long* d_counters, void* stream);

/* ------------------------------------------------------------------ */
/* Fused time step (SimulationManager._init_step / _step, src/simulation.py:622-660) */
/* ------------------------------------------------------------------ */

typedef struct pic_sim pic_sim;

typedef struct pic_species_desc {
    int capacity;    /* slots allocated for this species */
    double charge;   /* C (q_type) */
    double mass;     /* kg (m_type) */
    double np2c;     /* physical particles per macro-particle */
} pic_species_desc;

typedef struct pic_sim_desc {
    int nx, ny;                 /* nodes */
    double dx, dy;              /* m */
    double dt;                  /* s */
    double eps0;                /* F/m */
    int nspecies;
    pic_species_desc species[PIC_MAX_SPECIES];
    const uint8_t* h_dirichlet; /* nx*ny, 1 = Dirichlet node */
    const double* h_phi_bc;     /* nx*ny, potential on Dirichlet nodes (V) */
    double tol;                 /* multigrid relative residual */
    int max_cycles;
    pic_mg_options mg;
    int sort_interval;          /* steps between cell sorts (0 = never) */
    int tile;                   /* cells per tile side (16) */
    const pic_mcc_desc* mcc;    /* NULL: collisionless */
    unsigned long long seed;    /* Philox key */
    int use_graph;              /* capture the step in a CUDA graph */
    int min_cycles;             /* V-cycles of a step's solve run before its first convergence test
                                   (0: test after every cycle).  In the captured step they are chained
                                   launches; each further cycle is an iteration of a WHILE node. */
    int push_kernel;            /* pic_push_kernel: how the particle pass streams the particles */
} pic_sim_desc;

/* The particle pass's streaming schemes; all do the same arithmetic and give
 * bit-identical particles and the same charge (integer tile sums). */
typedef enum pic_push_kernel {
    PIC_PUSH_RING = 0,     /* the block streams chunks through one shared three-stage ring of bulk copies
                              (the default: the fastest measured) */
    PIC_PUSH_WARP = 1,     /* each warp streams its own groups of particles through its own stage buffers
                              (asynchronous copies), E tiles by bulk tensor copies, one charge-tile atomic
                              per particle and node */
    PIC_PUSH_WARP_AGG = 2, /* as PIC_PUSH_WARP, the charge deposited with warp-aggregated atomics */
    PIC_PUSH_PIPE = 3      /* as PIC_PUSH_RING, with a producer warp and consumer warps that meet on
                              mbarriers instead of one block barrier per chunk */
} pic_push_kernel;

typedef struct pic_sim_counters {
    unsigned long long absorbed[PIC_MAX_SPECIES];
    unsigned long long collisions[PIC_MAX_SPECIES][PIC_MAX_PROCESSES];
    unsigned long long null_candidates[PIC_MAX_SPECIES];
    unsigned long long born[PIC_MAX_SPECIES];
    unsigned long long dropped_births;
    unsigned long long nu_overflow;
    int count[PIC_MAX_SPECIES];   /* slots in use */
    int last_cycles;              /* V-cycles of the last solve */
    double last_rel_res;
    long long steps;
    /* particles collected by internal electrodes (grid-line segments of
     * internal Dirichlet nodes, src/collisions.py:73-175 in the reference,
     * where the tracing exists but is unused) */
    unsigned long long electrode_absorbed[PIC_MAX_SPECIES];
    /* collision candidates that found the candidate list full (sized at
     * eight times the expected count plus 65536): they skipped their
     * collision; nonzero only if the tables' bound was far off */
    unsigned long long candidate_overflow;
} pic_sim_counters;

int pic_sim_create(const pic_sim_desc* desc, void* stream, pic_sim** out);
int pic_sim_destroy(pic_sim* sim);

/* Copy n particles of species s (device or host arrays, grid units, m/s). */
int pic_sim_load_species(pic_sim* sim, int s, const float* x, const float* y, const float* vx, const float* vy,
                         const float* vz, int n, int from_host, void* stream);

/* _init_step: deposit, solve, E, and the half kick v -= q/m E dt/2. */
int pic_sim_init(pic_sim* sim, void* stream);

/* n_steps reference steps (_step: drift, deposit, solve, E, kick, MCC).
 * The kick+MCC of the last step is left pending until the next step or
 * pic_sim_sync; the state then equals the reference's after the same steps. */
int pic_sim_step(pic_sim* sim, int n_steps, void* stream);
int pic_sim_sync(pic_sim* sim, void* stream);

/* Current device arrays of species s (the sort swaps buffers). */
int pic_sim_species_arrays(pic_sim* sim, int s, float** x, float** y, float** vx, float** vy, float** vz);
/* The reference's R / V read back to the host (src/Particles.py:283-326 keeps
 * them as device arrays the caller copies): the slots in use of species s as
 * five consecutive rows x, y, vx, vy, vz of *count floats each in h_out
 * (page-locked memory for an asynchronous copy), by device-to-host copies on
 * `stream`.  *count (the slots in use, dead ones included) is read first,
 * synchronously.  PIC_ERR_OUT_OF_CAPACITY if 5 * count > capacity. */
int pic_sim_read_particles(pic_sim* sim, int s, float* h_out, long long capacity, int* count, void* stream);
/* The cell sort of every species, now (the sort a step runs every
 * sort_interval steps; Particles2D.sort_particles_sparse,
 * src/Particles.py:550-632).  Asynchronous on `stream`. */
int pic_sim_sort(pic_sim* sim, void* stream);
/* Device pointers of phi (FP64), rho (float32, last deposit), Ex, Ey (float32). */
int pic_sim_fields(pic_sim* sim, double** phi, float** rho, float** Ex, float** Ey);
/* Synchronises `stream` and reads counters. */
int pic_sim_read_counters(pic_sim* sim, pic_sim_counters* out, void* stream);

/* Diagnostics of the current state (the reference's Diagnostics,
 * src/simulation.py:116-345, computed on the device in FP64 with a fixed
 * reduction order).  Per unit depth; rho and E of the last field solve.
 * In r-z geometry the node volumes V_j (pic_rz_density) replace dx*dy (the
 * sums are then totals, not per unit depth), the flux is through the two end
 * disks and the outer cylinder (2 pi R dx per node), the divergence is
 * (1/r) d(r E_r)/dr + dE_z/dz (2 dE_r/dr on the axis), and the momentum
 * components are sums of the axial, radial and azimuthal velocities. */
typedef struct pic_sim_diag {
    long long live[PIC_MAX_SPECIES];        /* live particles */
    double kinetic[PIC_MAX_SPECIES];        /* J: sum of 1/2 m np2c |v|^2 (vx, vy, vz) */
    double momentum[PIC_MAX_SPECIES][3];    /* kg m/s: sum of m np2c v */
    double field_energy;                    /* J: 1/2 sum rho phi dx dy */
    double gauss_flux;                      /* V: outward node sum of E along the domain boundary */
    double gauss_charge;                    /* V: sum rho dx dy / eps0 */
    double div_error_l2;                    /* V/m^2: || div E - rho/eps0 || over the nodes */
} pic_sim_diag;
int pic_sim_diagnostics(pic_sim* sim, pic_sim_diag* out, void* stream);
/* The particle vertex buffer of the reference's renderer (Renderer.update_particles,
 * src/Render.py:544-571, an OpenGL VBO written through CUDA interop) as a
 * headless device buffer: d_out[capacity][3] float32 receives, for every live
 * particle in species order and slot order, 2 (x - x_min)/(x_max - x_min) - 1,
 * the same for y (positions in metres), and the species' type (index + 1).
 * Dead slots are skipped by a stable compaction.  *count (host) receives the
 * live particles; PIC_ERR_OUT_OF_CAPACITY if they exceed capacity (the
 * first `capacity` are written).  Synchronises `stream`. */
int pic_sim_particle_buffer(pic_sim* sim, float* d_out, int capacity, double x_min, double x_max, double y_min,
                            double y_max, int* count, void* stream);
/* The launch mode its Poisson solves use (pic_mg_effective_launch_mode of
 * the simulation's solver: PIC_MG_DST or the graph loop it falls back to). */
int pic_sim_solver_mode(pic_sim* sim, int* mode);
/* Kernel launches issued by this object since creation (all phases). */
long long pic_sim_kernel_launches(pic_sim* sim);

/* Per-phase device timing with CUDA events recorded on the launch stream. */
enum {
    PIC_PHASE_BUILD = 0, /* work items, step counter, candidates */
    PIC_PHASE_PUSH = 1,  /* the fused particle kernel           */
    PIC_PHASE_MERGE = 2, /* ionisation products                 */
    PIC_PHASE_RHS = 3,   /* rho -> f                            */
    PIC_PHASE_SOLVE = 4, /* multigrid                           */
    PIC_PHASE_EFIELD = 5,/* E = -grad(phi)                      */
    PIC_PHASE_SORT = 6,  /* cell sort                           */
    PIC_NUM_PHASES = 7
};
typedef struct pic_sim_profile {
    double ms[PIC_NUM_PHASES];         /* summed device time per phase */
    long long count[PIC_NUM_PHASES];   /* timed intervals per phase */
    long long mg_cycles;               /* V-cycles in the timed steps */
} pic_sim_profile;
/* enable = 1 starts recording (and clears what was recorded), 0 stops. */
int pic_sim_set_profiling(pic_sim* sim, int enable);
/* Failure detection of the particle pass (the reference's pass has no device
 * wait to bound, src/Particles.py:359-410): polls a wait on a bulk copy into
 * shared memory makes before the pass gives up its work unit and sets a
 * device error flag (the copy in flight is still waited for, with the
 * default limit, before the block exits).  The next pic_sim_read_counters
 * returns PIC_ERR_TIMEOUT and clears the flag; the particle state of that pass
 * is then incomplete and should be reloaded.  polls < 0 restores the default
 * (2^24 polls); 0 gives up at the first wait.  The same limit goes to the
 * simulation's multigrid (pic_mg_set_wait_limit).  Captured step graphs are
 * re-captured with the new limit. */
int pic_sim_set_wait_limit(pic_sim* sim, long long polls);
/* Synchronises the device and sums the recorded intervals. */
int pic_sim_read_profile(pic_sim* sim, pic_sim_profile* out);

/* ------------------------------------------------------------------ */
/* Ensembles of independent simulations                                */
/* ------------------------------------------------------------------ */

/* Many independent simulations stepped together: one CUDA graph holds a step
 * of every member, and a conditional WHILE node repeats it, so that n steps
 * of the whole ensemble are one graph launch.  Within a step every member is
 * an independent branch: its preparation (cell sort, work items), particle
 * pass and field solve, so that one member's pass overlaps another's solve.
 * Optionally (pic_ens_set_fused_pass) one persistent particle pass takes the
 * work items of all members from one queue between the preparations and the
 * solves.
 * Each member's cell sort sits under a conditional IF node that fires when
 * the member's own step count is a multiple of its sort interval; each
 * member's multigrid loop is a nested conditional WHILE node.  Members may
 * differ in grid size, particle counts, tile, sort interval and multigrid
 * options, keep their own state, and must have been created with use_graph
 * and a graph multigrid launch mode, then loaded and initialised.  The
 * reference runs one simulation per process (src/simulation.py:562-567);
 * this has no single counterpart there.  Members stay owned by the caller
 * and must outlive the ensemble. */
typedef struct pic_ens pic_ens;
int pic_ens_create(pic_sim* const* sims, int n, pic_ens** out);
int pic_ens_destroy(pic_ens* e);
/* n steps of every member, asynchronous on `stream`: one graph launch.  A
 * member fresh from pic_sim_init takes its first step without the kick,
 * which the graph does not hold, so while any member is fresh every member
 * takes its first of the n steps eagerly. */
int pic_ens_step(pic_ens* e, int n_steps, void* stream);
/* 1 when the members' particle passes run as one persistent launch whose
 * work queue spans every member's work items, 0 (the default) when each
 * member's pass is its own launch in its branch. */
int pic_ens_fused_pass(pic_ens* e, int* fused);
/* fused = 1 runs the members' particle passes as one launch over all members
 * where that applies (every member uses PIC_PUSH_RING and the same
 * geometry); 0 gives every member's pass its own launch in its branch (the
 * default: a member's pass then overlaps another member's field solve). */
int pic_ens_set_fused_pass(pic_ens* e, int fused);

/* ------------------------------------------------------------------ */
/* Hand-written adjoint of the collisionless step                      */
/* ------------------------------------------------------------------ */

/* Gradients of L = mean over nodes of (n_s - n_target)^2, the final number
 * density of one species after N collisionless steps, with respect to the
 * potentials of electrode segments (Dirichlet node groups) and to the
 * amplitude A of an initial-velocity perturbation v_0 + A dv.  The forward
 * model is the reference's step order (src/simulation.py:622-660: drift,
 * deposit, Poisson solve, E, kick; init: deposit, solve, E, backward half
 * kick) in FP64, with absorption on the grid edges treated as a fixed mask
 * in the adjoint.  The adjoint is hand-written: the CIC deposit's transpose
 * is a gather of the weight gradients, the Poisson solve is self-adjoint (one
 * extra multigrid solve per step with zero boundary values), the leapfrog runs
 * in reverse.  The forward pass stores a checkpoint every checkpoint_every
 * steps; the backward pass recomputes each segment from its checkpoint.
 * The reference has no differentiable path; this extends its step. */
#define PIC_ADJ_MAX_SEGMENTS 16

typedef struct pic_adj pic_adj;

typedef struct pic_adj_species {
    int n;          /* particles */
    double charge;  /* C */
    double mass;    /* kg */
    double np2c;    /* physical particles per macro-particle (per unit depth) */
} pic_adj_species;

typedef struct pic_adj_desc {
    int nx, ny;                 /* nodes */
    double dx, dy, dt, eps0;
    int nspecies;
    pic_adj_species species[PIC_MAX_SPECIES];
    const uint8_t* h_dirichlet; /* nx*ny, 1 = Dirichlet (the grid edges always are) */
    const int* h_segment;       /* nx*ny: electrode segment of a Dirichlet node, or -1 */
    const double* h_phi_fixed;  /* nx*ny potentials of Dirichlet nodes without a segment (NULL: 0) */
    int nseg;                   /* electrode segments (<= PIC_ADJ_MAX_SEGMENTS) */
    int steps;                  /* N */
    int checkpoint_every;       /* C */
    int loss_species;           /* s of the loss */
    double tol;                 /* relative residual of every Poisson solve (FP64 multigrid); 0: every
                                   solve runs exactly max_cycles V-cycles (a fixed linear map of its
                                   warm start and right-hand side, smooth in the parameters) */
    int max_cycles;
} pic_adj_desc;

int pic_adj_create(const pic_adj_desc* desc, pic_adj** out);
int pic_adj_destroy(pic_adj* a);
/* Initial state of species s (device FP64 arrays of desc.species[s].n):
 * positions in grid units, velocities and the perturbation direction dv in
 * m/s (dv NULL = 0). */
int pic_adj_set_particles(pic_adj* a, int s, const double* d_x, const double* d_y, const double* d_vx,
                          const double* d_vy, const double* d_dvx, const double* d_dvy, void* stream);
/* Target number density, device FP64 nx*ny (m^-3). */
int pic_adj_set_target(pic_adj* a, const double* d_target, void* stream);
/* N steps from the initial state with segment potentials h_V[nseg] (host)
 * and amplitude A; writes the loss (synchronises). */
int pic_adj_forward(pic_adj* a, const double* h_V, double A, double* loss, void* stream);
/* dL/dV[nseg] and dL/dA at the last forward's parameters (synchronises). */
int pic_adj_backward(pic_adj* a, double* h_dV, double* h_dA, void* stream);
/* With on = 1, later forward passes reuse the absorption steps of the last
 * forward pass instead of computing them: the loss is then smooth in the
 * parameters (absorption is the fixed mask the adjoint differentiates with),
 * which is what a finite-difference check of the adjoint needs.  on = 0
 * restores absorption at the walls. */
int pic_adj_freeze_absorption(pic_adj* a, int on);
/* Device arrays of the state after the last forward pass (death: first state
 * at which a particle is outside the grid). */
int pic_adj_state(pic_adj* a, double** x, double** y, double** ux, double** uy, int** death, double** phi);

#ifdef __cplusplus
}
#endif

#endif /* PICB200_H */
