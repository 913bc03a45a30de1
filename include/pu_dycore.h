/* pu_dycore: C-ABI of the B200 dynamical core.
 *
 * A drop-in for the reference's compressible, hydrostatically stratified
 * WENO finite-volume dycore, modules::Dynamics_Euler_Stratified_WenoFV
 * (model/modules/dynamics_rk.h:25-1355), at WENO order 9 on one GPU.
 *
 * The reference module is stateless and keeps everything in the coupler's
 * DataManager; its three entry points are
 *     void init(core::Coupler &)                      dynamics_rk.h:917-1246
 *     void time_step(core::Coupler &, real dt_phys)   dynamics_rk.h:103-137
 *     real compute_time_step(core::Coupler const &)   dynamics_rk.h:57-64
 * Here a handle (pu_dycore) holds the grid, options and device-resident
 * state; the coupler's arrays are passed in as a pu_state_view (host or
 * device pointers).  A host-side C++ wrapper with the reference's exact
 * module API is in porturb_b200/cpp/dynamics_rk.h.
 *
 * Conventions:
 *   - every function returns PU_OK (0) or a PU_ERR_* code; pu_last_error()
 *     gives a message (the reference aborts instead: Options.h:122-148,
 *     dynamics_rk.h:799, ParallelComm.h:315-323);
 *   - 3-D arrays are C-order (nz, ny, nx) doubles, the coupler's layout
 *     (dynamics_rk.h:1269-1277, 1322-1330);
 *   - one CUDA stream per handle (pu_config.stream, NULL = the legacy
 *     default stream); calls are asynchronous on that stream unless stated;
 *   - no internal host threads; a handle is not thread-safe (the reference's
 *     Coupler is not either).
 */
#ifndef PU_DYCORE_H
#define PU_DYCORE_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PU_MAX_TRACERS 4   /* water_vapor + up to three more advected tracers */
#define PU_ORD 9           /* WENO order; halo width PU_HS = (PU_ORD-1)/2 */
#define PU_HS 4

typedef enum {
  PU_OK = 0,
  PU_ERR_INVALID = 1,      /* bad argument or option (the reference aborts) */
  PU_ERR_CUDA = 2,         /* a CUDA call failed */
  PU_ERR_NONFINITE = 3,    /* the state became NaN/Inf during a step */
  PU_ERR_STATE = 4,        /* call out of order (e.g. time_step before init) */
  PU_ERR_NOMEM = 5,        /* device allocation failed */
  PU_ERR_UNSUPPORTED = 6,  /* configuration outside what this build supports */
  PU_ERR_TRANSPORT = 7     /* a host transport callback reported a failure */
} pu_status;

typedef enum { PU_BC_PERIODIC = 0, PU_BC_PRECURSOR = 1, PU_BC_WALL = 2 } pu_bc;
typedef enum { PU_F32 = 0, PU_F64 = 1 } pu_precision;
typedef enum { PU_WENO_PLAIN = 0, PU_WENO_LEARNED = 1 } pu_weno_mode;
/* Where coupler arrays live; PU_MEM_AUTO asks the library to inspect the
 * pointers (cudaPointerGetAttributes). */
typedef enum { PU_MEM_HOST = 0, PU_MEM_DEVICE = 1, PU_MEM_AUTO = 2 } pu_mem;

/* Grid, tracer registry and the coupler options the dycore reads
 * (dynamics_rk.h:508-531, 747, 930-933, 1262-1266, 1315-1319; defaults from
 * sc_init.h:31-51 and abl_neutral.cpp:36-47). */
typedef struct pu_config {
  int nx, ny, nz;                          /* coupler.get_nx/ny/nz */
  double dx, dy, dz;                       /* coupler.get_dx/dy/dz */
  int ntracers;                            /* coupler.get_num_tracers */
  int tracer_positive[PU_MAX_TRACERS];     /* add_tracer(...,positive,...) */
  int tracer_adds_mass[PU_MAX_TRACERS];    /* add_tracer(...,adds_mass,...) */
  int idWV;                                /* option "idWV": index of water_vapor */
  double R_d, R_v, cp_d, gamma_d, C0, grav;/* options of the same names */
  double cfl;                              /* option "cfl" (reference default 0.60) */
  double immersed_power;                   /* option "immersed_power" (default 5) */
  double latitude;                         /* option "latitude" in degrees (default 0) */
  int bc_x, bc_y, bc_z;                    /* options "bc_x/bc_y/bc_z" as pu_bc */
  int enable_gravity;                      /* option "enable_gravity" (default true) */
  int weno_all;                            /* option "weno_all" (default true) */
  int precision;                           /* pu_precision: stencil arithmetic type */
  int weno_mode;                           /* pu_weno_mode */
  int device;                              /* CUDA device ordinal */
  void *stream;                            /* cudaStream_t, or NULL */
  int z_chunk;                             /* 0: the tiled z kernel (FP32 with weno_all) or the z
                                              march with its own chunk; > 0: the z march with
                                              this many levels per work item (the same results) */
  int thread_loads;                        /* 0: the stage kernels stage their tiles through TMA
                                              where the grid allows it (nx % 4 == 0); 1: every
                                              tile is loaded by the threads (the same results) */
  int imm_all_levels;                      /* 0: on an immersed domain the stage kernels take the
                                              immersed code only on the levels (z chunks) that an
                                              immersed flag reaches; 1: on every level (the same
                                              results) */
  int serial_io;                           /* 0: pu_dycore_time_step on host arrays overlaps the
                                              copies with the steps, chunk by chunk, where the
                                              path allows it (FP32, weno_all, plain weights, walls
                                              in z, nz >= 64), and a decomposed tile with a
                                              transport runs its interior x/y tiles while its
                                              halos cross; 1: copies in, steps, copies out, and
                                              every x/y tile after the exchange (the same
                                              results) */
} pu_config;

/* The coupler-side state: density_dry, uvel, vvel, wvel, temp and the tracer
 * arrays in the order of the tracer registry. */
typedef struct pu_state_view {
  double *rho_d, *uvel, *vvel, *wvel, *temp;
  double *tracers[PU_MAX_TRACERS];
  int mem; /* pu_mem: where the pointers live */
} pu_state_view;

/* Global FP64 integrals of the dycore state, accumulated with compensated
 * (Neumaier) sums on the GPU.  Volumes in m^3, energies in J. */
typedef struct pu_diag {
  double mass;            /* sum rho dV */
  double rho_theta;       /* sum rho*theta dV */
  double kinetic;         /* sum 0.5 |rho u|^2 / rho dV */
  double internal;        /* sum p/(gamma-1) dV */
  double potential;       /* sum rho g z dV, z at cell centres */
  double total_energy;    /* kinetic + internal + potential */
  double tracer_mass[PU_MAX_TRACERS]; /* sum rho_q dV */
} pu_diag;

typedef struct pu_dycore pu_dycore;

/* Version of this library (major*10000 + minor*100 + patch). */
int pu_version(void);

/* Message of the last failed call on this host thread. */
const char *pu_last_error(void);

/* Creates a handle and allocates its device buffers.  Replaces the
 * construction of Dynamics_Euler_Stratified_WenoFV plus the option reads of
 * its members (dynamics_rk.h:25-39, 508-531). */
int pu_dycore_create(const pu_config *cfg, pu_dycore **out);

/* Frees the handle and its device buffers. */
int pu_dycore_destroy(pu_dycore *h);

/* init(coupler), dynamics_rk.h:917-1246: converts the coupler state, takes
 * the horizontal-mean hydrostatic profiles (FP64 on the GPU), extends them
 * isentropically into the z halos, computes the edge profiles, and builds
 * the immersed-boundary halos, flags (any_immersed within 10 cells) and
 * relaxation time scales from immersed_proportion ((nz,ny,nx) doubles in
 * `mem`; NULL = no immersed cells).  Synchronous. */
int pu_dycore_init(pu_dycore *h, const pu_state_view *coupler, const double *immersed_proportion, int mem);

/* init(coupler) when the coupler also holds windmill_proj_weight
 * (dynamics_rk.h:1019-1025): the projection weight ((nz,ny,nx) doubles in
 * `mem`, NULL = none) is added to a copy of immersed_proportion before the
 * immersed halos, flags and time scales are built.  A projection without
 * immersed_proportion is PU_ERR_INVALID (the reference aborts on the missing
 * entry). */
int pu_dycore_init_windmill(pu_dycore *h, const pu_state_view *coupler, const double *immersed_proportion,
                            const double *windmill_proj_weight, int mem);

/* compute_time_step(coupler), dynamics_rk.h:57-64: cfl*min(dx,dy,dz)/450. */
int pu_dycore_compute_time_step(const pu_dycore *h, double *dt);

/* time_step(coupler, dt_phys), dynamics_rk.h:103-137: converts the coupler
 * state in, runs ncycles = ceil(dt_phys/dt_dyn) SSPRK3 steps of
 * dt_phys/ncycles, converts back into the same arrays.  Synchronous; returns
 * PU_ERR_NONFINITE if the state became non-finite.  ncycles may be NULL.
 * On host arrays the copies overlap the steps chunk by chunk (see
 * pu_config.serial_io); the results are the same either way. */
int pu_dycore_time_step(pu_dycore *h, pu_state_view *coupler, double dt_phys, int *ncycles);

/* convert_coupler_to_dynamics (dynamics_rk.h:1304-1352) into the resident
 * state, and convert_dynamics_to_coupler (dynamics_rk.h:1251-1299) out of it.
 * store_state is synchronous and reports PU_ERR_NONFINITE like time_step. */
int pu_dycore_load_state(pu_dycore *h, const pu_state_view *coupler);
int pu_dycore_store_state(pu_dycore *h, pu_state_view *coupler);

/* nsteps calls of time_step_rk_3_3 (dynamics_rk.h:279-367) with step dt_dyn
 * on the resident state.  Asynchronous. */
int pu_dycore_advance(pu_dycore *h, double dt_dyn, int nsteps);

/* Conserved variables of the resident state (rho, rho*u, rho*v, rho*w,
 * rho*theta as (5,nz,ny,nx) and tracers as (ntr,nz,ny,nx), absolute values,
 * the reference's state/tracers arrays without halos).  Synchronous. */
int pu_dycore_get_conserved(pu_dycore *h, double *state, double *tracers, int mem);
int pu_dycore_set_conserved(pu_dycore *h, const double *state, const double *tracers, int mem);

/* The hydrostatic profiles hy_{dens,theta,pressure}_cells ((nz+2*PU_HS)
 * values each) and hy_{dens,theta,pressure}_edges (nz+1 each), as the values
 * the stencil arithmetic uses.  Any pointer may be NULL. */
int pu_dycore_get_hydrostasis(pu_dycore *h, double *dens_cells, double *theta_cells, double *pressure_cells,
                              double *dens_edges, double *theta_edges, double *pressure_edges);

/* Overwrites the cell profiles and recomputes the edge profiles: the
 * dycore's restart hook (dynamics_rk.h:1235-1242).  The resident state is
 * kept in absolute terms across the change. */
int pu_dycore_set_hydrostasis(pu_dycore *h, const double *dens_cells, const double *theta_cells,
                              const double *pressure_cells);

/* FP64 compensated global integrals of the resident state.  Synchronous. */
int pu_dycore_diagnostics(pu_dycore *h, pu_diag *out);

/* The fields the dycore adds to every output/restart file (its write hook,
 * dynamics_rk.h:1193-1233): density_pert = rho - hy_dens_cells,
 * theta_pert = rho*theta/rho - hy_theta_cells and
 * pressure_pert = C0*(rho*theta)^gamma - hy_pressure_cells, formed from the
 * coupler arrays v as convert_coupler_to_dynamics forms rho and rho*theta
 * (dynamics_rk.h:1304-1352), FP64, (nz,ny,nx) each; outputs in memory `mem`
 * (PU_MEM_HOST, PU_MEM_DEVICE or PU_MEM_AUTO).  Synchronous. */
int pu_dycore_perturbations(pu_dycore *h, const pu_state_view *v, double *density_pert, double *theta_pert,
                            double *pressure_pert, int mem);

/* Waits for all work of the handle; returns PU_ERR_NONFINITE if a step
 * produced a non-finite value since the last check. */
int pu_dycore_synchronize(pu_dycore *h);

/* Number of kernels this handle has launched since creation (for launch
 * accounting in benchmarks). */
long long pu_dycore_kernel_launches(const pu_dycore *h);

/* ---- Learned WENO weights -------------------------------------------------
 * No counterpart in the reference: a network (9 -> 32 -> 32 -> 5, ReLU,
 * softmax; bfloat16 weights and activations, FP32 biases and accumulation)
 * that maps a stencil normalised to its local range (the convention of
 * dynamics_rk.h:42-53) to the nonlinear weights of the left edge
 * (WenoLimiter.h:382-403); the right edge uses the mirrored stencil.  It is
 * trained on stencils harvested from the handle's resident state with the
 * plain limiter's weights as targets.  Parameter vector (PU_MLP_PARAMS floats):
 * W1 (32x9, row major), b1 (32), W2 (32x32), b2 (32), W3 (5x32), b3 (5). */
#define PU_MLP_PARAMS 1541
typedef struct pu_learn_stats {
  double loss_first, loss_last; /* mean cross-entropy of the first and last batch */
  long long steps, samples;     /* optimiser steps, harvested stencils */
  double ms;                    /* GPU time of the training loop */
} pu_learn_stats;

/* Appends n stencils of the resident state (random field, direction and cell,
 * away from immersed cells and z walls) with their plain left-edge weights to
 * the training set.  Synchronous. */
int pu_dycore_learned_harvest(pu_dycore *h, long long n, unsigned long long seed);
/* Adam steps on random batches of the training set (hand-written forward,
 * backward and Adam kernels), then installs the weights for inference. */
int pu_dycore_learned_train(pu_dycore *h, int steps, int batch, double lr, unsigned long long seed,
                            pu_learn_stats *out);
int pu_dycore_learned_get_weights(pu_dycore *h, float *theta);
int pu_dycore_learned_set_weights(pu_dycore *h, const float *theta);
/* Network weights of n normalised stencils (host arrays n*9 -> n*5).  With
 * use_mma the tensor-core path also returns the right-edge weights (wr). */
int pu_dycore_learned_eval(pu_dycore *h, const float *x, long long n, float *wl, float *wr, int use_mma);
/* Mean cross-entropy and its gradient over the n given samples (host arrays):
 * the training kernels' forward and backward pass, for checking. */
int pu_dycore_learned_gradient(pu_dycore *h, const float *x, const float *t, long long n, float *grad,
                               double *loss);
/* Selects PU_WENO_PLAIN or PU_WENO_LEARNED for the following steps.  Learned
 * needs trained or loaded weights, the FP32 build and weno_all (it replaces
 * the nonlinear limiter, which otherwise runs only near immersed cells):
 * PU_ERR_STATE / PU_ERR_UNSUPPORTED otherwise.  In learned mode the stencil
 * kernels evaluate the network with tensor-core MMAs inside the
 * reconstruction; stencils with an immersed cell or a z wall within reach,
 * or with a normalised neighbour jump above the threshold, use the plain
 * limiter. */
int pu_dycore_set_weno_mode(pu_dycore *h, int mode);
/* Largest normalised neighbour jump |x[m+1]-x[m]| (of the stencil scaled to
 * [0,1]) given learned weights; default 0.5; values >= 1 disable the check. */
int pu_dycore_learned_set_threshold(pu_dycore *h, double max_jump);
/* Stencils reconstructed with learned weights and stencils that fell back to
 * the plain limiter since the last call (counters are reset). */
int pu_dycore_learned_counts(pu_dycore *h, long long *learned, long long *fallback);

/* Per-kernel timing with CUDA events recorded on the handle's stream around
 * every stencil-kernel launch while enabled (no counterpart in the reference,
 * whose timers are YAKL's, dynamics_rk.h:104-106).  Kinds: 0 = x/y flux
 * kernel, 1 = z flux + stage kernel, 2 = everything else.  Enabling resets
 * the totals; pu_dycore_profile_read synchronizes. */
#define PU_PROFILE_KINDS 3
typedef struct pu_profile {
  double ms[PU_PROFILE_KINDS];
  long long launches[PU_PROFILE_KINDS];
} pu_profile;
int pu_dycore_profile(pu_dycore *h, int enable);
int pu_dycore_profile_read(pu_dycore *h, pu_profile *out);

/* A time step that allocates no device memory.
 *
 * No counterpart in the reference.  It is for callers that cannot call
 * cudaMalloc: a host model whose own allocator has already reserved the GPU's
 * memory, or a plug-in that runs inside a time loop where device allocation is
 * not allowed.  pu_dycore_create allocates its buffers, so such callers use this
 * entry point instead: it performs what pu_dycore_time_step does (convert the
 * coupler state in, ncycles = ceil(dt_phys/dt_dyn) SSPRK3 steps, convert back
 * into the same arrays) for an FP32 dycore without immersed cells, given the
 * configuration and the hydrostatic cell profiles (hy_dens_cells,
 * hy_theta_cells, hy_pressure_cells: nz+2*PU_HS host doubles each, e.g. from
 * pu_dycore_get_hydrostasis of an earlier init, or a restart file).
 *   - coupler arrays must be device memory (PU_MEM_DEVICE, or PU_MEM_AUTO
 *     resolving to device); there is no staging;
 *   - all working memory comes from one static device array of
 *     PU_NOALLOC_SCRATCH_BYTES bytes, which every GPU that loads the library
 *     holds until the process exits; grids that need more return
 *     PU_ERR_UNSUPPORTED (about 110 bytes per cell with two tracers, i.e. up
 *     to roughly 600k cells);
 *   - the configuration does not say whether the domain has immersed cells,
 *     and this call cannot detect them: on an urban or turbine domain it
 *     returns the step of the same grid without immersed cells (no error);
 *     such domains need pu_dycore_time_step;
 *   - the first call on a device looks up that array's device address
 *     (cudaGetSymbolAddress, with the device current) and keeps it; make that
 *     first call before any stream capture.  Resetting the device
 *     (cudaDeviceReset) while the library is loaded is not supported: the
 *     kept address would belong to the context that the reset destroyed;
 *   - every call shares the one array and it keeps the previous call's
 *     contents (only the error word is cleared per call), so calls whose GPU
 *     work overlaps -- on different streams or host threads -- race;
 *   - synchronous; returns PU_ERR_NONFINITE like pu_dycore_time_step. */
#define PU_NOALLOC_SCRATCH_BYTES (64u << 20)
int pu_dycore_time_step_noalloc(const pu_config *cfg, const double *hy_dens_cells, const double *hy_theta_cells,
                                const double *hy_pressure_cells, pu_state_view *coupler, double dt_phys,
                                int *ncycles);

/* The FP32 order-9 limiter (WenoLimiter<float,9>::compute_limited_edges,
 * WenoLimiter.h:349-437, in this library's arithmetic) on n stencils of 9
 * consecutive floats: the left and right edge values of each.  flags[i]
 * (NULL: all 1): bit 0 do_map, bit 1 imm_L, bit 2 imm_R.  variant 0: the
 * scalar form (the z march, the FP64-free fallbacks); 1: the packed
 * two-stencil form of the x/y kernel (both give the same bits); 2, 3: the
 * linear forms on the tensor cores (tcgen05.mma kind::tf32, three-term split,
 * A in shared memory / in tensor memory; the two give the same bits and
 * agree with the FP32 forms to rounding; not used by the dycore kernels);
 * 4: the packed one-edge form the x/y kernel uses for the halo cells that
 * close a tile's rows, on pairs (2i, 2i+1): the right edge of stencil 2i and
 * the left edge of stencil 2i+1, each the same bits as variants 0 and 1 (the
 * pair's other two outputs are NaN).
 * Host or device arrays (mem); synchronous, on the current device. */
int pu_weno9_edges_f32(const float *stencils, const unsigned char *flags, long long n, int variant, float *qL,
                       float *qR, int mem);

/* The learned weights' input convention on n stencils of 9 floats (host
 * arrays; synchronous, on the current device): x = (s - min)/(max - min), all
 * zeros when max - min <= 1e-20, and jump = the largest |x[m+1] - x[m]|, the
 * acceptance check of the learned path.  It follows the limiter's normalize
 * (WenoLimiter.h:85-96, threshold 1e-20), the form of the dycore's unused
 * normalize (dynamics_rk.h:42-53, which floors the range at 1e-10 instead);
 * the scale is applied as a multiply by the correctly rounded reciprocal of
 * the range. */
int pu_learned_normalize_f32(const float *stencils, long long n, float *x, float *jump);

/* The bounded wait of the stage kernels' TMA staging, made to run out (a
 * failure-detection check; no reference counterpart): one block waits on an
 * mbarrier whose announced copies are never issued, for at most limit_us
 * microseconds (0: the stage kernels' own limit, 20 ms; at most 1 s), and
 * gives up.  *completed = 1 if the wait saw the copies complete (it cannot;
 * the stage kernels report such a give-up as PU_ERR_CUDA), *ms the kernel's
 * time, *cycles thread 0's clock cycles in the wait (ms and cycles may be
 * NULL).  The context stays usable.  Synchronous, on the current device. */
int pu_check_bounded_wait(int limit_us, int *completed, double *ms, long long *cycles);

/* ---------------------------------------------------------------------------
 * Domain decomposition across GPUs (coupler.h:132-229): a handle can be one
 * (px, py) tile of an nproc_x x nproc_y grid of tiles over an nx_glob x
 * ny_glob domain; its cfg.nx, cfg.ny are the tile's sizes and the coupler
 * arrays it takes are the tile's.  Every stage the tile sends the 5 columns
 * (rows) of the stage input next to each x (y) edge to the neighbouring tile
 * and receives the neighbour's, which its x/y kernel reads beyond its edges
 * (the halo exchange of coupler.h:985-1165 and the edge exchange of
 * dynamics_rk.h:808-912).  Neighbours wrap periodically; precursor
 * conditions apply at the global edges only.  Init sums the hydrostatic
 * profiles over all tiles and builds the immersed flags from a 12-cell halo
 * of immersed_proportion.  Tiles must be at least 12 cells wide in x and y
 * (ny_glob == 1: one tile row, ny = 1); tiles in one column of the grid have
 * the same nx, tiles in one row the same ny.  Plain WENO only (no learned
 * weights).
 * ------------------------------------------------------------------------- */
typedef struct pu_decomp {
  int nproc_x, nproc_y;      /* tile grid; rank = py*nproc_x + px */
  int px, py;                /* this tile */
  long long nx_glob, ny_glob;
} pu_decomp;

#define PU_NCCL_ID_BYTES 128

/* The process grid the reference's coupler picks for nranks tasks
 * (coupler.h:148-171): nproc_y is the divisor of nranks whose
 * nproc_y/(nranks/nproc_y) is closest to ny_glob/nx_glob (the first of equals),
 * nproc_x = nranks/nproc_y; ny_glob == 1 gives nranks x 1.  Host only. */
int pu_decomp_process_grid(int nranks, long long nx_glob, long long ny_glob, int *nproc_x, int *nproc_y);
/* First index and size of tile p of nproc along an axis of n_glob cells
 * (coupler.h:176-183: beg = round(n_glob/nproc*p), end = round(n_glob/nproc*(p+1))-1).
 * Host only. */
int pu_decomp_tile(long long n_glob, int nproc, int p, long long *beg, long long *n);
/* Ranks of the tiles beyond the x-, x+, y-, y+ edges of tile (px, py)
 * (coupler.h:203-214).  Host only. */
int pu_decomp_neighbors(const pu_decomp *d, int nbr[4]);

/* A new NCCL unique id (PU_NCCL_ID_BYTES bytes) for pu_dycore_set_decomposition;
 * one rank makes it and the host broadcasts it to the others.  NCCL is loaded
 * from libnccl.so.2 on first use (the copy already in the process, if any). */
int pu_nccl_get_unique_id(unsigned char *id);

/* Makes the handle a tile of a decomposed domain; call before pu_dycore_init.
 * With an NCCL id, every tile is a separate rank (one process or thread per
 * GPU) and this call, init and every time step are collective over the
 * nproc_x*nproc_y ranks (it creates the NCCL communicator and checks that
 * the tiles' sizes fit together, failing on every rank alike if they do
 * not).  With id NULL the tiles of the grid are handles of one process on
 * one stream, driven by the pu_dycore_group_* calls. */
int pu_dycore_set_decomposition(pu_dycore *h, const pu_decomp *d, const unsigned char *nccl_id);

/* A host transport for a decomposed tile: the caller's own message layer
 * (MPI, a Python process group, ...) moves the halo slabs and the init
 * reductions through host memory, where the reference's coupler calls MPI
 * (ParallelComm.h send_receive / all_reduce, used by coupler.h:985-1165 for
 * the halos and dynamics_rk.h:976-978 for the column sums).  The library
 * calls these from the thread that drives the handle, during set-up, init and
 * every stage, with pinned host buffers it owns; each returns 0 on success
 * (anything else makes the dycore call return PU_ERR_TRANSPORT).
 *   exchange: for every direction d (x-, x+, y-, y+) with bytes[d] > 0, send
 *     snd[d] to rank nbr[d] and receive from rank nbr[d] into rcv[d]; what a
 *     rank sends as snd[d] its neighbour receives as rcv[d ^ 1] (a rank can be
 *     its own neighbour, and the x- and x+ neighbours can be one rank);
 *   allreduce_sum_f64: buf[0..n) = its sum over all ranks, in place; the same
 *     order of summation on every rank keeps the tiles' profiles identical;
 *   allgather: out = the `bytes` bytes of `in` of every rank, in rank order. */
typedef struct pu_host_transport {
  int (*exchange)(void *user, void *const *snd, void *const *rcv, const size_t *bytes, const int *nbr);
  int (*allreduce_sum_f64)(void *user, double *buf, size_t n);
  int (*allgather)(void *user, const void *in, void *out, size_t bytes);
  void *user;
} pu_host_transport;

/* Makes the handle tile (px, py) of a decomposed domain whose ranks talk
 * through the host transport t (copied; its user pointer must stay valid
 * while the handle lives); call before pu_dycore_init.  Like the NCCL form,
 * this call, init and every time step are collective over the
 * nproc_x*nproc_y ranks, and this call checks with allgather that the tiles
 * fit together, failing on every rank alike if they do not. */
int pu_dycore_set_decomposition_host(pu_dycore *h, const pu_decomp *d, const pu_host_transport *t);

/* init, advance and time_step of an in-process group: hs holds the n =
 * nproc_x*nproc_y tiles (any order) made with pu_dycore_set_decomposition(h,
 * d, NULL), on one device and one stream; views[i], props[i], projs[i] are
 * tile i's coupler arrays, immersed_proportion and windmill_proj_weight
 * (props / projs NULL, or entries NULL, for none).  The tiles advance stage
 * by stage together (pack, exchange by device copies, x/y and z kernels). */
int pu_dycore_group_init(pu_dycore *const *hs, int n, const pu_state_view *views, const double *const *props,
                         const double *const *projs, int mem);
int pu_dycore_group_advance(pu_dycore *const *hs, int n, double dt, int nsteps);
int pu_dycore_group_time_step(pu_dycore *const *hs, int n, pu_state_view *views, double dt_phys, int *ncycles);

#ifdef __cplusplus
}
#endif

#endif /* PU_DYCORE_H */
