/* METHOD-B200 C ABI: the per-timestep hot path of METHOD on one B200.
 *
 * Plain C types only (no CUDA or torch types), so that the reference's C++
 * classes, a ctypes loader or any FFI can bind it.  One handle owns one
 * simulation's device-resident state in METHOD's own layout,
 * ID(var,i,j,k) = var*Nx*Ny*Nz + i*Ny*Nz + j*Nz + k (Project/CPU/Include/simData.h:10),
 * ghost cells included, so host arrays of the reference can be uploaded and
 * downloaded with plain copies.
 *
 * Every entry point returns an mth_status.  Calls on one handle are ordered on
 * the handle's CUDA stream; calls that return data to the host synchronise.
 * Errors raised on the device (non-convergence) are sticky until read by
 * mth_sync / mth_get_stats, which return them as status codes.
 */
#ifndef METHOD_B200_H
#define METHOD_B200_H

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  MTH_OK = 0,
  MTH_ERR_C2P = 1,        /* primitive recovery did not converge (srrmhd.cc:576-579) */
  MTH_ERR_IMPLICIT = 2,   /* SSP2 implicit stage did not converge (SSP2.cc:89-98, 134-143) */
  MTH_ERR_INVALID = 3,    /* bad configuration or argument (simData.cc:100-106, weno.cc:13-20) */
  MTH_ERR_CUDA = 4        /* CUDA runtime error (no device, launch failure, ...) */
} mth_status;

enum { MTH_SRMHD = 0, MTH_SRRMHD = 1, MTH_HYBRID = 2 };       /* Model subclasses */
enum { MTH_OUTFLOW = 0, MTH_PERIODIC = 1, MTH_FLOW = 2 };     /* Bcs subclasses */
enum { MTH_RK2 = 0, MTH_RKSPLIT = 1, MTH_SSP2 = 2,             /* TimeIntegrator subclasses */
       MTH_SSP3 = 3, MTH_SSP2322 = 4, MTH_RKSPLIT2 = 5 };       /* (IMEX: SRRMHD only) */
enum { MTH_PLAIN_FP64 = 0, MTH_MIXED = 1 };                   /* precision of the flux path */
enum { MTH_GUESS_PREVIOUS = 0, MTH_GUESS_MLP = 1, MTH_GUESS_COLD = 2 }; /* C2P initial guess */
enum { MTH_C2P_HYBRD = 0, MTH_C2P_NEWTON = 1 };               /* C2P solver */

/* The Data constructor arguments (Project/CPU/Include/simData.h:205-218) plus
 * the choice of Model, WENO order, Bcs and TimeIntegrator. */
typedef struct {
  int model;                 /* MTH_SRMHD / MTH_SRRMHD / MTH_HYBRID */
  int nx, ny, nz;            /* interior cells; ny = 0 for 1D, nz = 0 for 2D */
  double xmin, xmax, ymin, ymax, zmin, zmax;
  double endTime, cfl;
  int Ng;                    /* ghost cells, >= WENO shift + 1 */
  double gamma, sigma, cp;
  int weno_order;            /* 3 or 5 (Weno3 / Weno5) */
  int bcs;                   /* MTH_OUTFLOW / MTH_PERIODIC / MTH_FLOW */
  int integrator;            /* MTH_RK2 / MTH_RKSPLIT / MTH_SSP2 / MTH_SSP3 / MTH_SSP2322 /
                                MTH_RKSPLIT2 (rkSplit2ndOrder.cc) */
  int precision;             /* MTH_PLAIN_FP64 / MTH_MIXED */
  int guess;                 /* MTH_GUESS_PREVIOUS / MTH_GUESS_MLP */
  int device;                /* CUDA device ordinal */
  int functional_sigma;      /* Data::functionalSigma: conductivity sigma * D^sigma_exp */
  double sigma_exp;          /* Data::gam (simData.h:86; the reference's default is 12) */
  /* x-slab decomposition (the counterpart of ParallelEnv's split over
   * nxRanks, Project/CPU/Src/parallelEnv.cc:16-127): when x_slab is set,
   * this handle holds interior columns [x_offset, x_offset + nx) of a domain
   * of x_global_nx columns whose bounds are xmin, xmax, and its x halo rows
   * are filled by the caller (mth_halo_*) instead of by the boundary
   * conditions.  RK2, RKSplit and SSP2 only. */
  int x_slab;
  int x_global_nx;
  int x_offset;
  /* 1: the REGIME resistive extension of SRMHD (REGIME.cc, Wright & Hawke
   * 2019) as RKSplit's model extension, as `REGIME ext(&data, &fvs);
   * RKSplit ti(&data, &model, &bcs, &fvs, &ext)`: SRMHD, RKSplit, one or two
   * dimensions; sigma is its conductivity.  With model MTH_HYBRID it is the
   * Hybrid model's useREGIME instead (hybrid.h:76). */
  int regime;
  /* MTH_HYBRID (Hybrid(data, sigmaCrossOver, sigmaSpan, useREGIME),
   * hybrid.cc:26-77): the conductivity at which the ideal and resistive
   * models are blended half and half, and the half-width of the blend. */
  double sigma_crossover;
  double sigma_span;
} mth_config;

typedef struct {
  long long c2p_cells;        /* cells solved by primitive recovery */
  long long c2p_evals;        /* residual evaluations spent by primitive recovery */
  long long c2p_unconverged;  /* cells left unconverged (after the SRMHD retry) */
  long long implicit_cells;   /* cells solved by SSP2 implicit stages */
  long long implicit_evals;   /* residual evaluations of the implicit stages */
  long long implicit_failed;  /* implicit solves that did not converge */
  long long steps;            /* time steps taken */
  double t, dt;               /* simulation time and last time step */
  int iters;                  /* Data::iters */
  long long c2p_fallbacks;    /* mixed form: Newton cells that fell back (guess / Powell hybrid) */
  long long implicit_fallbacks; /* mixed form: implicit cells re-solved by the Powell hybrid */
} mth_stats;

typedef struct mth_handle mth_handle;

/* Data + Model + Bcs + FluxMethod + TimeIntegrator construction, with the
 * reference's validation (Data::initData, WenoBase::checkSufficientGhostZones).
 * Allocates all device state. */
mth_status mth_create(const mth_config* cfg, mth_handle** out);
mth_status mth_destroy(mth_handle* h);
const char* mth_last_error(const mth_handle* h);

/* Extents: Nx, Ny, Nz, Ncons, Nprims, Naux, dims. */
mth_status mth_get_dims(const mth_handle* h, int* dims7);

/* InitialFunc + Simulation::set: takes the primitive state of every cell
 * (Nprims*Nx*Ny*Nz doubles) and derives cons/aux on the device
 * (Model::primsToAll, srmhd.cc:573-673 / srrmhd.cc:358-510) then applies the
 * boundary conditions (simulation.cc:80-101). */
mth_status mth_set_prims(mth_handle* h, const double* prims_host);

/* Whole-state upload / download in the reference layout.  Any pointer may be
 * NULL.  Download materialises ghost cells first (Bcs::apply). */
mth_status mth_upload(mth_handle* h, const double* cons, const double* prims, const double* aux);
mth_status mth_download(mth_handle* h, double* cons, double* prims, double* aux);

/* Bcs::apply (boundaryConds.h:46) on the device state. */
mth_status mth_apply_bcs(mth_handle* h);
/* Model::primsToAll on the device state. */
mth_status mth_prims_to_all(mth_handle* h);
/* Model::getPrimitiveVars (model.h:80) on the device state, guess = current prims/aux. */
mth_status mth_c2p(mth_handle* h);
/* FluxMethod::F (flux.h:72): fnet of the current state into fnet_host
 * (Ncons*Nx*Ny*Nz doubles, interior written, rest zero). */
mth_status mth_flux_F(mth_handle* h, double* fnet_host);
/* Model::sourceTerm of the current state (every cell) into source_host. */
mth_status mth_source(mth_handle* h, double* source_host);
/* Model::fluxVector (model.h:121) of the current state for direction dir
 * (0, 1, 2), every cell, into f_host (Ncons*Nx*Ny*Nz doubles).  As in the
 * reference, SRRMHD's z direction leaves f_host's Sz plane as it was. */
mth_status mth_flux_vector(mth_handle* h, int dir, double* f_host);

/* Model::getPrimitiveVarsSingleCell (model.h:85) applied to n independent
 * cells, with no simulation handle.  Arrays are variable-major with stride n
 * (cons[v*n + q]), host memory; prims/aux carry the initial guess in
 * (SRMHD: rho, v, aux h; SRRMHD: aux[10] = rho h W^2) and the solution out.
 * SRMHD solves with MINPACK hybrd1 at `tol` (the reference uses 1.4e-8,
 * srmhd.cc:308); SRRMHD uses the reference's secant iteration (tol unused).
 * Returns MTH_ERR_C2P when any cell did not converge. */
mth_status mth_c2p_cells(int model, double gamma, double sigma, long long n, const double* cons,
                         double* prims, double* aux, double tol, int device);

/* TimeIntegrator::step (timeInt.h:61) with an explicit dt; enqueued as one
 * CUDA graph launch, asynchronous. */
mth_status mth_step(mth_handle* h, double dt);
/* Simulation::updateTime (simulation.cc:104-133) n times: dt from cfl with the
 * slow start and end-time clamp, then step, t += dt, iters++. */
mth_status mth_update_time(mth_handle* h, int n);
/* Simulation::evolve without output: updateTime until t >= endTime. */
mth_status mth_evolve(mth_handle* h);
/* ---- x-slab decomposition: one domain over several handles (one per GPU).
 * A step is a sequence of parts that end where the reference applies the
 * boundary conditions to an intermediate state (TimeIntegrator::finalise):
 * RK2 / RKSplit 2 (predictor | corrector), SSP2 3 (stage 1 | stage 2 |
 * combination); SSP3 / SSP2322 1.  After each part the caller exchanges the
 * Ng-deep x halos of that part's state, which is what ParallelBcs::apply
 * does through swapGhostBuffers (Project/CPU/Src/parallelBoundaryConds.cc:
 * 11-30): pack the Ng interior rows next to each x face into a device
 * buffer of mth_halo_bytes, send them to the neighbour, unpack what the
 * neighbours sent into the ghost rows; at a physical outflow x face,
 * mth_halo_outflow fills the ghost rows instead.  part -1 is the handle's
 * main state (after mth_set_prims / mth_upload).  Buffers are device memory
 * laid out [cons vars | prims vars | aux vars][Ng rows][Ny*Nz]; every copy
 * is ordered on the handle's stream. */
mth_status mth_step_parts(const mth_handle* h, int* n_parts);
mth_status mth_step_part(mth_handle* h, double dt, int part);
/* Simulation::updateTime's dt for the next step, and its t += dt, iters++. */
mth_status mth_next_dt(const mth_handle* h, double* dt);
mth_status mth_advance_time(mth_handle* h, double dt);
mth_status mth_halo_bytes(const mth_handle* h, unsigned long long* bytes);
mth_status mth_halo_pack(mth_handle* h, int part, int side, void* dst);
mth_status mth_halo_unpack(mth_handle* h, int part, int side, const void* src);
mth_status mth_halo_outflow(mth_handle* h, int part, int side);

/* Waits for queued work and returns the first device-side error, if any. */
mth_status mth_sync(mth_handle* h);
mth_status mth_get_stats(mth_handle* h, mth_stats* s);
mth_status mth_reset_stats(mth_handle* h);

/* Drop-in form of TimeIntegrator::step(cons, prims, aux, dt) (timeInt.h:61)
 * on HOST arrays, the reference's own calling convention: uploads the
 * arrays the step reads, runs one step, downloads all three, and returns the
 * step's status.  The mixed form on 2D grids reads cons and only part of
 * prims / aux (SRMHD RK2: all prims, aux 0, 1, 4-8; SRRMHD RK2: prims 1-4,
 * aux 4-8, 10; SRRMHD SSP2: aux 10); every other case uploads all three.
 * Pinned host memory (mth_pin_host) makes the copies asynchronous DMA. */
mth_status mth_step_host(mth_handle* h, double* cons, double* prims, double* aux, double dt);
/* Bytes mth_step_host copies to and from the device per call. No reference
 * counterpart (accounting for the host-array step). */
mth_status mth_step_host_bytes(mth_handle* h, unsigned long long* h2d, unsigned long long* d2h);
/* Page-locks / releases a host range for fast copies (cudaHostRegister). */
mth_status mth_pin_host(void* ptr, unsigned long long bytes);
mth_status mth_unpin_host(void* ptr);

/* Runs queued work on the caller's CUDA stream (a cudaStream_t passed as an
 * opaque pointer; NULL restores the handle's own stream).  Graph launches,
 * copies and eager kernels of this handle are then ordered on that stream. */
mth_status mth_set_stream(mth_handle* h, void* stream);

/* Per-kernel timing of one step, run eagerly `reps` times with CUDA events
 * around every launch.  Fills up to max_out records; *n_out receives the
 * number of distinct kernels.  `bytes_per_launch` is the kernel's algorithmic
 * HBM traffic (each input array element read once, each output written once). */
typedef struct {
  char name[40];
  int launches;
  double total_ms;
  double bytes_per_launch;
} mth_kernel_time;
mth_status mth_profile_step(mth_handle* h, double dt, int reps, mth_kernel_time* out,
                            int max_out, int* n_out);

/* ---- Learned C2P guess (no counterpart in the reference) ------------------
 * An 8 -> 64 -> 64 -> 64 -> 2 ReLU network maps scale-free features of an
 * SRMHD conserved state to (log10(rho h W^2 / D), v^2).  Parameters are FP32
 * master values in a packed layout of MTH_MLP_NPARAM floats; the device runs
 * it with BF16 weights and activations and FP32 accumulation.  Statistics
 * are MTH_MLP_NSTAT floats: feature mean[8], 1/std[8], target mean[2], std[2]. */
#define MTH_MLP_NPARAM 9928
#define MTH_MLP_NSTAT 20
typedef struct {
  unsigned long long seed;
  long long n_samples;  /* training pairs the solver generates (primsToAll of random states) */
  int iterations;       /* Adam steps */
  int batch;            /* samples per step (multiple of 128 recommended) */
  float lr;             /* peak learning rate, cosine decay */
  double gamma;         /* adiabatic index */
  int model;            /* MTH_SRMHD (default) or MTH_SRRMHD: which feature map and pairs */
} mth_mlp_train_config;
/* Trains on the device with the project's forward/backward kernels. */
mth_status mth_mlp_train(const mth_mlp_train_config* cfg, float* params, float* stats,
                         float* final_loss, int device);
/* Gradient of the mean-squared error over n samples (host arrays: x [n][8]
 * standardised features, t [n][2] standardised targets) -> grad[MTH_MLP_NPARAM]. */
mth_status mth_mlp_grad(const float* params, int n, const float* x, const float* t, float* grad,
                        float* loss, int device);
/* Standardised outputs y [n][2] of standardised features x [n][8]. */
mth_status mth_mlp_forward(const float* params, int n, const float* x, float* y, int device);
/* The same on the tcgen05 tensor-core path (M = 128 products, accumulators in
 * tensor memory): the same weights and rounding points, FP32 sums in the
 * tensor cores' order.  No reference counterpart (the learned guess). */
mth_status mth_mlp_forward_tc(const float* params, int n, const float* x, float* y, int device);
/* Solver-generated training pairs: features [n][8], targets [n][2] (raw,
 * not standardised), optionally the conserved [9][n] and generating
 * primitive [8][n] states.  Output pointers may be host or device memory
 * (copies use unified addressing). */
mth_status mth_mlp_make_pairs(long long n, unsigned long long seed, double gamma, float* feat,
                              float* tgt, double* cons, double* prims, int device);
/* The same for SRRMHD: random primitive states (the distributions above,
 * plus E = -v x B + a departure of 10^U(-3,0) |B|) through SRRMHD primsToAll;
 * conserved [14][n], primitive [11][n]. */
mth_status mth_mlp_make_pairs_srrmhd(long long n, unsigned long long seed, double gamma,
                                     float* feat, float* tgt, double* cons, double* prims,
                                     int device);
/* Installs a trained network in a handle (precision MTH_MIXED, guess
 * MTH_GUESS_MLP); it must have been trained for the handle's model.  SRMHD:
 * Newton recovery starts from its Z; SRRMHD: the recovery and the implicit
 * stages' inner recoveries start from its Z (the previous state's Z is the
 * fallback, then the reference secant / Powell-hybrid solve). */
mth_status mth_set_mlp(mth_handle* h, const float* params, const float* stats);

/* Batched SRMHD primitive recovery of n independent cells (device arrays,
 * variable-major with stride n): cons [9][n] in; prims [8][n] / aux [13][n]
 * carry the previous-state guess in and the solution out.  method
 * MTH_C2P_HYBRD is the reference's Powell hybrid (tol 1.49011612e-7);
 * MTH_C2P_NEWTON is the 1D Newton in rho h W^2, falling back to the
 * previous-state guess and then to the Powell hybrid.  guess selects the
 * start: previous state, the network (mlp_params / mlp_stats, host arrays),
 * or a cold start from the conserved state alone. */
typedef struct {
  long long cells, iterations, unconverged, fallbacks;
} mth_c2p_batch_stats;
mth_status mth_c2p_batch(double gamma, long long n, const double* cons, double* prims,
                         double* aux, int method, int guess, const float* mlp_params,
                         const float* mlp_stats, void* stream, mth_c2p_batch_stats* stats);

/* Reusable workspace for batched primitive recovery: the same solve as
 * mth_c2p_batch without per-call allocation or synchronisation.  Create it
 * for up to max_n cells on a device (allocates the guess planes and
 * counters), install a trained network once if MTH_GUESS_MLP is used, then
 * enqueue runs on any stream of that device; each run resets the counters,
 * which mth_c2p_ctx_stats reads back (synchronising the stream; returns
 * MTH_ERR_C2P if cells stayed unconverged).  Runs that overlap on the GPU
 * share the workspace and race: order them on one stream.  No counterpart in
 * the reference (see mth_c2p_batch). */
typedef struct mth_c2p_ctx mth_c2p_ctx;
mth_status mth_c2p_ctx_create(long long max_n, int device, mth_c2p_ctx** out);
mth_status mth_c2p_ctx_destroy(mth_c2p_ctx* c);
mth_status mth_c2p_ctx_set_mlp(mth_c2p_ctx* c, const float* params, const float* stats);
mth_status mth_c2p_ctx_run(mth_c2p_ctx* c, double gamma, long long n, const double* cons,
                           double* prims, double* aux, int method, int guess, void* stream);
mth_status mth_c2p_ctx_stats(mth_c2p_ctx* c, void* stream, mth_c2p_batch_stats* stats);

/* Largest number of interior cells mth_c2p_srmhd_noalloc accepts per call. */
#define MTH_NOALLOC_MAX_CELLS (1 << 20)

/* SRMHD primitive recovery (the grid C2P of mth_c2p, with its neighbour-
 * average retry) for callers that may not allocate device memory: a host
 * application that owns all device memory through its own fixed pool, or a
 * latency-critical loop that cannot afford cudaMalloc and the synchronisation
 * it may bring.  No counterpart in the reference (its C2P is a host method).
 * All pointers but `unconverged` are device arrays in the reference layout
 * for a grid of nx x ny x nz interior cells with Ng ghosts (ny = 0: 1D,
 * nz = 0: 2D): cons (9 vars), prims_guess / aux_guess (the previous state,
 * 8 / 13 vars), prims / aux (8 / 13 vars, out; may alias the guesses),
 * solution (2 vars, in/out, the per-cell (v^2, rho h W^2) the retry averages,
 * ghost cells included; keep it across calls as the reference's
 * SRMHD::solution).  Work is enqueued on `stream` (a cudaStream_t, NULL =
 * default stream) of the calling thread's current context; the call
 * allocates nothing.  The failure queue and counters live in one fixed device
 * array (about 4 MiB per GPU, held until exit) shared by all calls: calls
 * that overlap on the GPU race on it, so order them on one stream.  Its
 * address is looked up once per CUDA context, by the first call made in that
 * context; make that call before any stream capture.  `unconverged` (host
 * memory, may be NULL): when given, the call waits for the stream and stores
 * the number of cells the retry left unconverged (the reference only prints
 * these, srmhd.cc:495-498; the status stays MTH_OK, as for mth_c2p).  Returns
 * MTH_ERR_INVALID, with a message on stderr, when the grid has more than
 * MTH_NOALLOC_MAX_CELLS interior cells or cell ids that overflow an int. */
mth_status mth_c2p_srmhd_noalloc(int nx, int ny, int nz, int Ng, double gamma,
                                 const double* cons, const double* prims_guess,
                                 const double* aux_guess, double* prims, double* aux,
                                 double* solution, void* stream, long long* unconverged);

/* SerialSaveData output (serialSaveData.cc:31-246) of the current state:
 * `which` is a mask of MTH_SAVE_* bits; files are
 * dir/Conserved/cons<app>.dat, dir/Primitive/prims<app>.dat,
 * dir/Auxiliary/aux<app>.dat, dir/Domain/domain<app>.dat and
 * dir/Constants/constants<app>.dat, byte for byte what the reference writes
 * (values formatted as "%.16f" on the device).  The directories must exist;
 * a file that cannot be opened gives MTH_ERR_INVALID (the reference exits).
 * The constants' dt is the last updateTime step, or the constructor's CFL dt
 * before the first one. */
enum { MTH_SAVE_CONS = 1, MTH_SAVE_PRIMS = 2, MTH_SAVE_AUX = 4, MTH_SAVE_DOMAIN = 8,
       MTH_SAVE_CONSTS = 16, MTH_SAVE_ALL = 31 };
mth_status mth_save_text(mth_handle* h, const char* dir, const char* app, int which);

/* Zero-copy access for frameworks that manage device memory themselves:
 * device pointers of cons, prims, aux (reference layout), valid until
 * mth_destroy. */
mth_status mth_device_state(mth_handle* h, double** cons, double** prims, double** aux);

/* ---- Ensembles: independent 2D simulations of uneven sizes advanced together.
 * No counterpart in the reference, where each Simulation owns one grid and
 * a parameter study runs them one after another.  Every member is a
 * Simulation of its own configuration (its own grid, dt from its own CFL
 * condition, t, iters: Simulation::updateTime per member); one ensemble step
 * advances every member by one of its own time steps.  Members are SRMHD with
 * MTH_RK2 (either precision) or SRRMHD with MTH_SSP2 (MTH_MIXED only); all
 * share precision, WENO order and device; nz must be 0, ny > 0.  Each phase
 * of the step is one persistent launch over a work list spanning all
 * members, and the whole step is one CUDA graph (dt is computed on the
 * device).  A member's results are identical to a single Simulation of the
 * same configuration (plain: the reference's, bit for bit). */
typedef struct mth_ensemble mth_ensemble;
mth_status mth_ensemble_create(const mth_config* cfgs, int n, mth_ensemble** out);
mth_status mth_ensemble_destroy(mth_ensemble* e);
const char* mth_ensemble_last_error(const mth_ensemble* e);
/* Initial primitive state of member m (host, Nprims*Nx*Ny*Nz doubles of that
 * member); derives cons/aux, applies the boundaries, resets t and iters. */
mth_status mth_ensemble_set_prims(mth_ensemble* e, int m, const double* prims_host);
/* Host copies of member m's state (any pointer may be NULL). */
mth_status mth_ensemble_download(mth_ensemble* e, int m, double* cons, double* prims,
                                 double* aux);
/* Installs a trained guess network (host arrays, MLP_NPARAM parameters and
 * MLP_NSTAT statistics as mth_mlp_train returns them) for ensembles created
 * with guess MTH_GUESS_MLP (precision MTH_MIXED): SRMHD members then start
 * every primitive recovery from its guess, as mth_set_mlp does for one
 * simulation. */
mth_status mth_ensemble_set_mlp(mth_ensemble* e, const float* params, const float* stats);
/* The same for the SRRMHD members: a network trained with model MTH_SRRMHD
 * seeds their recoveries and the inner recoveries of their implicit stages. */
mth_status mth_ensemble_set_mlp_srrmhd(mth_ensemble* e, const float* params, const float* stats);
mth_status mth_ensemble_set_stream(mth_ensemble* e, void* stream);
/* Autotuner, on the ensemble's own members: for each member size class
 * (nx <= 96, <= 192, larger) it times the flux phase at tile heights 4, 8,
 * 16 (rows of 32 cells) x persistent grids (one CTA per tile, 4 or 2 CTAs per
 * SM), and the recovery phases at 4, 8, 16 CTAs per SM, `reps` timed
 * launches each, and keeps the fastest; the tile heights are returned in ti3
 * (may be NULL).  Runs kernels on the current state but changes no member's
 * state. */
mth_status mth_ensemble_autotune(mth_ensemble* e, int reps, int* ti3);
/* What the autotuner chose, and the summed phase times (ms per repetition)
 * of the default choice (tile height 8, one CTA per tile, 8 CTAs per SM)
 * against the chosen one. */
typedef struct {
  int tile_height[3];  /* per size class */
  int flux_ctas[3];    /* flux-phase grid per size class; 0 = one CTA per tile */
  int cell_ctas;       /* grid of the cell phases */
  float default_ms, tuned_ms;
} mth_tuning_report;
mth_status mth_ensemble_tuning(const mth_ensemble* e, mth_tuning_report* t);
/* Enqueues n_steps ensemble steps (asynchronous; see mth_ensemble_sync). */
mth_status mth_ensemble_step(mth_ensemble* e, int n_steps);
/* Per-phase timing of `reps` ensemble steps run eagerly (one phase at a time,
 * CUDA events around each) into up to max_out records (bytes_per_launch 0);
 * *n_out receives the number of distinct phases.  The steps advance the
 * members like mth_ensemble_step. */
mth_status mth_ensemble_profile(mth_ensemble* e, int reps, mth_kernel_time* out, int max_out,
                                int* n_out);
/* Waits for the enqueued steps; returns MTH_ERR_C2P / MTH_ERR_IMPLICIT if any
 * member's solve failed (the reference's exceptions). */
mth_status mth_ensemble_sync(mth_ensemble* e);
mth_status mth_ensemble_stats(mth_ensemble* e, int m, mth_stats* s);
/* Total interior cells of all members, and the tile heights in use. */
mth_status mth_ensemble_info(const mth_ensemble* e, long long* interior_cells, int* ti3);

#ifdef __cplusplus
}
#endif
#endif /* METHOD_B200_H */
