/*
 * picard_gpu.h -- C ABI of the B200 (sm_100a) implementation of Picard's
 * per-timestep particle-in-cell loop.
 *
 * The reference (Guardiarch/Picard) is a set of Fortran 90 subroutines called
 * in a fixed order by `program picard` (picard.f90:554-674).  Every routine on
 * that path has one entry point here, with the reference subroutine it replaces
 * cited beside it.  A Fortran host binds these through an `iso_c_binding`
 * interface module (bind(C, name="...")); a C or C++ host calls them directly.
 *
 * State model.  The reference passes its state arrays (real_particles,
 * int_particles, U, E, N, F, C, D) to every subroutine.  Here the state lives
 * on the device inside a `picard_ctx`, created once from a `picard_params`
 * block; the per-subroutine entry points take the context plus the scalars the
 * reference passes that can change from call to call (dt, iteration, maxerr,
 * maxit).  Host copies in the reference's own column-major layouts are moved
 * with picard_gpu_set_particles / picard_gpu_get_particles and
 * picard_gpu_set_field / picard_gpu_get_field.
 *
 * Errors.  The reference has no status reporting.  Every entry point returns a
 * picard_status; picard_gpu_last_error() gives a message for the last failure
 * on the calling thread.  No entry point aborts the process.
 *
 * Threading.  A context is bound to one CUDA stream; calls on one context must
 * come from one host thread at a time.  Different contexts are independent.
 */
#ifndef PICARD_GPU_H
#define PICARD_GPU_H

#include <stdint.h>

#if defined(__GNUC__)
#define PICARD_API __attribute__((visibility("default")))
#else
#define PICARD_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define PICARD_MAX_SPECIES 8

typedef enum picard_status {
  PICARD_OK = 0,
  PICARD_ERR_BAD_ARG = 1,       /* argument out of range / inconsistent params   */
  PICARD_ERR_CAPACITY = 2,      /* particle count would exceed max_per_proc       */
  PICARD_ERR_NOT_CONVERGED = 3, /* Jacobi ran 2*maxit+1 sweeps without converging */
  PICARD_ERR_TIMEOUT = 4,       /* a bounded device wait gave up                  */
  PICARD_ERR_CUDA = 5,          /* CUDA runtime error (message has the details)   */
  PICARD_ERR_STATE = 6          /* call made in the wrong state                   */
} picard_status;

/* Particle storage on the device.
 * F64:    SoA FP64 positions and velocities, the reference's arithmetic.  Cell
 *         indices and the removed/wrapped particle sets match the FP64 oracle
 *         bit for bit.
 * CELL32: packed int32 CIC base-node index + 32-bit fixed-point in-cell
 *         offsets + FP32 velocity (28 B per particle + 1 B species).  The
 *         performance layout. */
typedef enum picard_layout { PICARD_LAYOUT_F64 = 0, PICARD_LAYOUT_CELL32 = 1 } picard_layout;

/* Jacobi arithmetic.
 * F64:        every sweep in FP64 (24 B per node per sweep).
 * F32_REFINE: the iterate is held as an FP64 anchor plus an FP32 increment; the
 *             FP32 sweeps advance the increment and an FP64 pass folds it into
 *             the anchor every few sweeps.  Same iterate sequence and stopping
 *             rule as the FP64 sweeps (12 B per node per sweep).
 * SPECTRAL:   the same iterate in closed form: the sweep operator is diagonal
 *             in the product of per-axis sine (open) or Fourier (periodic)
 *             bases, so the residual norm of every iterate is a Parseval sum
 *             and the iterate of the stopping sweep is one forward transform of
 *             the initial residual, a per-mode factor and one inverse
 *             transform, all in FP64.  Same stopping sweep and iterate as the
 *             FP64 sweeps, to rounding; independent of the sweep count. */
typedef enum picard_solver {
  PICARD_SOLVER_F64 = 0,
  PICARD_SOLVER_F32_REFINE = 1,
  PICARD_SOLVER_SPECTRAL = 2
} picard_solver;

/* Fields that can be copied in the reference's layouts (picard.f90:95-113). */
typedef enum picard_field {
  PICARD_FIELD_U = 0, /* U(Nx+2,Ny+2,Nz+2)            */
  PICARD_FIELD_E = 1, /* E(3,Nx+2,Ny+2,Nz+2)          */
  PICARD_FIELD_N = 2, /* N(species,Nx+2,Ny+2,Nz+2)    */
  PICARD_FIELD_C = 3, /* C(Nx+2,Ny+2,Nz+2)            */
  PICARD_FIELD_F = 4, /* F(species,3,Nx+2,Ny+2,Nz+2)  */
  PICARD_FIELD_D = 5  /* D(2Nx+1,2Ny+1,2Nz+1)         */
} picard_field;

/* Run parameters.  The first block is what picard.f90:41-302 hard-codes, for a
 * single domain (iprocs = jprocs = kprocs = 1, so Nx = Nx_local).  Species
 * index s (0-based) is the reference's species s+1: 0 = electrons, 1 = H+.
 * Two-index arrays keep the reference's memory order: v0[s][c] is v0(c+1,s+1).
 * picard_params_derive() fills the second block from the first, following
 * picard.f90:333-467; like the reference, it also rewrites density[] and ppc[]
 * (inactive species get 0, electron density and ppc follow quasi-neutrality). */
typedef struct picard_params {
  /* ---- inputs ---- */
  int32_t nx, ny, nz;          /* cells per axis (Nx_local, Ny_local, Nz_local)   */
  int32_t species;             /* active species, 2..8                            */
  int32_t max_per_proc;        /* particle capacity                               */
  int32_t xflow, yflow, zflow; /* nonzero: open axis; zero: periodic axis         */
  int32_t maxit;               /* Jacobi sweep cap (2*maxit+1 sweeps at most)     */
  int32_t produce_dt_scaled;   /* 0: ParticlesProduce.f90:70 as written (a rate
                                  per step); 1: rate multiplied by dt             */
  int32_t gyration[8], fluid[8];
  int32_t ppc[8];
  double xmin, xmax, ymin, ymax, zmin, zmax;
  double dt, maxerr;
  double mass[8], charge[8], density[8], kelvin[8];
  double v0[8][4];
  double B0[4];
  double vn[8], Qn[8], nu_i[8], nu_d[8], Ek[8];
  uint64_t seed;               /* Philox key for every stochastic step            */
  /* ---- derived (picard_params_derive) ---- */
  double Lx_min, Lx_max, Ly_min, Ly_max, Lz_min, Lz_max;
  double dxyz[3], dV;
  int32_t ipp[8], epp[8], hpp[8];
  double n2p[8], eta[8];
  double ve[4], E0[4];
  double tB[8][4], sB[8][4];
  double u0;                   /* energy-log normalisation, picard.f90:476-480    */
} picard_params;

typedef struct picard_ctx picard_ctx;

/* ---------------------------------------------------------------- params */

/* Fill the inputs with the reference defaults of picard.f90:145-302 on one
 * rank (Nx_local = Ny_local = Nz_local = 30, species = 3). */
PICARD_API int picard_params_default(picard_params* p);

/* picard.f90:333-467: domain extents, dxyz, dV, quasi-neutral electron density,
 * ipp/epp/hpp/ppc, n2p, eta, mass-weighted bulk velocity ve, motional field
 * E0 = -ve x B0, Boris factors tB and sB, energy normalisation u0. */
PICARD_API int picard_params_derive(picard_params* p);

/* ---------------------------------------------------------------- context */

PICARD_API int picard_gpu_create(const picard_params* p, int32_t layout, int32_t solver, picard_ctx** out);
PICARD_API int picard_gpu_destroy(picard_ctx* ctx);
PICARD_API int picard_gpu_synchronize(picard_ctx* ctx);
PICARD_API const char* picard_gpu_last_error(void);
/* Device bytes held by a context created with these arguments (for admission
 * by memory budget); nothing is allocated.  Not counted: buffers a context
 * allocates on first use -- the flux accumulators of GridifyAll (48 B per
 * node and species), the second particle buffer and scratch of
 * picard_gpu_sort_particles, and the pointer-jumping scratch of
 * picard_gpu_bc_outflow (8 B per removed particle, up to 8 B per particle of
 * capacity). */
PICARD_API int picard_gpu_footprint(const picard_params* p, int32_t layout, int32_t solver, uint64_t* bytes);
/* Context memory comes from the device's stream-ordered pool.  By default the
 * pool hands freed memory back to the driver at the next synchronisation, so
 * a process that creates and releases many contexts (parameter sweeps, the
 * serving loop) maps memory again for every one.  This keeps up to `bytes` of
 * freed memory in the pool of `device` for reuse (the serving loop sets its
 * budget).  No counterpart in the reference (its arrays are static). */
PICARD_API int picard_gpu_pool_keep(int32_t device, uint64_t bytes);

/* Particles in the reference layout: real_particles(8, n) column-major
 * (x, y, z, vx, vy, vz, tmp, tmp) and int_particles(n) holding the 1-based
 * species number (picard.f90:74-92). */
PICARD_API int picard_gpu_set_particles(picard_ctx* ctx, const double* real_particles,
                             const int32_t* int_particles, int32_t num_local);
PICARD_API int picard_gpu_get_particles(picard_ctx* ctx, double* real_particles, int32_t* int_particles,
                             int32_t capacity, int32_t* num_local);
PICARD_API int picard_gpu_get_num_local(picard_ctx* ctx, int32_t* num_local);

/* Fields in the reference layout (see picard_field). */
PICARD_API int picard_gpu_get_field(picard_ctx* ctx, int32_t which, double* out);
PICARD_API int picard_gpu_set_field(picard_ctx* ctx, int32_t which, const double* in);

/* ------------------------------------------- one entry per reference routine */

PICARD_API int picard_gpu_calc_distance(picard_ctx* ctx);                       /* CalcDistance.f90:1-95        */
PICARD_API int picard_gpu_particles_initialize(picard_ctx* ctx);                /* ParticlesInitialize.f90:2-125*/
PICARD_API int picard_gpu_bc_inflow(picard_ctx* ctx, int32_t iteration);        /* BCinflow.f90:2-476           */
PICARD_API int picard_gpu_advance_position(picard_ctx* ctx, double dt);         /* AdvancePosition.f90:4-19     */
PICARD_API int picard_gpu_particles_produce(picard_ctx* ctx, int32_t iteration);/* ParticlesProduce.f90:1-113   */
/* BCoutflow removes in place and leaves the particles in the order of the
 * reference's loop (each removed particle replaced by the current last one). */
PICARD_API int picard_gpu_bc_outflow(picard_ctx* ctx);                          /* BCoutflow.f90:5-87           */
PICARD_API int picard_gpu_particles_transfer(picard_ctx* ctx);                  /* ParticlesTransfer.f90:2-614  */
/* Stable counting sort of the particles by cell: by the node-centred cell
 * that holds each particle (x fastest, then y, z), particles of one cell in
 * their previous order -- the order ParticlesInitialize creates them in,
 * which the loop's deposit and gather work best on and which cell crossings,
 * BCoutflow's hole filling and appended particles wear down.  No reference
 * counterpart: it takes the place of the MPI particle migration of
 * ParticlesTransfer.f90:48-482 in keeping each domain's particles local.  A
 * permutation: every particle keeps every bit and the deposit gives the same
 * N bits.  The first call allocates a second particle buffer and scratch (up
 * to 53 (F64) or 33 (CELL32) bytes per particle of capacity plus 24 bytes per
 * particle for the runs); an array already in cell order is left in place
 * after two passes over the keys.  Synchronises once. */
PICARD_API int picard_gpu_sort_particles(picard_ctx* ctx);
PICARD_API int picard_gpu_particles_gridify(picard_ctx* ctx);                  /* ParticlesGridify.f90:1-296   */
PICARD_API int picard_gpu_particles_gridify_all(picard_ctx* ctx);               /* ParticlesGridifyAll.f90:1-455*/
PICARD_API int picard_gpu_bc_potentials(picard_ctx* ctx);                       /* BCpotentials.f90:1-145       */
/* Returns PICARD_ERR_NOT_CONVERGED after 2*maxit+1 sweeps (the reference only
 * prints "Maximum iteration reached!", CalcEpotential.f90:67-69); U holds the
 * last iterate either way.  *sweeps receives the number of sweeps done. */
PICARD_API int picard_gpu_calc_epotential(picard_ctx* ctx, double maxerr, int32_t maxit,
                               int32_t* sweeps);                     /* CalcEpotential.f90:4-246     */
PICARD_API int picard_gpu_calc_efield(picard_ctx* ctx);                         /* CalcEfield.f90:3-232         */
PICARD_API int picard_gpu_bc_fields(picard_ctx* ctx);                           /* BCfields.f90:3-94            */
PICARD_API int picard_gpu_advance_velocity(picard_ctx* ctx, double dt);         /* AdvanceVelocity.f90:6-125    */
PICARD_API int picard_gpu_advance_velocity_exp(picard_ctx* ctx, double deltat,
                                    double dt);                      /* AdvanceVelocity.f90:128-236  */
PICARD_API int picard_gpu_advance_velocity_imp(picard_ctx* ctx, double deltat,
                                    double dt);                      /* AdvanceVelocity.f90:239-347  */
/* Largest species*(Nx+2)*(Ny+2)*(Nz+2) that picard_gpu_particles_gridify_noalloc
 * accepts: its scratch is a fixed 16 MiB array of int64 accumulators. */
#define PICARD_NOALLOC_MAX_WORDS 2097152

/* The charge deposit of picard_gpu_particles_gridify for callers that cannot
 * allocate device memory when they call it -- for example a Fortran host whose
 * device arrays live in a pool another runtime (OpenACC, CUDA Fortran)
 * reserved up front, or a server that has already committed all of the HBM to
 * resident runs.  It has no counterpart in the reference: it is an extra
 * entry point of this library, not a replacement of a Picard subroutine.
 * Nothing is allocated: the caller passes device pointers to the FP64
 * positions x, y, z and the 1-based species numbers (int_particles) of
 * num_local particles, and device outputs N (species x (Nx+2)(Ny+2)(Nz+2),
 * species fastest, as ParticlesGridify's N) and C ((Nx+2)(Ny+2)(Nz+2)); the
 * work is queued on `stream` (a cudaStream_t of the current device, NULL for
 * its default stream; a stream of another device is not supported).
 * Particles are expected where the reference deposits them, after BCoutflow
 * and ParticlesTransfer: inside [min, max] on every axis.  A particle farther
 * than half a cell outside the domain on some axis (NaN included), or whose
 * species number is outside 1..species, is not deposited.
 * Scratch is one fixed array of PICARD_NOALLOC_MAX_WORDS int64 words that
 * every device holds from the first use of the library until exit; larger
 * grids are rejected with PICARD_ERR_BAD_ARG.  Each call looks up the array's
 * address on the current device (cudaGetSymbolAddress); the first call on a
 * device also loads the library's device code there, so make that first call
 * before any stream capture.  All calls share the array: calls that overlap
 * on the GPU race and must be ordered by the caller. */
PICARD_API int picard_gpu_particles_gridify_noalloc(const picard_params* p, const double* x, const double* y,
                                                    const double* z, const int32_t* int_particles,
                                                    int32_t num_local, double* N, double* C, void* stream);

/* picard.f90:651-665: out[0] = uP, out[1] = uE, out[2] = uB (un-normalised,
 * FP64), *num = num_local. */
PICARD_API int picard_gpu_energy(picard_ctx* ctx, double out[3], int32_t* num);

/* ------------------------------------------------------------ statistics */

/* Counters of the work a context has done since creation or the last
 * picard_gpu_reset_stats.  sweep_ms is the device time of the Jacobi sweep
 * kernels, taken with CUDA events on the context's stream around every batch
 * of sweeps (the hottest kernel of the loop); kernel_launches counts the
 * kernels this library launched in the process over the same interval. */
typedef struct picard_stats {
  int64_t kernel_launches;
  int64_t solves;          /* CalcEpotential calls                          */
  int64_t sweeps;          /* Jacobi iterations accepted, summed over solves */
  int64_t sweep_launches;  /* sweep kernels run (replays and overshoot too)  */
  double sweep_ms;         /* device time of those sweep launches            */
  int64_t anchor_launches; /* FP64 anchor passes (F32_REFINE solver)         */
  double anchor_ms;
  double last_residual;    /* ||b - L U|| of the last accepted iterate       */
  double last_bnorm;       /* ||b|| of the last solve                        */
  int64_t steps;           /* main-loop iterations run                       */
  int64_t particle_steps;  /* live particles summed over those iterations   */
  int64_t h2d_bytes;       /* host-to-device bytes copied by the library     */
  int64_t d2h_bytes;       /* device-to-host bytes copied by the library     */
  /* device time of the phases of picard_gpu_run_fused iterations (CUDA
   * events at the phase boundaries, host waits included): particle movement
   * (advance, produce, outflow, wrap, inflow), deposit, BCpotentials, Jacobi
   * solve, E-field + velocity push */
  double phase_ms[5];
  int64_t last_sweeps;     /* Jacobi iterations of the most recent solve     */
  int64_t spectral_transforms; /* SOLVER_SPECTRAL: 3-axis transforms run     */
  double spectral_transform_ms; /* their device time (with the initial residual
                                 * and the per-mode scaling)                   */
} picard_stats;

PICARD_API int picard_gpu_get_stats(picard_ctx* ctx, picard_stats* out);
PICARD_API int picard_gpu_reset_stats(picard_ctx* ctx);
/* The cudaStream_t every kernel of this context runs on (for callers that
 * record their own CUDA events around library calls). */
PICARD_API int picard_gpu_get_stream(picard_ctx* ctx, void** stream);

/* ---------------------------------------------------------------- options */

typedef enum picard_bcpot_method {
  PICARD_BCPOT_DIRECT = 0,
  PICARD_BCPOT_TENSOR = 1,
  PICARD_BCPOT_FFT = 2
} picard_bcpot_method;

typedef enum picard_option {
  /* BCpotentials method (picard_bcpot_method).  0: FP64 direct sum (the
   * default of the F64 layout).  1: tensor cores (three-way BF16 split, FP32
   * accumulation folded into FP64 every 512 K-values).  2: FP64 FFT
   * convolution over each face's tangential axes (the default of the CELL32
   * layout where every open face is at most 512 x 1024 cells, else 1). */
  PICARD_OPT_BCPOT_TENSOR = 0,
  /* Launch shape of the TMA Jacobi sweep (open boundaries with the F32_REFINE
   * solver).  It never changes a result bit.  SWEEP_CTAS: > 0 persistent grid
   * of that many CTAs, -1 one CTA per tile, 0 re-run the launch tuner (which
   * picks both knobs at context creation).  SWEEP_PDL: 1 programmatic
   * dependent launch between consecutive sweeps, 0 plain stream order.
   * SWEEP_STAGES: shared-memory stages per CTA, 1 or 2 (2 prefetches the
   * CTA's next tile). */
  PICARD_OPT_SWEEP_CTAS = 1,
  PICARD_OPT_SWEEP_PDL = 2,
  PICARD_OPT_SWEEP_STAGES = 3,
  /* Register-resident sweeps (one cooperative launch per batch of sweeps, w
   * in registers, r in shared memory): 0 off (the TMA kernel with the shape
   * above), 1..5 on with CTA shape 0..4 (32 x 8 x 8 up to 32 x 32 x 32 nodes)
   * when that grid fits on the device, else PICARD_ERR_STATE.  Never changes
   * a result bit. */
  PICARD_OPT_SWEEP_RESIDENT = 4,
  /* TMA sweep tile width: 0 32-wide tiles, one node per thread; 1 64-wide
   * tiles, two x-adjacent nodes per thread in packed FP32 pair arithmetic.
   * Never changes a result bit. */
  PICARD_OPT_SWEEP_PAIRS = 5,
  /* 1: x-pair sweeps two at a time (one launch computes sweeps s and s+1 of
   * a tile, the intermediate iterate in shared memory); 0 one per launch.
   * Never changes a result bit. */
  PICARD_OPT_SWEEP_FUSED = 6,
  /* Test of the bounded device waits.  1: the grid barrier of the
   * register-resident sweep (PICARD_OPT_SWEEP_RESIDENT) waits for one
   * arrival more than its grid makes, with a poll limit of 2^14 polls, so
   * every CTA's wait runs out and returns; the solve then fails with
   * PICARD_ERR_TIMEOUT and the context stays usable.  0 (the default): off.
   * Nothing else uses it. */
  PICARD_OPT_WAIT_TEST = 7,
  /* 1: the x-pair sweep reads r from global memory and stages only the w box
   * (with one CTA per tile and one stage, or two sweeps per launch; otherwise
   * ignored); 0 r box by TMA.  Never changes a result bit. */
  PICARD_OPT_SWEEP_R_GLOBAL = 8,
  /* k > 0: picard_gpu_run_fused sorts the particles by cell
   * (picard_gpu_sort_particles) in the ParticlesTransfer slot of every
   * iteration divisible by k; 0 (the default): never.  The per-subroutine
   * loops never sort (their particles stay in the reference's order). */
  PICARD_OPT_SORT_EVERY = 9
} picard_option;
/* Reads an option's current value (SWEEP_CTAS: 0 means one CTA per tile). */
PICARD_API int picard_gpu_get_option(picard_ctx* ctx, int32_t option, int32_t* value);
PICARD_API int picard_gpu_set_option(picard_ctx* ctx, int32_t option, int32_t value);

/* ----------------------------------------------------------- main loop */

/* One line of the reference's energy log (picard.f90:667-671). */
typedef void (*picard_log_fn)(int32_t iteration, double time, int32_t num_local,
                              double uP_norm, double uE_norm, double uB_norm, void* user);

/* picard.f90:554-674 call for call, iterations iter_start+1 .. iter_end, with
 * the write-step branch off (writeFields = writeParticles = .false.).  log_fn
 * (may be NULL) is called every log_interval iterations.  *sweeps_total
 * (may be NULL) accumulates Jacobi sweeps. */
PICARD_API int picard_gpu_run(picard_ctx* ctx, int32_t iter_start, int32_t iter_end, int32_t log_interval,
                   picard_log_fn log_fn, void* user, int64_t* sweeps_total);

/* The same iterations through the fused device path: the velocity push of one
 * step and the position advance of the next in one particle pass, BCoutflow
 * with the periodic wrap in place, inflow candidates generated, advanced and
 * filtered on the device and appended after BCoutflow in candidate order.
 * Results equal picard_gpu_run's within the parity tolerances (the same
 * particles; the inflow ones sit at the end instead of before the produced
 * ones), and the particle order is deterministic: two runs from the same state
 * hold the same particles in the same slots. */
PICARD_API int picard_gpu_run_fused(picard_ctx* ctx, int32_t iter_start, int32_t iter_end,
                         int64_t* sweeps_total);

/* Batched parameter sweep: iterations iter_start+1 .. iter_end of the fused
 * loop for n independent contexts (runs) together.  Every run's particle
 * phases are issued on its own stream before any is waited for, and the
 * Jacobi sweeps of all runs advance in lockstep rounds with one launch per
 * sweep over the tiles of every run (open boundaries, F32_REFINE solver;
 * other runs solve on their own).  Each run's result is bit-identical to
 * picard_gpu_run_fused on that run alone.  sweeps_total (may be NULL) is an
 * array of n counters accumulating each run's Jacobi sweeps. */
PICARD_API int picard_batch_run_fused(picard_ctx** ctxs, int32_t n, int32_t iter_start, int32_t iter_end,
                                      int64_t* sweeps_total);
/* One iteration of every run of a batch whose runs are at different points:
 * run r takes iteration iterations[r] (the continuous-batching step of the
 * serving loop, where runs join and leave between steps). */
PICARD_API int picard_batch_step(picard_ctx** ctxs, int32_t n, const int32_t* iterations, int64_t* sweeps_total);

#ifdef __cplusplus
}
#endif

#endif /* PICARD_GPU_H */
