// context.cuh -- the device state behind a picard_ctx.
#pragma once

#include <string>
#include <vector>

#include "common.cuh"
#include "grid.cuh"
#include "kernels.cuh"

namespace picard {
// Longest round of FP32 sweeps between two FP64 anchors (solve_f32.cuh): the
// host reads a round's residual norms in one copy, so fewer, longer rounds mean
// fewer host round trips and anchor passes per solve.
constexpr int kMaxSweepsPerRound = 4096;

// Scratch of the counting sort by cell (sort.cu), sized for `cap`
// particles on first use.
struct SortBuf {
  long long cap = 0;
  uint32_t* key[2] = {nullptr, nullptr};  // run keys (radix ping-pong)
  int* val[2] = {nullptr, nullptr};       // run ids
  int* run_start = nullptr;               // [runs + 1]
  int* tile_counts = nullptr;             // heads per 2,048-particle tile
  int* tile_offsets = nullptr;
  int* hist = nullptr;                    // [256][tiles of runs]
  int* hist_off = nullptr;
  int* info = nullptr;                    // runs, descents, scan totals
  int* scan_scratch = nullptr;
};
// FFT BCpotentials (bcpot_fft.cu): slice transforms of D and stage buffers.
struct BcFft;

// Closed-form Jacobi solve (spectral.cu): per-axis orthonormal bases of the
// sweep operator and the compact FP64 interior arrays the transforms use.
struct SpectralPlan {
  double* Q[3] = {nullptr, nullptr, nullptr};   // periodic axes: [n_d][n_d], row = mode
  double* QT[3] = {nullptr, nullptr, nullptr};  // transposes
  // open axes: the sine basis folded by its even/odd symmetry (spectral.cu
  // folded_basis), modes in the order [even | odd]
  int folded[3] = {0, 0, 0};
  double* Qe[3] = {nullptr, nullptr, nullptr};
  double* QeT[3] = {nullptr, nullptr, nullptr};
  double* QoR[3] = {nullptr, nullptr, nullptr};
  double* QoRT[3] = {nullptr, nullptr, nullptr};
  double* om[3] = {nullptr, nullptr, nullptr};  // a_d (2 - sigma_d) per mode
  double* T[2] = {nullptr, nullptr};            // nx*ny*nz each
  double* partial = nullptr;                    // [norm_blocks][32]
  double* sums = nullptr;                       // [32]
  unsigned int* counter = nullptr;              // blocks done in an evaluation (re-armed by the last)
  int norm_blocks = 0;
  long long evals = 0;                          // Parseval evaluations (launch pairs)
};
}  // namespace picard

struct picard_ctx {
  picard_params prm;
  picard::KParams K;
  int layout = 0, solver = 0;
  int device = 0;
  cudaStream_t st = nullptr;
  long long capacity = 0;

  // particles: two buffers of each layout's arrays (compaction ping-pong)
  picard::PartF64 f64 = {};  // the particles (one layout allocated)
  picard::PartC32 c32 = {};
  int* d_count = nullptr;    // live particle count
  int* d_err = nullptr;
  int* d_info = nullptr;     // small device results read with a count (BCoutflow window)
  long long num_local = 0;   // host mirror of *d_count

  // node arrays (plane-major, see common.cuh)
  unsigned long long* Nacc = nullptr;  // [species][nodes] fixed point
  unsigned long long* Facc = nullptr;  // [species*3][nodes], allocated on first gridify_all
  double* N = nullptr;                 // [species][nodes]
  double* F = nullptr;                 // [species*3][nodes]
  double* C = nullptr;
  double* U = nullptr;
  double* E = nullptr;                 // [3][nodes]
  float4* E32 = nullptr;               // CELL32 gather copy
  double* D = nullptr;                 // (2Nx+1)(2Ny+1)(2Nz+1)

  // Jacobi
  double* b = nullptr;
  double* U1 = nullptr;     // second FP64 iterate / anchor buffer
  double* Usnap = nullptr;  // FP64 solver: iterate at the batch start
  float* w[2] = {nullptr, nullptr};  // padded FP32 layout (grid.cuh f32_pitch)
  float* r = nullptr;                 // two padded FP32 arrays
  CUtensorMap tmw[2];                 // TMA descriptors of w[0], w[1] (w boxes)
  CUtensorMap tmr[2];                 // TMA descriptors of r, r + f32_elems (r boxes)
  CUtensorMap tmw2[2], tmr2[2];       // the same for the x-pair sweep's wider boxes
  CUtensorMap tmw3[2], tmr3[2];       // two-sweep kernel: w boxes 72 x 12 x zc+4, r boxes 72 x 10 x zc+2
  double* partials = nullptr;  // [m_max + 1][nblocks]
  double* r2 = nullptr;        // [m_max + 1]
  picard::JacobiGeom G;
  picard::SpectralPlan spec;  // SOLVER_SPECTRAL
  int m_max = picard::kMaxSweepsPerRound;
  double last_residual = 0.0, last_bnorm = 0.0;
  long long last_sweeps = 0;

  // scratch
  int* blk_counts = nullptr;     // BCoutflow block counts and offsets
  int* blk_offsets = nullptr;
  uint2* out_words = nullptr;    // BCoutflow keep words (outflow.cuh)
  int* jump[2] = {nullptr, nullptr};  // BCoutflow pointer jumping (allocated on first use)
  long long jump_cap = 0;
  int* inflow_counts = nullptr;  // fused BCinflow block counts and offsets
  int* inflow_offsets = nullptr;
  picard::InflowStage inflow_stage;  // fused BCinflow survivors (allocated on first use)
  int* cell_counts = nullptr;
  int* cell_offsets = nullptr;
  double* red_partial = nullptr;
  double* red_result = nullptr;  // [8]
  int red_blocks = 0;
  double* h_pinned = nullptr;    // [m_max + 16] host staging
  int* h_pinned_i = nullptr;     // [16]

  // register-resident sweeps (jacobi_resident.cu)
  float* res_faces = nullptr;
  unsigned int* res_bar = nullptr;
  long long res_faces_cap = 0;  // floats

  int wait_test = 0;  // PICARD_OPT_WAIT_TEST
  // counting sort by cell (sort.cu): the second particle buffer and the
  // scratch are allocated on the first sort
  int sort_every = 0;      // PICARD_OPT_SORT_EVERY
  picard::PartF64 f64b = {};
  picard::PartC32 c32b = {};
  picard::SortBuf sortbuf;
  long long sort_geom_keys = 0;
  long long stats_sorts = 0, stats_sorts_moved = 0;
  // BCpotentials method (PICARD_OPT_BCPOT_TENSOR): 0 FP64 direct sum, 1 tensor
  // cores (bcpot_tc.cu), 2 FP64 FFT convolution (bcpot_fft.cu)
  int bcpot_tensor = 0;
  picard::BcFft* bcfft = nullptr;
  void* tc_cs = nullptr;
  double* tc_partial = nullptr;

  picard::InflowTable inflow;
  std::vector<void*> allocs;

  // statistics (picard_gpu_get_stats)
  picard_stats stats = {};
  long long launches_at_reset = 0;
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  cudaEvent_t pev[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};  // phase boundaries
};

namespace picard {
int fail(int code, const std::string& msg);
int check_cuda(cudaError_t e, const char* what);
picard::KParams make_kparams(const picard_params& p);
picard::InflowTable make_inflow_table(const picard_params& p);
// Reads the device particle count into ctx->num_local after surfacing any
// device-side capacity error.
int sync_count_public(picard_ctx* c);
// The same in two halves, so that many contexts' counts travel together:
// count_issue queues the copies, count_collect waits for the context's stream.
int count_issue(picard_ctx* c);
// BCpotentials without waiting for the device: a tensor-core timeout stays in
// the context's error word, which the Jacobi solve that follows reads.
int bc_potentials_async(picard_ctx* c);
// Waits for the context's stream and reports a capacity overflow or a device
// wait that gave up, recorded in the context's error word.
int check_dev_err_public(picard_ctx* c);
int count_collect(picard_ctx* c);
// BCoutflow in place on the context's particles (wrap != 0: with the
// ParticlesTransfer periodic wrap); *d_count receives the survivors.  Does not
// synchronise.
cudaError_t launch_outflow(picard_ctx* c, int wrap);
// The fused BCinflow of `iteration`, appended at *d_count in candidate order.
// Does not synchronise.
cudaError_t launch_inflow_fused(picard_ctx* c, int iteration);
// Device memory owned by the context (zeroed, freed with it).
int dev_alloc(picard_ctx* c, void** p, size_t bytes);
// Times the launch shapes of the TMA sweep on this context's buffers and keeps
// the fastest (cached per grid and device unless `fresh`).
int tune_sweep(picard_ctx* c, bool fresh);
// PICARD_OPT_SWEEP_RESIDENT: 0 off, q + 1 resident with CTA shape q.
int set_resident(picard_ctx* c, int value);
int resident_option_value(const picard_ctx* c);
// Stable counting sort of the context's particles by cell; synchronises once
// to read the run count.
int sort_particles(picard_ctx* c);
// SOLVER_SPECTRAL (spectral.cu): device buffers of the closed-form solve,
// their size in bytes, and the solve itself (the iterate of the reference's
// stopping sweep, or of sweep smax when no iterate passes).
int spectral_alloc(picard_ctx* c);
// FFT BCpotentials (bcpot_fft.cu): device bytes of its scratch, whether every
// open face fits its shared-memory FFTs (tangential lengths up to 512 and
// 1024 cells), the launch sequence (U zeroed, the face values written; the
// slice transforms of D are computed first when D changed), and upkeep.
long long bcpot_fft_bytes(const KParams& K);
int bcpot_fft_supported(const KParams& K);
int bc_potentials_fft(picard_ctx* c);
// BCpotentials of a batch of runs: the runs with the FFT method go through one
// launch per stage for all of them on bst (rev[r]: an event per run; bev: one
// event), the others through their own method on their own streams.  Each
// run's stream is ordered after its BCpotentials; nothing waits on the host.
int bc_potentials_batch(picard_ctx** ctxs, int n, cudaStream_t bst, cudaEvent_t* rev, cudaEvent_t bev);
void bcpot_fft_invalidate(picard_ctx* c);
void bcpot_fft_free(picard_ctx* c);
long long spectral_bytes(const KParams& K);
int solve_spectral(picard_ctx* c, double tol, long long smax, int maxit, long long* sweeps, bool* converged);
// The same solve as a resumable state machine, so that a batch of runs can
// take its host round trips together: spec_begin queues the initial residual,
// the forward transform and the first Parseval evaluation; after the run's
// stream has been synchronised, spec_collect reads the evaluation and queues
// the next one, or the scaling, inverse transform and update of U (then
// done is set; spec_account books the device time once the stream has passed
// that work).
struct SpecSolve {
  picard_ctx* c = nullptr;
  double tol2 = 0.0, r2_hit = 0.0, f1 = 0.0;  // f1: ||r_1||^2 from the doubling pass
  long long smax = 0, dmax = 0, lo = 0, hi = 0;
  long long d0 = 0, step = 0, d = 0;  // pending evaluation; the accepted sweep count
  int count = 0;
  bool doubling = false, final_eval = false, done = false, converged = true;
};
int spec_begin(SpecSolve& Q, picard_ctx* c, double tol, long long smax, int maxit);
int spec_collect(SpecSolve& Q);
int spec_finish_issue(SpecSolve& Q);
int spec_apply_issue(SpecSolve& Q);
void spec_account(SpecSolve& Q);
}  // namespace picard

#define PICARD_CUDA(expr)                                          \
  do {                                                             \
    int rc_ = ::picard::check_cuda((expr), #expr);                 \
    if (rc_ != PICARD_OK) return rc_;                              \
  } while (0)
#define PICARD_TRY(expr)      \
  do {                        \
    int rc_ = (expr);         \
    if (rc_ != PICARD_OK) return rc_; \
  } while (0)
