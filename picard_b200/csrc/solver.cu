// solver.cu -- CalcEpotential (CalcEpotential.f90:4-246) on the device.
//
// The host walks the sweep sequence in batches.  A batch starts at iterate a
// (the anchor), runs up to m sweeps, reduces each sweep's residual partials
// in a fixed order and reads the m residual norms back with one copy.  The
// first iterate d that meets the reference's test -- checked at the top of
// sweep d+1, so only while d+1 <= maxit -- ends the solve; if d is not the
// last iterate of the batch it is rebuilt by replaying d - a sweeps from the
// anchor.  Without a hit the loop stops after 2*maxit+1 sweeps, like the
// reference, and reports PICARD_ERR_NOT_CONVERGED.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "context.cuh"
#include "picard_gpu.h"
#include "solve_f32.cuh"

using namespace picard;

namespace {

std::mutex g_resident_mu;

// Next batch length: sweeps until the predicted hit, from the last two
// residual norms, clamped to [16, m_max].
int next_batch(double r2_prev, double r2_last, double tol2, int m_max) {
  if (!(r2_prev > 0.0) || !(r2_last > 0.0) || !(r2_last < r2_prev)) return 64;
  double per = std::log(r2_last / r2_prev);  // < 0
  double need = std::log(tol2 / r2_last) / per;
  if (!(need > 0.0)) return 16;
  double m = need * 0.9;
  if (m < 16) m = 16;
  if (m > m_max) m = m_max;
  return int(m);
}

bool passes(double r2, double tol) { return std::sqrt(r2) <= tol; }

// Device time between two events recorded on the context stream (call after
// the stream has been synchronised past the second one).
double elapsed_ms(picard_ctx* c, int a, int b) {
  float ms = 0.0f;
  if (cudaEventElapsedTime(&ms, c->ev[a], c->ev[b]) != cudaSuccess) return 0.0;
  return ms;
}

// A sweep that gave up waiting for its TMA tiles recorded kDevTimeout.
int check_timeout(picard_ctx* c) {
  PICARD_CUDA(cudaMemcpyAsync(c->h_pinned_i + 4, c->d_err, sizeof(int), cudaMemcpyDeviceToHost, c->st));
  PICARD_CUDA(cudaStreamSynchronize(c->st));
  c->stats.d2h_bytes += sizeof(int);
  if (c->h_pinned_i[4] == kDevTimeout) {
    PICARD_CUDA(cudaMemsetAsync(c->d_err, 0, sizeof(int), c->st));
    return fail(PICARD_ERR_TIMEOUT, "a bounded device wait (TMA tiles, tensor-core MMAs or a grid barrier) gave up");
  }
  return PICARD_OK;
}

int read_r2(picard_ctx* c, int count) {
  PICARD_CUDA(cudaMemcpyAsync(c->h_pinned, c->r2, sizeof(double) * count, cudaMemcpyDeviceToHost, c->st));
  PICARD_CUDA(cudaStreamSynchronize(c->st));
  c->stats.d2h_bytes += (int64_t)sizeof(double) * count;
  return PICARD_OK;
}

// ------------------------------------------------------------- FP64 sweeps
int solve_f64(picard_ctx* c, double tol, long long smax, int maxit, long long* sweeps, bool* converged) {
  const KParams& K = c->K;
  const int nb = c->G.nblocks;
  double* buf[2] = {c->U, c->U1};
  PICARD_CUDA(cudaMemcpyAsync(c->U1, c->U, sizeof(double) * K.nodes, cudaMemcpyDeviceToDevice, c->st));
  long long a = 0;
  int m = 64;
  double r2_prev = 0.0, r2_last = 0.0;
  const double tol2 = tol * tol;
  for (;;) {
    int m_eff = int(std::min<long long>(m, smax - a));
    PICARD_CUDA(cudaMemcpyAsync(c->Usnap, buf[a % 2], sizeof(double) * K.nodes, cudaMemcpyDeviceToDevice, c->st));
    PICARD_CUDA(cudaEventRecord(c->ev[0], c->st));
    for (int t = 1; t <= m_eff; ++t) {
      long long s = a + t;
      PICARD_CUDA(launch_sweep_f64(K, c->G, buf[(s - 1) % 2], buf[s % 2], c->b, c->partials + (size_t)(t - 1) * nb,
                                   c->st));
    }
    PICARD_CUDA(cudaEventRecord(c->ev[1], c->st));
    PICARD_CUDA(launch_reduce_sweeps(c->partials, nb, m_eff, c->r2, c->st));
    PICARD_TRY(read_r2(c, m_eff));
    c->stats.sweep_launches += m_eff;
    c->stats.sweep_ms += elapsed_ms(c, 0, 1);
    long long hit = -1;
    for (int t = 1; t <= m_eff; ++t) {
      long long d = a + t - 1;  // sweep a+t measured the residual of iterate d
      double r2 = c->h_pinned[t - 1];
      if (d >= 1) {
        r2_prev = r2_last;
        r2_last = r2;
        c->last_residual = std::sqrt(r2);
      }
      if (d >= 1 && d + 1 <= maxit && passes(r2, tol)) {
        hit = d;
        break;
      }
    }
    if (hit >= 0) {
      long long last = a + m_eff;
      if (hit != last - 1) {  // rebuild iterate `hit` from the anchor
        PICARD_CUDA(cudaMemcpyAsync(buf[a % 2], c->Usnap, sizeof(double) * K.nodes, cudaMemcpyDeviceToDevice, c->st));
        for (long long s = a + 1; s <= hit; ++s)
          PICARD_CUDA(launch_sweep_f64(K, c->G, buf[(s - 1) % 2], buf[s % 2], c->b, c->partials, c->st));
        c->stats.sweep_launches += hit - a;
      }
      if (hit % 2 == 1)
        PICARD_CUDA(cudaMemcpyAsync(c->U, c->U1, sizeof(double) * K.nodes, cudaMemcpyDeviceToDevice, c->st));
      *sweeps = hit;
      *converged = true;
      return PICARD_OK;
    }
    a += m_eff;
    if (a >= smax) {
      if (a % 2 == 1)
        PICARD_CUDA(cudaMemcpyAsync(c->U, c->U1, sizeof(double) * K.nodes, cudaMemcpyDeviceToDevice, c->st));
      *sweeps = a;
      *converged = false;
      return PICARD_OK;
    }
    m = next_batch(r2_prev, r2_last, tol2, c->m_max);
  }
}

// ---------------------------------------------- FP32 increment + FP64 anchor
//
// The loop is a resumable state machine (F32Solve, solve_f32.cuh) so that the
// batched loop (batch.cu) can advance many runs' solves in lockstep, running the
// sweeps of a round for all runs in one launch per sweep; solve_f32 drives one
// run with its own sweep launches.

}  // namespace

namespace picard {

// The increment ping-pongs between c->w[0] and c->w[1]; *wcur names the
// buffer holding the latest iterate, and every launch writes the other one --
// a launch never writes the buffer it reads (the two-sweep kernel included:
// its CTAs load their halos from the input while others store their tiles).

// One sweep of run c: reads w[in] and the anchor residual R[rsel], writes
// w[1 - in] and the sweep's tile partials.
static cudaError_t single_sweep(picard_ctx* c, int in, int rsel, double* partial, int w_zero) {
  const KParams& K = c->K;
  float* R[2] = {c->r, c->r + f32_elems(K)};
  const int out = 1 - in;
  if (c->G.tma && c->G.pairs)
    return launch_sweep_tma2(K, c->G, &c->tmw2[in], &c->tmr2[rsel], R[rsel], c->w[out], partial, w_zero, c->d_err,
                             c->st);
  if (c->G.tma)
    return launch_sweep_tma(K, c->G, &c->tmw[in], &c->tmr[rsel], c->w[out], partial, w_zero, c->d_err, c->st);
  return launch_sweep_f32(K, c->G, c->w[in], c->w[out], R[rsel], partial, w_zero, c->st);
}

int run_sweeps_single(picard_ctx* c, int count, int rsel, double* partial_base, int* wcur) {
  const KParams& K = c->K;
  const int nb = c->G.nblocks;
  float* R[2] = {c->r, c->r + f32_elems(K)};
  if (c->G.res) {
    // one resident launch at a time on the device: its CTAs must all be
    // resident together, which another cooperative grid could prevent
    std::lock_guard<std::mutex> lk(g_resident_mu);
    const int out = 1 - *wcur;
    PICARD_CUDA(launch_sweeps_resident(K, c->G, R[rsel], nullptr, c->w[out], c->res_faces, c->res_bar, partial_base,
                                       count, 1, c->d_err, c->st, c->wait_test));
    PICARD_CUDA(cudaStreamSynchronize(c->st));
    *wcur = out;
    return PICARD_OK;
  }
  int t = 1;
  if (c->G.tma && c->G.pairs && c->G.fused2) {
    // sweeps t and t+1 per launch
    for (; t + 1 <= count; t += 2) {
      const int out = 1 - *wcur;
      PICARD_CUDA(launch_sweep2_tma(K, c->G, &c->tmw3[*wcur], &c->tmr3[rsel], R[rsel], c->w[out],
                                    partial_base + (size_t)(t - 1) * nb, partial_base + (size_t)t * nb,
                                    t == 1 ? 1 : 0, c->d_err, c->st));
      *wcur = out;
    }
  }
  for (; t <= count; ++t) {
    PICARD_CUDA(single_sweep(c, *wcur, rsel, partial_base + (size_t)(t - 1) * nb, t == 1 ? 1 : 0));
    *wcur = 1 - *wcur;
  }
  return PICARD_OK;
}

int f32_begin(F32Solve& S, picard_ctx* c, double tol, long long smax, int maxit, double sigma) {
  const KParams& K = c->K;
  S = F32Solve();
  S.c = c;
  S.tol = tol;
  S.tol2 = tol * tol;
  S.smax = smax;
  S.maxit = maxit;
  S.sigma = sigma;
  S.V[0] = c->U;
  S.V[1] = c->U1;
  S.R[0] = c->r;
  S.R[1] = c->r + f32_elems(K);
  PICARD_CUDA(cudaMemcpyAsync(c->U1, c->U, sizeof(double) * K.nodes, cudaMemcpyDeviceToDevice, c->st));
  // anchor 0: r = (b - L U_0) / sigma
  PICARD_CUDA(launch_anchor(K, c->G, S.V[S.vcur], S.V[1 - S.vcur], nullptr, c->b, S.R[S.rcur], sigma, c->partials, 1,
                            c->st));
  S.vcur = 1 - S.vcur;
  return PICARD_OK;
}

int f32_plan(F32Solve& S) {
  S.m_eff = int(std::min<long long>(S.m, S.smax - S.a));
  return S.m_eff;
}

int f32_issue_tail(F32Solve& S) {
  picard_ctx* c = S.c;
  const KParams& K = c->K;
  const int nb = c->G.nblocks;
  // next anchor: fold w_{a+m_eff} (in w[wcur]) into V, exact FP64 residual of that iterate
  PICARD_CUDA(cudaEventRecord(c->ev[1], c->st));
  PICARD_CUDA(launch_anchor(K, c->G, S.V[S.vcur], S.V[1 - S.vcur], c->w[S.wcur], c->b, S.R[1 - S.rcur], S.sigma,
                            c->partials + (size_t)S.m_eff * nb, 0, c->st));
  PICARD_CUDA(cudaEventRecord(c->ev[2], c->st));
  PICARD_CUDA(launch_reduce_sweeps(c->partials, nb, S.m_eff + 1, c->r2, c->st));
  PICARD_CUDA(cudaMemcpyAsync(c->h_pinned, c->r2, sizeof(double) * (S.m_eff + 1), cudaMemcpyDeviceToHost, c->st));
  PICARD_CUDA(cudaMemcpyAsync(c->h_pinned_i + 4, c->d_err, sizeof(int), cudaMemcpyDeviceToHost, c->st));
  c->stats.d2h_bytes += (int64_t)sizeof(double) * (S.m_eff + 1) + (int64_t)sizeof(int);
  return PICARD_OK;
}

int f32_finish(F32Solve& S, bool timed_sweeps) {
  picard_ctx* c = S.c;
  const KParams& K = c->K;
  PICARD_CUDA(cudaStreamSynchronize(c->st));
  if (c->h_pinned_i[4] == kDevTimeout) {
    PICARD_CUDA(cudaMemsetAsync(c->d_err, 0, sizeof(int), c->st));
    return fail(PICARD_ERR_TIMEOUT, "a bounded device wait (TMA tiles, tensor-core MMAs or a grid barrier) gave up");
  }
  c->stats.sweep_launches += S.m_eff;
  if (timed_sweeps) c->stats.sweep_ms += elapsed_ms(c, 0, 1);
  c->stats.anchor_launches += 1;
  c->stats.anchor_ms += elapsed_ms(c, 1, 2);
  const double sigma = S.sigma;
  const long long an = S.a + S.m_eff;
  if (const char* v = std::getenv("PICARD_SOLVE_LOG"); v && *v && *v != '0') {
    double sum = 0.0;
    for (int t = 0; t <= S.m_eff; ++t) sum += c->h_pinned[t];
    std::fprintf(stderr, "picard solve %dx%dx%d seed=%llu a=%lld m=%d r2[1]=%.17g r2[m]=%.17g sum=%.17g\n", c->K.nx,
                 c->K.ny, c->K.nz, (unsigned long long)c->prm.seed, S.a, S.m_eff, S.m_eff > 1 ? c->h_pinned[1] : 0.0,
                 c->h_pinned[S.m_eff], sum);
  }
  long long hit = -1;
  // sweep a+t (t >= 2) measured iterate a+t-1 in FP32 (scaled by sigma^2);
  // the anchor measured iterate a+m_eff in FP64
  for (int t = 2; t <= S.m_eff + 1; ++t) {
    long long d = S.a + t - 1;
    double r2 = t <= S.m_eff ? c->h_pinned[t - 1] * sigma * sigma : c->h_pinned[S.m_eff];
    S.r2_prev = S.r2_last;
    S.r2_last = r2;
    c->last_residual = std::sqrt(r2);
    if (d >= 1 && d + 1 <= S.maxit && passes(r2, S.tol)) {
      hit = d;
      break;
    }
  }
  if (hit >= 0) {
    if (hit == an) {
      // the new anchor holds the iterate
      if (S.V[1 - S.vcur] != c->U)
        PICARD_CUDA(cudaMemcpyAsync(c->U, S.V[1 - S.vcur], sizeof(double) * K.nodes, cudaMemcpyDeviceToDevice, c->st));
    } else {
      // replay sweeps a+1..hit from the old anchor (unchanged in V[vcur])
      int wr = S.wcur;
      PICARD_TRY(run_sweeps_single(c, int(hit - S.a), S.rcur, c->partials, &wr));
      c->stats.sweep_launches += hit - S.a;
      PICARD_CUDA(launch_finalize(K, S.V[S.vcur], c->w[wr], sigma, c->U, 0, c->st));
    }
    S.sweeps = hit;
    S.converged = true;
    S.done = true;
    return PICARD_OK;
  }
  S.vcur = 1 - S.vcur;
  S.rcur = 1 - S.rcur;
  S.a = an;
  if (S.a >= S.smax) {
    if (S.V[S.vcur] != c->U)
      PICARD_CUDA(cudaMemcpyAsync(c->U, S.V[S.vcur], sizeof(double) * K.nodes, cudaMemcpyDeviceToDevice, c->st));
    S.sweeps = S.a;
    S.converged = false;
    S.done = true;
    return PICARD_OK;
  }
  S.m = next_batch(S.r2_prev, S.r2_last, S.tol2, c->m_max);
  return PICARD_OK;
}

}  // namespace picard

namespace {

int solve_f32(picard_ctx* c, double tol, long long smax, int maxit, double sigma, long long* sweeps,
              bool* converged) {
  F32Solve S;
  PICARD_TRY(f32_begin(S, c, tol, smax, maxit, sigma));
  while (!S.done) {
    f32_plan(S);
    PICARD_CUDA(cudaEventRecord(c->ev[0], c->st));
    PICARD_TRY(run_sweeps_single(c, S.m_eff, S.rcur, c->partials, &S.wcur));
    PICARD_TRY(f32_issue_tail(S));
    PICARD_TRY(f32_finish(S, true));
  }
  *sweeps = S.sweeps;
  *converged = S.converged;
  return PICARD_OK;
}

}  // namespace

namespace picard {

int epot_rhs_issue(picard_ctx* c) {
  // b = -C/(dV eps0) and ||b||^2 over the interior (CalcEpotential.f90:50-54)
  PICARD_CUDA(launch_rhs(c->K, c->C, c->b, c->red_partial, c->red_result + 4, c->st));
  PICARD_CUDA(cudaMemcpyAsync(c->h_pinned + kPinnedB2, c->red_result + 4, sizeof(double), cudaMemcpyDeviceToHost,
                              c->st));
  c->stats.d2h_bytes += sizeof(double);
  return PICARD_OK;
}

EpotSetup epot_setup(picard_ctx* c, double maxerr, int32_t maxit) {
  const KParams& K = c->K;
  EpotSetup e;
  const double b2 = c->h_pinned[kPinnedB2];
  e.bnorm = std::sqrt(b2);
  e.tol = maxerr * e.bnorm;
  e.smax = 2LL * maxit + 1;
  e.maxit = maxit;
  c->last_bnorm = e.bnorm;
  // the check at the top of sweep 1 uses r_global = ||b||^2 (CalcEpotential.f90:55-61)
  e.trivial = 1 <= maxit && std::sqrt(b2) <= e.tol;
  long long nint = (long long)K.nx * K.ny * K.nz;
  e.sigma = std::sqrt(b2 / (double)nint);
  if (!(e.sigma > 0.0)) e.sigma = 1.0;
  return e;
}

int epot_finish(picard_ctx* c, const EpotSetup& e, long long sweeps, bool converged, int32_t* sweeps_out) {
  if (e.trivial) c->last_residual = e.bnorm;
  PICARD_CUDA(launch_refresh_periodic(c->K, c->U, c->st));
  c->last_sweeps = sweeps;
  c->stats.solves += 1;
  c->stats.sweeps += sweeps;
  c->stats.last_residual = c->last_residual;
  c->stats.last_bnorm = e.bnorm;
  if (sweeps_out) *sweeps_out = int32_t(sweeps);
  if (!converged)
    return fail(PICARD_ERR_NOT_CONVERGED,
                "Jacobi reached 2*maxit+1 = " + std::to_string(e.smax) + " sweeps without meeting maxerr");
  return PICARD_OK;
}

}  // namespace picard

extern "C" int picard_gpu_calc_epotential(picard_ctx* c, double maxerr, int32_t maxit, int32_t* sweeps_out) {
  if (!c) return fail(PICARD_ERR_BAD_ARG, "ctx is NULL");
  if (maxit < 0) return fail(PICARD_ERR_BAD_ARG, "maxit must be >= 0");
  PICARD_TRY(epot_rhs_issue(c));
  PICARD_CUDA(cudaStreamSynchronize(c->st));
  const EpotSetup e = epot_setup(c, maxerr, maxit);
  long long sweeps = 0;
  bool converged = true;
  if (e.trivial) {
    sweeps = 0;
  } else if (c->solver == PICARD_SOLVER_F64) {
    PICARD_TRY(solve_f64(c, e.tol, e.smax, maxit, &sweeps, &converged));
  } else if (c->solver == PICARD_SOLVER_SPECTRAL) {
    PICARD_TRY(solve_spectral(c, e.tol, e.smax, maxit, &sweeps, &converged));
  } else {
    PICARD_TRY(solve_f32(c, e.tol, e.smax, maxit, e.sigma, &sweeps, &converged));
  }
  return epot_finish(c, e, sweeps, converged, sweeps_out);
}

// ------------------------------------------------------- sweep launch tuner
//
// Picks how the FP32 sweeps run -- the TMA sweep kernel with one CTA per tile
// and one shared-memory stage, or a persistent grid of k CTAs per SM (two
// stages, k up to the kernel's occupancy; or one stage at full occupancy),
// each with and without programmatic dependent launch; or the
// register-resident sweep with each CTA shape whose grid fits on the device
// at once -- by timing a short run of sweeps of each candidate on this
// context's own buffers.  PICARD_TUNE_LOG=1 prints the
// timings to stderr.  The shape does not change a
// single bit of the results, so the choice is free to differ from process to
// process.  Choices are cached per (grid, tile depth, device) for the life of
// the process.
namespace picard {

namespace {
struct SweepShape {
  int ctas, pdl, stages;
  int res;      // 0: TMA sweep kernel; q + 1: resident sweep with CTA shape q
  int pairs;    // TMA sweep: 1 the x-pair kernel
  int fused2;   // x-pair sweeps two per launch
  int rglobal;  // x-pair sweep, one CTA per tile: r from global memory
};
std::mutex g_tune_mu;
std::map<std::tuple<int, int, int, int, int>, SweepShape> g_tuned;

int apply_shape(picard_ctx* c, const SweepShape& sh) {
  c->G.ctas = sh.ctas;
  c->G.pdl = sh.pdl;
  c->G.stages = sh.stages;
  c->G.pairs = sh.pairs;
  c->G.fused2 = sh.fused2;
  c->G.rglobal = sh.rglobal;
  c->G.res = 0;
  if (sh.res > 0) {
    if (!resident_plan(c->K, c->G, sh.res - 1)) return fail(PICARD_ERR_STATE, "resident sweep shape does not fit");
    const long long need = resident_face_floats(c->G);
    if (need > c->res_faces_cap) {
      void* q = nullptr;
      PICARD_TRY(dev_alloc(c, &q, sizeof(float) * (size_t)need));
      c->res_faces = static_cast<float*>(q);
      c->res_faces_cap = need;
    }
    if (!c->res_bar) {
      void* q = nullptr;
      PICARD_TRY(dev_alloc(c, &q, sizeof(unsigned int)));
      c->res_bar = static_cast<unsigned int*>(q);
    }
  }
  return PICARD_OK;
}
}  // namespace

int set_resident(picard_ctx* c, int value) {
  if (value == 0) {
    c->G.res = 0;
    return PICARD_OK;
  }
  if (!c->G.tma || !c->w[0]) return fail(PICARD_ERR_STATE, "resident sweeps need open boundaries and the F32_REFINE solver");
  SweepShape sh{0, 0, 1, value, 0, 0, 0};
  JacobiGeom g = c->G;
  if (!resident_plan(c->K, g, value - 1)) return fail(PICARD_ERR_STATE, "resident sweep shape does not fit the device");
  c->G.res = 0;
  c->G.res_by = 0;
  // keep the TMA launch shape, switch the sweeps to the resident kernel
  const int ctas = c->G.ctas, pdl = c->G.pdl, stages = c->G.stages;
  sh.ctas = ctas;
  sh.pdl = pdl;
  sh.stages = stages;
  sh.pairs = c->G.pairs;
  sh.fused2 = c->G.fused2;
  sh.rglobal = c->G.rglobal;
  return apply_shape(c, sh);
}

int resident_option_value(const picard_ctx* c) {
  if (!c->G.res) return 0;
  for (int q = 0; q < kResidentShapes; ++q) {
    JacobiGeom g = c->G;
    if (resident_plan(c->K, g, q) && g.res_by == c->G.res_by && g.res_nz == c->G.res_nz) return q + 1;
  }
  return 0;
}

int tune_sweep(picard_ctx* c, bool fresh) {
  if (!c->G.tma || !c->w[0]) return PICARD_OK;
  const auto key = std::make_tuple(c->K.nx, c->K.ny, c->K.nz, c->G.zc, c->device);
  auto apply = [&](const SweepShape& sh) -> int { return apply_shape(c, sh); };
  if (const char* v = std::getenv("PICARD_SWEEP_TUNE"); v && v[0] == '0' && !fresh) {
    // no timing: the x-pair kernel, one CTA per tile, PDL (the 32-wide
    // kernel when the grid is at most one tile wide)
    return apply(SweepShape{0, 1, 1, 0, c->K.nx > 32 ? 1 : 0, 0, 0});
  }
  if (!fresh) {
    SweepShape cached;
    bool hit = false;
    {
      std::lock_guard<std::mutex> lk(g_tune_mu);
      auto it = g_tuned.find(key);
      if (it != g_tuned.end()) {
        cached = it->second;
        hit = true;
      }
    }
    if (hit) return apply(cached);
  }
  int sms = 148;
  PICARD_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device));
  std::vector<SweepShape> cand;
  for (int pairs = 0; pairs <= 1; ++pairs) {
    const int occ1 = pairs ? sweep_tma2_occupancy(c->G, 1) : sweep_tma_occupancy(c->G, 1);
    const int occ2 = pairs ? sweep_tma2_occupancy(c->G, 2) : sweep_tma_occupancy(c->G, 2);
    const int tiles = pairs ? sweep_tma2_tiles(c->K, c->G) : c->G.nblocks;
    for (int pdl = 1; pdl >= 0; --pdl) {
      cand.push_back({0, pdl, 1, 0, pairs, 0, 0});  // one CTA per tile
      if (pairs) cand.push_back({0, pdl, 1, 0, pairs, 0, 1});  // the same, r from global memory
      for (int k = 1; k <= occ2; ++k)
        if ((long long)k * sms < tiles) cand.push_back({k * sms, pdl, 2, 0, pairs, 0, 0});
      if ((long long)occ1 * sms < tiles) cand.push_back({occ1 * sms, pdl, 1, 0, pairs, 0, 0});
    }
  }
  if (c->G.zc <= 8)
    for (int pdl = 1; pdl >= 0; --pdl)
      for (int rg = 0; rg <= 1; ++rg) cand.push_back({0, pdl, 1, 0, 1, 1, rg});  // two sweeps per launch
  for (int q = 0; q < kResidentShapes; ++q) {
    JacobiGeom g = c->G;
    if (resident_plan(c->K, g, q)) cand.push_back({0, 0, 1, q + 1, 0, 0, 0});
  }
  constexpr int kReps = 24;
  std::vector<float> best(cand.size(), 1e30f);
  for (int round = 0; round < 2; ++round) {
    for (size_t q = 0; q < cand.size(); ++q) {
      PICARD_TRY(apply(cand[q]));
      float ms = 0.0f;
      if (c->G.res) {
        std::lock_guard<std::mutex> lk(g_resident_mu);
        PICARD_CUDA(launch_sweeps_resident(c->K, c->G, c->r, nullptr, c->w[0], c->res_faces, c->res_bar,
                                           c->partials, 2, 1, c->d_err, c->st));
        PICARD_CUDA(cudaEventRecord(c->ev[0], c->st));
        PICARD_CUDA(launch_sweeps_resident(c->K, c->G, c->r, nullptr, c->w[0], c->res_faces, c->res_bar,
                                           c->partials, kReps, 1, c->d_err, c->st));
        PICARD_CUDA(cudaEventRecord(c->ev[1], c->st));
        PICARD_CUDA(cudaEventSynchronize(c->ev[1]));
      } else {
        // reads w[in], writes w[1 - in] (the launch after reads what this one wrote)
        auto one = [&](int s) {
          const int in = (s - 1) % 2, out = 1 - in;
          if (c->G.fused2)  // sweeps s, s+1
            return launch_sweep2_tma(c->K, c->G, &c->tmw3[in], &c->tmr3[0], c->r, c->w[out], c->partials,
                                     c->partials + c->G.nblocks, 0, c->d_err, c->st);
          return c->G.pairs ? launch_sweep_tma2(c->K, c->G, &c->tmw2[in], &c->tmr2[0], c->r, c->w[out], c->partials,
                                                0, c->d_err, c->st)
                            : launch_sweep_tma(c->K, c->G, &c->tmw[in], &c->tmr[0], c->w[out], c->partials, 0,
                                               c->d_err, c->st);
        };
        const int step = c->G.fused2 ? 2 : 1;
        int q2 = 1;
        for (int s = 1; s <= 2 * step; s += step) PICARD_CUDA(one(q2++));
        PICARD_CUDA(cudaEventRecord(c->ev[0], c->st));
        for (int s = 1; s <= kReps; s += step) PICARD_CUDA(one(q2++));
        PICARD_CUDA(cudaEventRecord(c->ev[1], c->st));
        PICARD_CUDA(cudaEventSynchronize(c->ev[1]));
      }
      PICARD_CUDA(cudaEventElapsedTime(&ms, c->ev[0], c->ev[1]));
      best[q] = std::min(best[q], ms / kReps);
    }
  }
  PICARD_TRY(check_timeout(c));
  size_t pick = 0;
  for (size_t q = 1; q < cand.size(); ++q)
    if (best[q] < best[pick]) pick = q;
  if (const char* v = std::getenv("PICARD_TUNE_LOG"); v && *v && *v != '0') {
    for (size_t q = 0; q < cand.size(); ++q) {
      if (cand[q].res)
        std::fprintf(stderr, "picard sweep tune %dx%dx%d zc=%d: resident shape %d  %.3f us%s\n", c->K.nx, c->K.ny,
                     c->K.nz, c->G.zc, cand[q].res - 1, best[q] * 1e3, q == pick ? "  <- picked" : "");
      else
        std::fprintf(stderr,
                     "picard sweep tune %dx%dx%d zc=%d: pairs=%d fused2=%d rglobal=%d ctas=%d pdl=%d stages=%d  "
                     "%.3f us%s\n",
                     c->K.nx, c->K.ny, c->K.nz, c->G.zc, cand[q].pairs, cand[q].fused2, cand[q].rglobal, cand[q].ctas,
                     cand[q].pdl, cand[q].stages, best[q] * 1e3, q == pick ? "  <- picked" : "");
    }
  }
  PICARD_TRY(apply(cand[pick]));
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tuned[key] = cand[pick];
  return PICARD_OK;
}

}  // namespace picard
