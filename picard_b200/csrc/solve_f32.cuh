// solve_f32.cuh -- the F32_REFINE Jacobi loop of CalcEpotential
// (CalcEpotential.f90:55-96) as a resumable state machine.
//
// A round runs m_eff sweeps from the current anchor a (w = 0, the increment
// restarts at every anchor), then one FP64 anchor pass folds the last
// increment into V and recomputes the exact residual; the sweeps' and the
// anchor's residual norms (per-tile partials reduced in a fixed order) come
// back to the host in one copy, and the first iterate d that meets the
// reference's stop test -- checked at the top of sweep d+1, so only while
// d+1 <= maxit -- ends the solve (rebuilt by replaying d - a sweeps from the
// anchor when it is not the anchor itself).
//
//   f32_begin       anchor 0 on the context stream
//   f32_plan        m_eff of the next round
//   (the caller runs sweeps a+1 .. a+m_eff, partials of sweep a+t at
//    ctx->partials + (t-1) * nblocks, S.wcur following the latest iterate:
//    run_sweeps_single, or the batched multi-run launch)
//   f32_issue_tail  anchor, reduction and the host copy, asynchronously
//   f32_finish      after the copy: stop test, replay, next batch length
#pragma once

#include "context.cuh"

namespace picard {

struct F32Solve {
  picard_ctx* c = nullptr;
  double tol = 0.0, tol2 = 0.0, sigma = 1.0;
  long long smax = 0;
  int maxit = 0;
  double* V[2] = {nullptr, nullptr};
  float* R[2] = {nullptr, nullptr};
  int vcur = 0, rcur = 0;
  int wcur = 0;  // buffer (ctx->w[wcur]) holding the latest increment
  long long a = 0;
  int m = 64, m_eff = 0;
  double r2_prev = 0.0, r2_last = 0.0;
  long long sweeps = 0;
  bool converged = true, done = false;
};

// CalcEpotential's set-up and wrap-up around the solve loop.
constexpr int kPinnedB2 = kMaxSweepsPerRound + 8;  // slot of ||b||^2 in ctx->h_pinned (past the r2 copies)
struct EpotSetup {
  double bnorm = 0.0, tol = 0.0, sigma = 1.0;
  long long smax = 0;
  int maxit = 0;
  bool trivial = false;  // ||b|| meets the test at the top of sweep 1: zero sweeps
};
// b and ||b||^2 (kernel + host copy, asynchronous)
int epot_rhs_issue(picard_ctx* c);
// after the copy has landed
EpotSetup epot_setup(picard_ctx* c, double maxerr, int32_t maxit);
// periodic ghost refresh, statistics, status
int epot_finish(picard_ctx* c, const EpotSetup& e, long long sweeps, bool converged, int32_t* sweeps_out);

int f32_begin(F32Solve& S, picard_ctx* c, double tol, long long smax, int maxit, double sigma);
int f32_plan(F32Solve& S);
int f32_issue_tail(F32Solve& S);
// timed_sweeps: the context's events ev[0] and ev[1] bracket the round's sweeps
int f32_finish(F32Solve& S, bool timed_sweeps);
// count sweeps of one run with its own launches, the first from w = 0; each
// launch reads ctx->w[*wcur] and writes the other buffer, *wcur following.
int run_sweeps_single(picard_ctx* c, int count, int rsel, double* partial_base, int* wcur);

}  // namespace picard
