// spectral.cu -- CalcEpotential's Jacobi iterate (CalcEpotential.f90:55-96)
// evaluated in closed form in the eigenbasis of the sweep.
//
// One reference sweep is U <- U - af * res with res = b - L U (L the 7-point
// Laplacian over the interior; ghosts held fixed on open faces, wrapped on
// periodic axes; CalcEpotential.f90:74-92, with af/d^2 = a_d).  A sweep
// changes only interior nodes, so the residual of iterate d is
//   r_d = G^d r_0,  G = ax S_x + ay S_y + az S_z,
// S_d the neighbour-sum operator of axis d with zero ghosts (open) or wrap
// (periodic), and
//   U_d = U_0 - af * sum_{j<d} G^j r_0.
// Each S_d is diagonalised by an orthonormal basis Q_d of its axis:
//   open:     Q[m][i] = sqrt(2/(n+1)) sin(pi (m+1)(i+1)/(n+1)), eigenvalue
//             2 cos(pi (m+1)/(n+1))  (the discrete sine transform, DST-I);
//   periodic: the real Fourier basis 1/sqrt(n), sqrt(2/n) cos / sin(2 pi f i/n)
//             and (-1)^i/sqrt(n), eigenvalue 2 cos(2 pi f/n).
// In the product basis Q = Qz Qy Qx the operator G is diagonal with
// g = 1 - omg, omg = sum_d a_d (2 - sigma_d) (2 (ax + ay + az) = 1), so with
// rh = Q r_0:
//   ||r_d||^2 = sum_m g_m^(2d) rh_m^2            (Parseval),
//   U_d = U_0 - af Q^T [ (1 - g^d)/(1 - g) rh ].
// ||r_d|| does not increase with d (|g| <= 1), and the stopping sweep of the
// reference -- the first iterate d >= 1 with d + 1 <= maxit and
// ||r_d|| <= maxerr ||b|| -- is found by a bracketing search: each launch
// evaluates the Parseval sum at up to kSpecPoints sweep counts.
//
// The transforms are dense per-axis products (FP64, 2n flops per node and
// axis): the z and y passes multiply Q_d from the left onto planes/rows of
// the compact interior array, the x pass multiplies rows by Q_x^T from the
// right.  Everything is FP64; the result equals the FP64 sweeps' iterate to
// rounding (the sweeps themselves round each of their d updates).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "context.cuh"
#include "picard_gpu.h"

namespace picard {

namespace {

constexpr int kSpecPoints = 32;     // sweep counts per evaluation launch
constexpr int kSpecThreads = 256;
constexpr int kGemmBM = 64, kGemmBN = 64, kGemmBK = 16;

// r_0 = b - L U over the interior, compact x-fastest (CalcEpotential.f90:83-92;
// periodic axes read the wrapped interior instead of the ghost).
__global__ void spec_r0_kernel(KParams P, double idx2, double idy2, double idz2, const double* __restrict__ U,
                               const double* __restrict__ b, double* __restrict__ R) {
  const long long n = (long long)P.nx * P.ny * P.nz;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int i = int(t % P.nx) + 1;
    const int j = int((t / P.nx) % P.ny) + 1;
    const int k = int(t / ((long long)P.nx * P.ny)) + 1;
    const int im = (i == 1 && !P.xflow) ? P.nx : i - 1, ip = (i == P.nx && !P.xflow) ? 1 : i + 1;
    const int jm = (j == 1 && !P.yflow) ? P.ny : j - 1, jp = (j == P.ny && !P.yflow) ? 1 : j + 1;
    const int km = (k == 1 && !P.zflow) ? P.nz : k - 1, kp = (k == P.nz && !P.zflow) ? 1 : k + 1;
    const double u = U[node_index(P, i, j, k)];
    const double lap = (U[node_index(P, ip, j, k)] + U[node_index(P, im, j, k)] - 2.0 * u) * idx2 +
                       (U[node_index(P, i, jp, k)] + U[node_index(P, i, jm, k)] - 2.0 * u) * idy2 +
                       (U[node_index(P, i, j, kp)] + U[node_index(P, i, j, km)] - 2.0 * u) * idz2;
    R[t] = b[node_index(P, i, j, k)] - lap;
  }
}

// C[o] (M x N) = A[o] (M x K, K contiguous: A[m*lda + k]) * B[o] (K x N),
// B[k*ldb + n] (N contiguous) or, with KB, B[n*ldb + k] (K contiguous).
// Tiles of 64 x 64, K chunks of 16, 256 threads with 4 x 4 outputs each (rows
// ty + 16a, columns tx + 16c).  Batch o = blockIdx.z with element strides
// sa, sb, sc.
template <bool KB>
__global__ void __launch_bounds__(256) spec_gemm_kernel(const double* __restrict__ A, int lda, long long sa,
                                                        const double* __restrict__ B, int ldb, long long sb,
                                                        double* __restrict__ C, int ldc, long long sc, int M, int N,
                                                        int K) {
  __shared__ double As[kGemmBK][kGemmBM + 2];
  __shared__ double Bs[kGemmBK][kGemmBN + 2];
  const int tid = threadIdx.x;
  const int tx = tid & 15, ty = tid >> 4;
  const int m0 = blockIdx.y * kGemmBM, n0 = blockIdx.x * kGemmBN;
  A += sa * blockIdx.z;
  B += sb * blockIdx.z;
  C += sc * blockIdx.z;
  double acc[4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int c = 0; c < 4; ++c) acc[a][c] = 0.0;
  for (int k0 = 0; k0 < K; k0 += kGemmBK) {
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int q = tid + 256 * e;
      const int m = q >> 4, k = q & 15;  // A: k fastest
      const int gm = m0 + m, gk = k0 + k;
      As[k][m] = (gm < M && gk < K) ? A[(long long)gm * lda + gk] : 0.0;
      if (KB) {
        const int n = q >> 4, kk = q & 15;
        const int gn = n0 + n, gkk = k0 + kk;
        Bs[kk][n] = (gn < N && gkk < K) ? B[(long long)gn * ldb + gkk] : 0.0;
      } else {
        const int kk = q >> 6, n = q & 63;
        const int gn = n0 + n, gkk = k0 + kk;
        Bs[kk][n] = (gn < N && gkk < K) ? B[(long long)gkk * ldb + gn] : 0.0;
      }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < kGemmBK; ++k) {
      double av[4], bv[4];
#pragma unroll
      for (int a = 0; a < 4; ++a) av[a] = As[k][ty + 16 * a];
#pragma unroll
      for (int c = 0; c < 4; ++c) bv[c] = Bs[k][tx + 16 * c];
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int c = 0; c < 4; ++c) acc[a][c] = fma(av[a], bv[c], acc[a][c]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    const int gm = m0 + ty + 16 * a;
    if (gm >= M) continue;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const int gn = n0 + tx + 16 * c;
      if (gn < N) C[(long long)gm * ldc + gn] = acc[a][c];
    }
  }
}

// x^e for e >= 0 by binary powering.
__device__ inline double ipow(double x, long long e) {
  double r = 1.0;
  while (e > 0) {
    if (e & 1) r *= x;
    x *= x;
    e >>= 1;
  }
  return r;
}

// Parseval sums f(d_t) = sum_m g_m^(2 d_t) rh_m^2 at the sweep counts
// d_t = d0 + t*step (doubling == 0) or d_t = d0 * 2^t (doubling == 1), for
// t < count.  Modes with g^2 <= g2_skip add nothing (the caller bounds what
// they could add far below the stop test's resolution).  Per-block partials
// in a fixed order; the last block to finish sums them (in block order) into
// out[t] and re-arms the counter.
__global__ void __launch_bounds__(kSpecThreads) spec_norms_kernel(const double* __restrict__ Rh, int nx, int ny,
                                                                  int nz, const double* __restrict__ omx,
                                                                  const double* __restrict__ omy,
                                                                  const double* __restrict__ omz, long long d0,
                                                                  long long step, int count, int doubling,
                                                                  double g2_skip, double* __restrict__ partial,
                                                                  unsigned int* counter, double* __restrict__ out) {
  double acc[kSpecPoints];
#pragma unroll
  for (int t = 0; t < kSpecPoints; ++t) acc[t] = 0.0;
  const long long n = (long long)nx * ny * nz;
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    const int mx = int(q % nx), my = int((q / nx) % ny), mz = int(q / ((long long)nx * ny));
    const double g = 1.0 - (omx[mx] + omy[my] + omz[mz]);
    const double g2 = g * g;
    if (g2 <= g2_skip) continue;
    const double r = Rh[q];
    const double w = r * r;
    const double x = ipow(g2, d0);
    if (doubling) {
      double y = x;  // d0 * 2^t: a chain of squarings
#pragma unroll
      for (int t = 0; t < kSpecPoints; ++t) {
        if (t < count) acc[t] = fma(w, y, acc[t]);
        y *= y;
      }
    } else {
      // x h^t with h^t from the binary digits of t: 32 short independent
      // chains instead of one chain of 32 dependent products
      double hp[5];
      hp[0] = ipow(g2, step);
#pragma unroll
      for (int b = 1; b < 5; ++b) hp[b] = hp[b - 1] * hp[b - 1];
#pragma unroll
      for (int t = 0; t < kSpecPoints; ++t) {
        double y = x;
#pragma unroll
        for (int b = 0; b < 5; ++b)
          if (t & (1 << b)) y *= hp[b];
        if (t < count) acc[t] = fma(w, y, acc[t]);
      }
    }
  }
  __shared__ double sh[kSpecThreads / 32][kSpecPoints];
  __shared__ bool last;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int t = 0; t < kSpecPoints; ++t) {
    double v = acc[t];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) sh[wid][t] = v;
  }
  __syncthreads();
  if (threadIdx.x < kSpecPoints) {
    double s = 0.0;
    for (int w2 = 0; w2 < kSpecThreads / 32; ++w2) s += sh[w2][threadIdx.x];
    partial[(long long)blockIdx.x * kSpecPoints + threadIdx.x] = s;
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(counter, 1u) == gridDim.x - 1;
  __syncthreads();
  if (!last) return;
  __threadfence();
  // the last block: out[t] = sum_b partial[b][t], warp w taking points w, w + 8, ...
  for (int t = wid; t < kSpecPoints; t += kSpecThreads / 32) {
    double s = 0.0;
    for (int b2 = lane; b2 < (int)gridDim.x; b2 += 32) s += __ldcg(partial + (long long)b2 * kSpecPoints + t);
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) out[t] = s;
  }
  if (threadIdx.x == 0) *counter = 0u;
}

// rh -> -af (1 - g^d)/(1 - g) rh in place.  For g > 0 the factor is
// -expm1(d log1p(-omg))/omg (no cancellation near g = 1); a mode with
// omg == 0 (every axis periodic, the constant mode) takes d.
__global__ void spec_scale_kernel(double* __restrict__ Rh, int nx, int ny, int nz, const double* __restrict__ omx,
                                  const double* __restrict__ omy, const double* __restrict__ omz, long long d,
                                  double af) {
  const long long n = (long long)nx * ny * nz;
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    const int mx = int(q % nx), my = int((q / nx) % ny), mz = int(q / ((long long)nx * ny));
    const double omg = omx[mx] + omy[my] + omz[mz];
    double f;
    if (omg == 0.0) {
      f = (double)d;
    } else if (omg < 1.0) {
      f = -expm1((double)d * log1p(-omg)) / omg;
    } else {
      const double g = 1.0 - omg;  // in [-1, 0]
      f = (1.0 - ipow(g, d)) / omg;
    }
    Rh[q] = -af * f * Rh[q];
  }
}

// U(interior) += D (compact).
__global__ void spec_apply_kernel(KParams P, const double* __restrict__ D, double* __restrict__ U) {
  const long long n = (long long)P.nx * P.ny * P.nz;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int i = int(t % P.nx) + 1;
    const int j = int((t / P.nx) % P.ny) + 1;
    const int k = int(t / ((long long)P.nx * P.ny)) + 1;
    U[node_index(P, i, j, k)] += D[t];
  }
}

// In-place fold along one axis of an (O, n, I) array (element (o, i, t) at
// (o n + i) I + t): for i < n/2, x[i] <- x[i] + x[n-1-i] and x[n-1-i] <-
// x[i] - x[n-1-i] (the middle of an odd n unchanged); unfold is the same
// butterfly after the inverse products (E + O, E - O).
__global__ void spec_fold_kernel(double* __restrict__ x, long long O, int n, long long I) {
  const int h = n / 2;
  const long long pairs = O * h * I;
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < pairs;
       q += (long long)gridDim.x * blockDim.x) {
    const long long t = q % I;
    const long long r = q / I;
    const int i = int(r % h);
    const long long o = r / h;
    double* row = x + o * n * I + t;
    const double a = row[(long long)i * I], b = row[(long long)(n - 1 - i) * I];
    row[(long long)i * I] = a + b;
    row[(long long)(n - 1 - i) * I] = a - b;
  }
}

int stream_blocks(long long n) {
  long long b = (n + kSpecThreads - 1) / kSpecThreads;
  return int(std::max<long long>(1, std::min<long long>(b, 148LL * 8)));
}

// One axis basis: Q (n x n, row = mode), its transpose, and a_d (2 - sigma)
// per mode.
void axis_basis(int n, bool periodic, double a, std::vector<double>& Q, std::vector<double>& QT,
                std::vector<double>& om);

// The sine basis folded by its symmetry Q[m][n-1-i] = (-1)^m Q[m][i]: with
// hs = ceil(n/2), h = floor(n/2), the even modes 2k come from the folded sums
// x[i] + x[n-1-i] (i < h) and the middle x[h] through Qe (hs x hs), the odd
// modes 2k+1 from the differences x[i] - x[n-1-i], held at position n-1-i,
// through QoR[k][j] = Q[2k+1][h-1-j] (h x h).  Modes are kept in the order
// [even | odd]; om follows that order.
void folded_basis(int n, double a, std::vector<double>& Qe, std::vector<double>& QeT, std::vector<double>& QoR,
                  std::vector<double>& QoRT, std::vector<double>& om) {
  std::vector<double> Q, QT, om0;
  axis_basis(n, false, a, Q, QT, om0);
  const int h = n / 2, hs = n - h;
  Qe.assign((size_t)hs * hs, 0.0);
  QeT.assign((size_t)hs * hs, 0.0);
  QoR.assign((size_t)std::max(h, 1) * std::max(h, 1), 0.0);
  QoRT.assign(QoR.size(), 0.0);
  om.assign(n, 0.0);
  for (int k = 0; k < hs; ++k) {
    for (int i = 0; i < hs; ++i) {
      Qe[(size_t)k * hs + i] = Q[(size_t)(2 * k) * n + i];
      QeT[(size_t)i * hs + k] = Q[(size_t)(2 * k) * n + i];
    }
    om[k] = om0[2 * k];
  }
  for (int k = 0; k < h; ++k) {
    for (int j = 0; j < h; ++j) {
      QoR[(size_t)k * h + j] = Q[(size_t)(2 * k + 1) * n + (h - 1 - j)];
      QoRT[(size_t)j * h + k] = QoR[(size_t)k * h + j];
    }
    om[hs + k] = om0[2 * k + 1];
  }
}

void axis_basis(int n, bool periodic, double a, std::vector<double>& Q, std::vector<double>& QT,
                std::vector<double>& om) {
  const double pi = 3.14159265358979323846264338327950288;
  Q.assign((size_t)n * n, 0.0);
  QT.assign((size_t)n * n, 0.0);
  om.assign(n, 0.0);
  if (!periodic) {
    const double s = std::sqrt(2.0 / (n + 1));
    const long long per = 2LL * (n + 1);
    for (int m = 0; m < n; ++m) {
      for (int i = 0; i < n; ++i) {
        const long long p = ((long long)(m + 1) * (i + 1)) % per;  // sin(pi p/(n+1)) has period 2(n+1)
        Q[(size_t)m * n + i] = s * std::sin(pi * (double)p / (double)(n + 1));
      }
      const double h = std::sin(pi * (m + 1) / (2.0 * (n + 1)));
      om[m] = a * 4.0 * h * h;  // a (2 - 2 cos(theta)) = 4 a sin^2(theta/2)
    }
  } else {
    int row = 0;
    auto put = [&](int f, int kind) {  // kind 0: constant, 1: cos, 2: sin, 3: alternating
      for (int i = 0; i < n; ++i) {
        double v;
        const long long p = ((long long)f * i) % n;
        if (kind == 0) v = 1.0 / std::sqrt((double)n);
        else if (kind == 3) v = (i % 2 ? -1.0 : 1.0) / std::sqrt((double)n);
        else if (kind == 1) v = std::sqrt(2.0 / n) * std::cos(2.0 * pi * (double)p / n);
        else v = std::sqrt(2.0 / n) * std::sin(2.0 * pi * (double)p / n);
        Q[(size_t)row * n + i] = v;
      }
      const double h = std::sin(pi * f / (double)n);
      om[row] = a * 4.0 * h * h;
      ++row;
    };
    put(0, 0);
    for (int f = 1; 2 * f < n; ++f) {
      put(f, 1);
      put(f, 2);
    }
    if (n % 2 == 0 && n >= 2) put(n / 2, 3);
  }
  for (int m = 0; m < n; ++m)
    for (int i = 0; i < n; ++i) QT[(size_t)i * n + m] = Q[(size_t)m * n + i];
}

template <bool KB>
cudaError_t gemm(const double* A, int lda, long long sa, const double* B, int ldb, long long sb, double* C, int ldc,
                 long long sc, int M, int N, int K, int batch, cudaStream_t st) {
  dim3 grid((N + kGemmBN - 1) / kGemmBN, (M + kGemmBM - 1) / kGemmBM, batch);
  note_launch();
  spec_gemm_kernel<KB><<<grid, 256, 0, st>>>(A, lda, sa, B, ldb, sb, C, ldc, sc, M, N, K);
  return cudaGetLastError();
}

cudaError_t fold(picard_ctx* c, double* x, long long O, int n, long long I) {
  if (n < 2) return cudaSuccess;
  note_launch();
  spec_fold_kernel<<<stream_blocks(O * (n / 2) * I), kSpecThreads, 0, c->st>>>(x, O, n, I);
  return cudaGetLastError();
}

// One axis pass from `in` to `out`.  Axis d of length n has outer extent O
// and inner extent I (x: O = ny nz, I = 1; y: O = nz, I = nx; z: O = 1, I =
// nx ny).  Dense axes (periodic): out = Q in (forward) or Q^T in (inverse)
// along the axis.  Folded axes (open): forward folds `in` in place and applies
// Qe and QoR to its two halves; inverse applies Qe^T and QoR^T to the two
// halves of `in` and unfolds `out` in place.
cudaError_t axis_pass(picard_ctx* c, int d, bool forward, double* in, double* out) {
  SpectralPlan& S = c->spec;
  const int nx = c->K.nx, ny = c->K.ny, nz = c->K.nz;
  const int n = d == 0 ? nx : d == 1 ? ny : nz;
  const long long O = d == 0 ? (long long)ny * nz : d == 1 ? nz : 1;
  const long long I = d == 0 ? 1 : d == 1 ? nx : (long long)nx * ny;
  const long long plane = (long long)nx * ny;
  cudaError_t e;
  if (!S.folded[d]) {
    if (d == 0) {
      // x: out[r][m] = sum_i in[r][i] Q[m][i] (B K-contiguous), or sum_m in[r][m] Q[m][i]
      return forward ? gemm<true>(in, nx, 0, S.Q[0], nx, 0, out, nx, 0, ny * nz, nx, nx, 1, c->st)
                     : gemm<false>(in, nx, 0, S.Q[0], nx, 0, out, nx, 0, ny * nz, nx, nx, 1, c->st);
    }
    const double* M = forward ? S.Q[d] : S.QT[d];
    if (d == 1) return gemm<false>(M, ny, 0, in, nx, plane, out, nx, plane, ny, nx, ny, nz, c->st);
    return gemm<false>(M, nz, 0, in, (int)plane, 0, out, (int)plane, 0, nz, (int)plane, nz, 1, c->st);
  }
  const int h = n / 2, hs = n - h;
  if (forward && (e = fold(c, in, O, n, I))) return e;
  const double* Me = forward ? S.Qe[d] : S.QeT[d];
  const double* Mo = forward ? S.QoR[d] : S.QoRT[d];
  if (d == 0) {
    if (forward) {
      if ((e = gemm<true>(in, nx, 0, Me, hs, 0, out, nx, 0, ny * nz, hs, hs, 1, c->st))) return e;
      if (h > 0 && (e = gemm<true>(in + hs, nx, 0, Mo, h, 0, out + hs, nx, 0, ny * nz, h, h, 1, c->st))) return e;
    } else {
      if ((e = gemm<false>(in, nx, 0, S.Qe[0], hs, 0, out, nx, 0, ny * nz, hs, hs, 1, c->st))) return e;
      if (h > 0 && (e = gemm<false>(in + hs, nx, 0, S.QoR[0], h, 0, out + hs, nx, 0, ny * nz, h, h, 1, c->st)))
        return e;
    }
  } else if (d == 1) {
    if ((e = gemm<false>(Me, hs, 0, in, nx, plane, out, nx, plane, hs, nx, hs, nz, c->st))) return e;
    if (h > 0 && (e = gemm<false>(Mo, h, 0, in + (long long)hs * nx, nx, plane, out + (long long)hs * nx, nx, plane, h,
                                  nx, h, nz, c->st)))
      return e;
  } else {
    if ((e = gemm<false>(Me, hs, 0, in, (int)plane, 0, out, (int)plane, 0, hs, (int)plane, hs, 1, c->st))) return e;
    if (h > 0 && (e = gemm<false>(Mo, h, 0, in + (long long)hs * plane, (int)plane, 0, out + (long long)hs * plane,
                                  (int)plane, 0, h, (int)plane, h, 1, c->st)))
      return e;
  }
  if (!forward) return fold(c, out, O, n, I);
  return cudaSuccess;
}

// Forward: Qz Qy Qx of T[0] into T[1] (x, y, z passes ping-ponging T[0] and
// T[1]); inverse: Qx^T Qy^T Qz^T of T[1] into T[0].
cudaError_t transform(picard_ctx* c, bool forward) {
  SpectralPlan& S = c->spec;
  cudaError_t e;
  if (forward) {
    if ((e = axis_pass(c, 0, true, S.T[0], S.T[1]))) return e;
    if ((e = axis_pass(c, 1, true, S.T[1], S.T[0]))) return e;
    return axis_pass(c, 2, true, S.T[0], S.T[1]);
  }
  if ((e = axis_pass(c, 2, false, S.T[1], S.T[0]))) return e;
  if ((e = axis_pass(c, 1, false, S.T[0], S.T[1]))) return e;
  return axis_pass(c, 0, false, S.T[1], S.T[0]);
}

// Queues the evaluation of f at count (<= kSpecPoints) sweep counts and the
// copy of the sums to c->h_pinned[0..count); the caller waits on the stream.
int issue_norms(picard_ctx* c, long long d0, long long step, int count, bool doubling, double g2_skip) {
  SpectralPlan& S = c->spec;
  note_launch();
  spec_norms_kernel<<<S.norm_blocks, kSpecThreads, 0, c->st>>>(S.T[1], c->K.nx, c->K.ny, c->K.nz, S.om[0], S.om[1],
                                                                S.om[2], d0, step, count, doubling ? 1 : 0, g2_skip,
                                                                S.partial, S.counter, S.sums);
  PICARD_CUDA(cudaGetLastError());
  PICARD_CUDA(cudaMemcpyAsync(c->h_pinned, S.sums, sizeof(double) * count, cudaMemcpyDeviceToHost, c->st));
  c->stats.d2h_bytes += (int64_t)sizeof(double) * count;
  S.evals += 1;
  return PICARD_OK;
}

}  // namespace

int spectral_alloc(picard_ctx* c) {
  SpectralPlan& S = c->spec;
  const KParams& K = c->K;
  const long long n = (long long)K.nx * K.ny * K.nz;
  const JacobiCoef J = jacobi_coef(K);
  const double a[3] = {J.ax, J.ay, J.az};
  const int len[3] = {K.nx, K.ny, K.nz};
  const bool per[3] = {!K.xflow, !K.yflow, !K.zflow};
  for (int d = 0; d < 3; ++d) {
    void* p = nullptr;
    if (!per[d]) {
      std::vector<double> Qe, QeT, QoR, QoRT, om;
      folded_basis(len[d], a[d], Qe, QeT, QoR, QoRT, om);
      double** dst[5] = {&S.Qe[d], &S.QeT[d], &S.QoR[d], &S.QoRT[d], &S.om[d]};
      const std::vector<double>* srcv[5] = {&Qe, &QeT, &QoR, &QoRT, &om};
      for (int t = 0; t < 5; ++t) {
        PICARD_TRY(dev_alloc(c, &p, sizeof(double) * srcv[t]->size()));
        *dst[t] = static_cast<double*>(p);
        // no wait: an asynchronous copy from pageable memory returns once the
        // host data is staged, so the vectors may go out of scope
        PICARD_CUDA(cudaMemcpyAsync(*dst[t], srcv[t]->data(), sizeof(double) * srcv[t]->size(),
                                    cudaMemcpyHostToDevice, c->st));
        c->stats.h2d_bytes += (int64_t)(sizeof(double) * srcv[t]->size());
      }
      S.folded[d] = 1;
      continue;
    }
    std::vector<double> Q, QT, om;
    axis_basis(len[d], per[d], a[d], Q, QT, om);
    PICARD_TRY(dev_alloc(c, &p, sizeof(double) * Q.size()));
    S.Q[d] = static_cast<double*>(p);
    PICARD_TRY(dev_alloc(c, &p, sizeof(double) * QT.size()));
    S.QT[d] = static_cast<double*>(p);
    PICARD_TRY(dev_alloc(c, &p, sizeof(double) * om.size()));
    S.om[d] = static_cast<double*>(p);
    PICARD_CUDA(cudaMemcpyAsync(S.Q[d], Q.data(), sizeof(double) * Q.size(), cudaMemcpyHostToDevice, c->st));
    PICARD_CUDA(cudaMemcpyAsync(S.QT[d], QT.data(), sizeof(double) * QT.size(), cudaMemcpyHostToDevice, c->st));
    PICARD_CUDA(cudaMemcpyAsync(S.om[d], om.data(), sizeof(double) * om.size(), cudaMemcpyHostToDevice, c->st));
    // no wait: an asynchronous copy from pageable memory returns once the host
    // data is staged, so the vectors may go out of scope
    c->stats.h2d_bytes += (int64_t)sizeof(double) * (Q.size() + QT.size() + om.size());
  }
  void* p = nullptr;
  PICARD_TRY(dev_alloc(c, &p, sizeof(double) * n));
  S.T[0] = static_cast<double*>(p);
  PICARD_TRY(dev_alloc(c, &p, sizeof(double) * n));
  S.T[1] = static_cast<double*>(p);
  S.norm_blocks = stream_blocks(n);
  PICARD_TRY(dev_alloc(c, &p, sizeof(double) * (size_t)S.norm_blocks * kSpecPoints));
  S.partial = static_cast<double*>(p);
  PICARD_TRY(dev_alloc(c, &p, sizeof(double) * kSpecPoints));
  S.sums = static_cast<double*>(p);
  PICARD_TRY(dev_alloc(c, &p, sizeof(unsigned int)));  // zeroed
  S.counter = static_cast<unsigned int*>(p);
  return PICARD_OK;
}

long long spectral_bytes(const KParams& K) {
  const long long n = (long long)K.nx * K.ny * K.nz;
  return 8LL * (2 * n + 2LL * ((long long)K.nx * K.nx + (long long)K.ny * K.ny + (long long)K.nz * K.nz) + K.nx +
                K.ny + K.nz + (long long)stream_blocks(n) * kSpecPoints + kSpecPoints);
}

// The stopping-sweep search: the first d in [1, dmax] with f(d) <= tol^2
// (checked at the top of sweep d + 1 <= maxit).  Invariant: f(lo) > tol^2
// (lo = 0: no sweep yet), and f(hi) <= tol^2 when hi <= dmax (hi = dmax + 1:
// no passing d known).  The first evaluation doubles d from 1 up to the
// first power of two >= dmax; later ones take evenly spaced candidates of
// (lo, hi).

// Modes whose g^2 is at most the returned value add at most 2^-60 tol^2 to
// any f(d) the uniform passes evaluate (d > lo): sum over those modes of
// w g^(2d) <= g2_max^(d-1) f(1).  None is skipped while lo < 2 or f(1) is
// unknown.
static double skip_threshold(const SpecSolve& Q) {
  if (Q.lo < 2 || !(Q.f1 > 0.0) || !(Q.tol2 > 0.0)) return -1.0;
  const double ratio = Q.tol2 * 0x1p-60 / Q.f1;
  if (!(ratio < 1.0)) return -1.0;
  return std::exp(std::log(ratio) / double(Q.lo - 1));
}

int spec_begin(SpecSolve& Q, picard_ctx* c, double tol, long long smax, int maxit) {
  SpectralPlan& S = c->spec;
  const KParams& K = c->K;
  const long long n = (long long)K.nx * K.ny * K.nz;
  const JacobiCoef J = jacobi_coef(K);
  Q = SpecSolve();
  Q.c = c;
  Q.tol2 = tol * tol;
  Q.smax = smax;
  Q.dmax = (long long)maxit - 1;
  Q.lo = 0;
  Q.hi = Q.dmax + 1;
  PICARD_CUDA(cudaEventRecord(c->ev[0], c->st));
  note_launch();
  spec_r0_kernel<<<stream_blocks(n), kSpecThreads, 0, c->st>>>(K, 1.0 / J.dx2, 1.0 / J.dy2, 1.0 / J.dz2, c->U, c->b,
                                                                S.T[0]);
  PICARD_CUDA(cudaGetLastError());
  PICARD_CUDA(transform(c, true));
  PICARD_CUDA(cudaEventRecord(c->ev[1], c->st));
  if (Q.dmax >= 1) {
    int cnt = 1;
    while (cnt < kSpecPoints && (1LL << (cnt - 1)) < Q.dmax) ++cnt;
    Q.d0 = 1;
    Q.step = 0;
    Q.count = cnt;
    Q.doubling = true;
    return issue_norms(c, 1, 0, cnt, true, -1.0);
  }
  return spec_finish_issue(Q);
}

int spec_collect(SpecSolve& Q) {
  picard_ctx* c = Q.c;
  if (Q.final_eval) {  // f(smax) of a solve without a hit
    c->last_residual = std::sqrt(c->h_pinned[0]);
    Q.final_eval = false;
    return spec_apply_issue(Q);
  }
  if (Q.doubling) {
    Q.f1 = c->h_pinned[0];  // f(1)
    for (int t = 0; t < Q.count; ++t) {
      const long long d = 1LL << t;
      if (d > Q.dmax) break;
      if (c->h_pinned[t] <= Q.tol2) {
        Q.hi = d;
        Q.r2_hit = c->h_pinned[t];
        break;
      }
      Q.lo = d;
    }
    Q.doubling = false;
  } else {
    long long nlo = Q.d0 + Q.step * (Q.count - 1);
    for (int t = 0; t < Q.count; ++t) {
      if (c->h_pinned[t] <= Q.tol2) {
        Q.hi = Q.d0 + Q.step * t;
        Q.r2_hit = c->h_pinned[t];
        nlo = Q.hi - Q.step;
        break;
      }
    }
    Q.lo = nlo;
  }
  if (Q.hi - Q.lo > 1) {
    const long long span = Q.hi - 1 - Q.lo;  // candidates lo + 1 .. hi - 1
    Q.step = (span + kSpecPoints - 1) / kSpecPoints;
    Q.count = int(span / Q.step);
    Q.d0 = Q.lo + Q.step;
    return issue_norms(c, Q.d0, Q.step, Q.count, false, skip_threshold(Q));
  }
  return spec_finish_issue(Q);
}

int spec_finish_issue(SpecSolve& Q) {
  picard_ctx* c = Q.c;
  if (Q.hi <= Q.dmax) {
    Q.d = Q.hi;
    Q.converged = true;
    c->last_residual = std::sqrt(Q.r2_hit);
    return spec_apply_issue(Q);
  }
  Q.d = Q.smax;
  Q.converged = false;
  Q.final_eval = true;
  return issue_norms(c, Q.smax, 1, 1, false, -1.0);
}

int spec_apply_issue(SpecSolve& Q) {
  picard_ctx* c = Q.c;
  SpectralPlan& S = c->spec;
  const KParams& K = c->K;
  const long long n = (long long)K.nx * K.ny * K.nz;
  const JacobiCoef J = jacobi_coef(K);
  PICARD_CUDA(cudaEventRecord(c->ev[2], c->st));
  note_launch();
  spec_scale_kernel<<<stream_blocks(n), kSpecThreads, 0, c->st>>>(S.T[1], K.nx, K.ny, K.nz, S.om[0], S.om[1],
                                                                   S.om[2], Q.d, J.af);
  PICARD_CUDA(cudaGetLastError());
  PICARD_CUDA(transform(c, false));
  note_launch();
  spec_apply_kernel<<<stream_blocks(n), kSpecThreads, 0, c->st>>>(K, S.T[0], c->U);
  PICARD_CUDA(cudaGetLastError());
  PICARD_CUDA(cudaEventRecord(c->ev[3], c->st));
  Q.done = true;
  return PICARD_OK;
}

// Device time of a finished solve (after its stream has passed ev[3]).
void spec_account(SpecSolve& Q) {
  picard_ctx* c = Q.c;
  float f0 = 0.f, f1 = 0.f;
  cudaEventElapsedTime(&f0, c->ev[0], c->ev[1]);
  cudaEventElapsedTime(&f1, c->ev[2], c->ev[3]);
  c->stats.spectral_transforms += 2;
  c->stats.spectral_transform_ms += f0 + f1;
}

int solve_spectral(picard_ctx* c, double tol, long long smax, int maxit, long long* sweeps, bool* converged) {
  SpecSolve Q;
  PICARD_TRY(spec_begin(Q, c, tol, smax, maxit));
  for (;;) {
    PICARD_CUDA(cudaStreamSynchronize(c->st));
    if (Q.done) break;
    PICARD_TRY(spec_collect(Q));
  }
  spec_account(Q);
  *sweeps = Q.d;
  *converged = Q.converged;
  return PICARD_OK;
}

}  // namespace picard
