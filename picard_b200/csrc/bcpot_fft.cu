// bcpot_fft.cu -- BCpotentials (BCpotentials.f90:36-139) as FP64 FFT
// convolutions over the faces.
//
// The face potential of the reference is a direct sum over every interior
// cell; for the x0 face, node (0, j, k), with 0-based interior cells (a,b,c):
//   U = (2 tau eps0)^-1 sum_{a,b,c} C(a,b,c) D(a+1, b-j, c-k)
// and the x1 face takes D(a-Nx, ...) (BCpotentials.f90:53-63 with one rank;
// D(ox,oy,oz) the CalcDistance table, even in every offset).  For each plane
// a of cells along the face normal this is a 2-D correlation over the two
// tangential axes with the kernel slice D(s, ., .), s = a+1 (x0) or Nx-a (x1),
// so in the 2-D Fourier domain of the tangential axes (lengths LP, LQ: powers
// of two >= 2n-1, so the circular convolution reproduces every needed
// offset without wrap-around):
//   U^(kP,kQ) = sum_a C^_a(kP,kQ) E^_s(a)(kP,kQ)
// with E_s the slice laid out circularly; E_s is real and even, so its
// transform is real.  Per face pair: a real-to-complex FFT of every cell
// plane (rows along P keep LP/2+1 outputs, then columns along Q), the
// contraction over planes against the precomputed slice transforms (the
// constant (2 tau eps0)^-1 / (LP LQ) folded in), and one inverse FFT per face.
// FP64 throughout: radix-4 Stockham FFTs (one radix-2 stage for odd powers
// of two) in shared memory with twiddles computed on the host.  The slice transforms depend only on D and are
// computed on the first call after D changes.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "context.cuh"

namespace picard {

namespace {

constexpr int kFftThreads = 256;
constexpr int kColElems = 1024;   // B2 * LQ per column CTA (4 elements per thread)
constexpr int kRowElems = 2048;   // B1 * LP per row CTA

__device__ inline double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// B sequences of length L (a power of two) in x (x[b*L + i]); Stockham
// stages ping-pong between x and y: one radix-2 stage when log2 L is odd, then
// radix-4 stages.  Returns the buffer holding the transform (natural order).
// tw[t] = exp(-2 pi i t / L), t < L; inv uses the conjugates (no scaling).
__device__ double2* fft_batch(double2* x, double2* y, int L, int logL, int B, const double2* __restrict__ tw,
                              bool inv) {
  int s = 0;  // log2 of the sub-transform length Ns done so far
  if (logL & 1) {
    const int half = L >> 1;
    for (int e = threadIdx.x; e < B * half; e += blockDim.x) {
      const int b = e >> (logL - 1), j = e & (half - 1);
      const double2* xb = x + (b << logL);
      double2* yb = y + (b << logL);
      const double2 v0 = xb[j], v1 = xb[j + half];
      yb[2 * j] = make_double2(v0.x + v1.x, v0.y + v1.y);
      yb[2 * j + 1] = make_double2(v0.x - v1.x, v0.y - v1.y);
    }
    __syncthreads();
    double2* t = x;
    x = y;
    y = t;
    s = 1;
  }
  const int quarter = L >> 2;
  for (; s < logL; s += 2) {
    const int Ns = 1 << s;
    const int tws = logL - 2 - s;  // twiddle index of factor r = r (j mod Ns) L / (4 Ns)
    for (int e = threadIdx.x; e < B * quarter; e += blockDim.x) {
      const int b = e >> (logL - 2), j = e & (quarter - 1);
      const double2* xb = x + (b << logL);
      double2* yb = y + (b << logL);
      const int k = j & (Ns - 1);
      double2 w1 = tw[k << tws], w2 = tw[(2 * k) << tws], w3 = tw[(3 * k) << tws];
      if (inv) {
        w1.y = -w1.y;
        w2.y = -w2.y;
        w3.y = -w3.y;
      }
      const double2 v0 = xb[j];
      const double2 v1 = cmul(xb[j + quarter], w1);
      const double2 v2 = cmul(xb[j + 2 * quarter], w2);
      const double2 v3 = cmul(xb[j + 3 * quarter], w3);
      const double2 a0 = make_double2(v0.x + v2.x, v0.y + v2.y), a1 = make_double2(v0.x - v2.x, v0.y - v2.y);
      const double2 a2 = make_double2(v1.x + v3.x, v1.y + v3.y);
      const double2 d = make_double2(v1.x - v3.x, v1.y - v3.y);
      const double2 a3 = inv ? make_double2(-d.y, d.x) : make_double2(d.y, -d.x);  // (v1 - v3) * (+-i)
      const int idx = ((j & ~(Ns - 1)) << 2) + k;
      yb[idx] = make_double2(a0.x + a2.x, a0.y + a2.y);
      yb[idx + Ns] = make_double2(a1.x + a3.x, a1.y + a3.y);
      yb[idx + 2 * Ns] = make_double2(a0.x - a2.x, a0.y - a2.y);
      yb[idx + 3 * Ns] = make_double2(a1.x - a3.x, a1.y - a3.y);
    }
    __syncthreads();
    double2* t = x;
    x = y;
    y = t;
  }
  return x;
}

// Geometry of one face pair: A the normal axis, P and Q the tangential axes.
struct FaceGeom {
  int nA, nP, nQ;
  int LP, LQ, logP, logQ, HP;
  long long sA, sP, sQ;      // node-array strides (elements)
  long long dA, dP, dQ;      // D-table strides
  long long d0;              // D-table index of offset (0, 0, 0)
  long long base;            // node index of interior cell (0, 0, 0)
  long long face0, face1;    // node index of face node (p, q) = (0, 0) on the two faces
  int G;                     // plane groups of the contraction
  int B1, B2;                // rows per row CTA, columns per column CTA
};

// Distance along a circular axis of length L to offset index t (the kernel
// slice is nonzero for |offset| < n).
__device__ inline int circ_off(int t, int L, int n, bool& ok) {
  const int d = t <= L - t ? t : L - t;
  ok = d < n;
  return d;
}

// Stage 1: FFT along P of rows.  mode 0: the charge rows (a, q), a in
// [a0, a0+B1), q = blockIdx.y < nQ, from C; mode 1: the kernel rows (s, tQ)
// of slices s0 + a (a < count), tQ = blockIdx.y < LQ, from D.  Output
// W[(a * rowsQ + q) * HP + kP], kP < HP.
__device__ __forceinline__ void bcfft_rows_body(const FaceGeom& F, int mode, const double* __restrict__ src, int s0,
                                                int count, const double2* __restrict__ tw, double2* __restrict__ W,
                                                int bx, int by) {
  extern __shared__ double2 smem[];
  const int B = F.B1;
  double2* x = smem;
  double2* y = smem + B * F.LP;
  const int a0 = bx * B;
  const int q = by;
  const int rowsQ = mode == 0 ? F.nQ : F.LQ;
  const int na = mode == 0 ? F.nA : count;
  const bool afast = F.sA == 1 && mode == 0;
  bool okq = true;
  int dq = 0;
  if (mode == 1) dq = circ_off(q, F.LQ, F.nQ, okq);
  for (int e = threadIdx.x; e < B * F.LP; e += blockDim.x) {
    int b, p;
    if (afast) {
      b = e % B;
      p = e / B;
    } else {
      b = e >> F.logP;
      p = e & (F.LP - 1);
    }
    const int a = a0 + b;
    double v = 0.0;
    if (a < na) {
      if (mode == 0) {
        if (p < F.nP) v = src[F.base + (long long)a * F.sA + (long long)p * F.sP + (long long)q * F.sQ];
      } else {
        bool okp;
        const int dp = circ_off(p, F.LP, F.nP, okp);
        if (okp && okq) v = src[F.d0 + (long long)(s0 + a) * F.dA + (long long)dp * F.dP + (long long)dq * F.dQ];
      }
    }
    x[(b << F.logP) + p] = make_double2(v, 0.0);
  }
  __syncthreads();
  const double2* X = fft_batch(x, y, F.LP, F.logP, B, tw, false);
  for (int e = threadIdx.x; e < B * F.HP; e += blockDim.x) {
    const int b = e / F.HP, k = e - b * F.HP;
    const int a = a0 + b;
    if (a < na) W[((long long)a * rowsQ + q) * F.HP + k] = X[(b << F.logP) + k];
  }
}

// Stage 2: FFT along Q of the columns kP in [k0, k0+B2).
// mode 0 (contraction): planes a of group blockIdx.y; each thread keeps the
// sums of its (kP, kQ) elements against Dh[s0(a)] and Dh[s1(a)] and writes the
// group's partial to S[(g * 2 + f) * HP * LQ + kP * LQ + kQ].
// mode 1 (kernel transforms): slices a < count of W, real part times scale
// to Dh[(s0 + a) * HP * LQ + kP * LQ + kQ].
__device__ __forceinline__ void bcfft_cols_body(const FaceGeom& F, int mode, const double2* __restrict__ W, int s0,
                                                int count, double scale, const double2* __restrict__ tw,
                                                double* __restrict__ Dh, double2* __restrict__ S, int bx, int by) {
  extern __shared__ double2 smem[];
  const int B = F.B2;
  double2* x = smem;
  double2* y = smem + B * F.LQ;
  const int k0 = bx * B;
  const int rowsQ = mode == 0 ? F.nQ : F.LQ;
  const long long plane = (long long)F.HP * F.LQ;
  int a_lo, a_hi;
  if (mode == 0) {
    const int per = (F.nA + F.G - 1) / F.G;
    a_lo = by * per;
    a_hi = min(F.nA, a_lo + per);
  } else {
    a_lo = by;
    a_hi = min(count, a_lo + 1);
  }
  double2 acc0[kColElems / kFftThreads], acc1[kColElems / kFftThreads];
#pragma unroll
  for (int u = 0; u < kColElems / kFftThreads; ++u) acc0[u] = acc1[u] = make_double2(0.0, 0.0);
  for (int a = a_lo; a < a_hi; ++a) {
    for (int e = threadIdx.x; e < B * F.LQ; e += blockDim.x) {
      const int q = e / B, b = e - q * B;  // kP fastest: contiguous in W
      const int k = k0 + b;
      double2 v = make_double2(0.0, 0.0);
      if (k < F.HP && q < rowsQ) v = W[((long long)a * rowsQ + q) * F.HP + k];
      x[(b << F.logQ) + q] = v;
    }
    __syncthreads();
    const double2* X = fft_batch(x, y, F.LQ, F.logQ, B, tw, false);
#pragma unroll
    for (int u = 0; u < kColElems / kFftThreads; ++u) {
      const int e = threadIdx.x + u * kFftThreads;  // B * LQ == kColElems
      const int b = e >> F.logQ, kq = e & (F.LQ - 1);
      const int k = k0 + b;
      if (k >= F.HP) continue;
      const double2 v = X[e];
      if (mode == 0) {
        const double d0 = Dh[(long long)a * plane + (long long)k * F.LQ + kq];                   // s = a + 1
        const double d1 = Dh[(long long)(F.nA - 1 - a) * plane + (long long)k * F.LQ + kq];      // s = nA - a
        acc0[u].x = fma(v.x, d0, acc0[u].x);
        acc0[u].y = fma(v.y, d0, acc0[u].y);
        acc1[u].x = fma(v.x, d1, acc1[u].x);
        acc1[u].y = fma(v.y, d1, acc1[u].y);
      } else {
        Dh[(long long)(s0 + a) * plane + (long long)k * F.LQ + kq] = v.x * scale;
      }
    }
    __syncthreads();
  }
  if (mode != 0) return;
#pragma unroll
  for (int u = 0; u < kColElems / kFftThreads; ++u) {
    const int e = threadIdx.x + u * kFftThreads;
    const int b = e >> F.logQ, kq = e & (F.LQ - 1);
    const int k = k0 + b;
    if (k >= F.HP) continue;
    S[((long long)by * 2 + 0) * plane + (long long)k * F.LQ + kq] = acc0[u];
    S[((long long)by * 2 + 1) * plane + (long long)k * F.LQ + kq] = acc1[u];
  }
}

// Stage 3a: sum of the group partials (fixed order) and the inverse FFT along
// Q of columns kP in [k0, k0+B2) of face f = blockIdx.y; V[(f*nQ + q)*HP + kP]
// for q < nQ.
__device__ __forceinline__ void bcfft_invq_body(const FaceGeom& F, const double2* __restrict__ S,
                                                const double2* __restrict__ tw, double2* __restrict__ V, int bx,
                                                int by) {
  extern __shared__ double2 smem[];
  const int B = F.B2;
  double2* x = smem;
  double2* y = smem + B * F.LQ;
  const int k0 = bx * B, f = by;
  const long long plane = (long long)F.HP * F.LQ;
  for (int e = threadIdx.x; e < B * F.LQ; e += blockDim.x) {
    const int b = e >> F.logQ, kq = e & (F.LQ - 1);
    const int k = k0 + b;
    double2 v = make_double2(0.0, 0.0);
    if (k < F.HP)
      for (int g = 0; g < F.G; ++g) {
        const double2 s = S[((long long)g * 2 + f) * plane + (long long)k * F.LQ + kq];
        v.x += s.x;
        v.y += s.y;
      }
    x[e] = v;
  }
  __syncthreads();
  const double2* X = fft_batch(x, y, F.LQ, F.logQ, B, tw, true);
  for (int e = threadIdx.x; e < B * F.nQ; e += blockDim.x) {
    const int q = e / B, b = e - q * B;
    const int k = k0 + b;
    if (k < F.HP) V[((long long)f * F.nQ + q) * F.HP + k] = X[(b << F.logQ) + q];
  }
}

// Stage 3b: inverse real FFT along P of rows q in [q0, q0+B1) of face f =
// blockIdx.y (the spectrum's upper half from Hermitian symmetry); the real
// parts p < nP are the face potential.
__device__ __forceinline__ void bcfft_invp_body(const FaceGeom& F, const double2* __restrict__ V,
                                                const double2* __restrict__ tw, double* __restrict__ U, int bx,
                                                int by) {
  extern __shared__ double2 smem[];
  const int B = F.B1;
  double2* x = smem;
  double2* y = smem + B * F.LP;
  const int q0 = bx * B, f = by;
  for (int e = threadIdx.x; e < B * F.LP; e += blockDim.x) {
    const int b = e >> F.logP, k = e & (F.LP - 1);
    const int q = q0 + b;
    double2 v = make_double2(0.0, 0.0);
    if (q < F.nQ) {
      if (k < F.HP) {
        v = V[((long long)f * F.nQ + q) * F.HP + k];
      } else {
        v = V[((long long)f * F.nQ + q) * F.HP + (F.LP - k)];
        v.y = -v.y;
      }
    }
    x[e] = v;
  }
  __syncthreads();
  const double2* X = fft_batch(x, y, F.LP, F.logP, B, tw, true);
  const long long face = f == 0 ? F.face0 : F.face1;
  for (int e = threadIdx.x; e < B * F.nP; e += blockDim.x) {
    const int b = e / F.nP, p = e - b * F.nP;
    const int q = q0 + b;
    if (q < F.nQ) U[face + (long long)p * F.sP + (long long)q * F.sQ] = X[(b << F.logP) + p].x;
  }
}

__global__ void __launch_bounds__(kFftThreads) bcfft_rows_kernel(FaceGeom F, int mode, const double* __restrict__ src,
                                                                 int s0, int count, const double2* __restrict__ tw,
                                                                 double2* __restrict__ W) {
  bcfft_rows_body(F, mode, src, s0, count, tw, W, blockIdx.x, blockIdx.y);
}

__global__ void __launch_bounds__(kFftThreads) bcfft_cols_kernel(FaceGeom F, int mode, const double2* __restrict__ W,
                                                                 int s0, int count, double scale,
                                                                 const double2* __restrict__ tw,
                                                                 double* __restrict__ Dh, double2* __restrict__ S) {
  bcfft_cols_body(F, mode, W, s0, count, scale, tw, Dh, S, blockIdx.x, blockIdx.y);
}

__global__ void __launch_bounds__(kFftThreads) bcfft_invq_kernel(FaceGeom F, const double2* __restrict__ S,
                                                                 const double2* __restrict__ tw,
                                                                 double2* __restrict__ V) {
  bcfft_invq_body(F, S, tw, V, blockIdx.x, blockIdx.y);
}

__global__ void __launch_bounds__(kFftThreads) bcfft_invp_kernel(FaceGeom F, const double2* __restrict__ V,
                                                                 const double2* __restrict__ tw,
                                                                 double* __restrict__ U) {
  bcfft_invp_body(F, V, tw, U, blockIdx.x, blockIdx.y);
}

// One face pair of one run in a batched launch: its geometry and buffers,
// and per stage (rows, columns + contraction, inverse along Q, inverse along
// P) the first block of its blocks in the launch and its blocks along x.
struct FftJob {
  FaceGeom F;
  const double* C;
  double2* W;
  const double2* twP;
  const double2* twQ;
  double* Dh;
  double2* S;
  double2* V;
  double* U;
  long long start[4];
  int bx[4];
};

// One stage for every face pair of every run of a batch in one launch: block
// b belongs to the job with the largest start <= b (binary search), and runs
// that job's block (local % bx, local / bx) of the stage.
__global__ void __launch_bounds__(kFftThreads) bcfft_batch_kernel(const FftJob* __restrict__ jobs, int njobs,
                                                                  int stage) {
  const long long b = blockIdx.x;
  int lo = 0, hi = njobs - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (jobs[mid].start[stage] <= b) lo = mid;
    else hi = mid - 1;
  }
  const FftJob& J = jobs[lo];
  const FaceGeom F = J.F;
  const long long local = b - J.start[stage];
  const int bx = int(local % J.bx[stage]), by = int(local / J.bx[stage]);
  if (stage == 0) bcfft_rows_body(F, 0, J.C, 0, F.nA, J.twP, J.W, bx, by);
  else if (stage == 1) bcfft_cols_body(F, 0, J.W, 0, 0, 0.0, J.twQ, J.Dh, J.S, bx, by);
  else if (stage == 2) bcfft_invq_body(F, J.S, J.twQ, J.V, bx, by);
  else bcfft_invp_body(F, J.V, J.twP, J.U, bx, by);
}

int pow2_at_least(int v) {
  int L = 1;
  while (L < v) L <<= 1;
  return L;
}
int ilog2(int L) {
  int l = 0;
  while ((1 << l) < L) ++l;
  return l;
}

FaceGeom face_geom(const KParams& K, int axis) {
  const int n[3] = {K.nx, K.ny, K.nz};
  const long long s[3] = {1, K.nxp, (long long)K.nxp * K.nyp};
  const long long DX = 2LL * K.nx + 1, DY = 2LL * K.ny + 1;
  const long long ds[3] = {1, DX, DX * DY};
  const int P = axis == 0 ? 1 : 0, Q = axis == 2 ? 1 : 2;
  FaceGeom F;
  F.nA = n[axis];
  F.nP = n[P];
  F.nQ = n[Q];
  F.LP = pow2_at_least(2 * F.nP - 1);
  F.LQ = pow2_at_least(2 * F.nQ - 1);
  F.logP = ilog2(F.LP);
  F.logQ = ilog2(F.LQ);
  F.HP = F.LP / 2 + 1;
  F.sA = s[axis];
  F.sP = s[P];
  F.sQ = s[Q];
  F.dA = ds[axis];
  F.dP = ds[P];
  F.dQ = ds[Q];
  F.d0 = (long long)K.nx + DX * ((long long)K.ny + DY * (long long)K.nz);
  F.base = 1 + K.nxp * (1 + (long long)K.nyp * 1);
  F.face0 = F.base - F.sA;                       // plane 0 along A, tangential (1, 1)
  F.face1 = F.base + (long long)F.nA * F.sA;     // plane nA + 1
  F.B1 = std::max(1, std::min(16, kRowElems / F.LP));
  F.B2 = std::max(1, kColElems / F.LQ);  // B2 * LQ == kColElems (LQ a power of two <= kColElems)
  const int colblocks = (F.HP + F.B2 - 1) / F.B2;
  F.G = std::max(1, std::min(F.nA, (4 * 148 + colblocks - 1) / colblocks));
  return F;
}

bool fits(const FaceGeom& F) { return F.LP <= kRowElems && F.LQ <= kColElems; }

}  // namespace

// Device scratch of the FFT BCpotentials: per face axis the slice transforms,
// shared stage buffers, twiddle tables.
long long bcpot_fft_bytes(const KParams& K) {
  const int flows[3] = {K.xflow, K.yflow, K.zflow};
  long long dh = 0, w = 0, s = 0, v = 0, tw = 0;
  for (int a = 0; a < 3; ++a) {
    if (!flows[a]) continue;
    FaceGeom F = face_geom(K, a);
    dh += (long long)F.nA * F.HP * F.LQ * 8;
    w += std::max((long long)F.nA * F.nQ, (long long)F.LQ) * F.HP * 16;
    s += (long long)F.G * 2 * F.HP * F.LQ * 16;
    v += 2LL * F.nQ * F.HP * 16;
    tw += (long long)(F.LP + F.LQ) * 16;
  }
  return dh + w + s + v + tw;
}

int bcpot_fft_supported(const KParams& K) {
  const int flows[3] = {K.xflow, K.yflow, K.zflow};
  for (int a = 0; a < 3; ++a)
    if (flows[a] && !fits(face_geom(K, a))) return 0;
  return 1;
}

namespace {

// One face pair's plan and buffers: its own stage buffers, so that the face
// pairs of a run can go through a batched stage at the same time.
struct AxisPlan {
  FaceGeom F;
  double* Dh = nullptr;
  double2* twP = nullptr;
  double2* twQ = nullptr;
  double2* W = nullptr;  // row transforms
  long long w_elems = 0;
  double2* S = nullptr;  // the contraction's group partials
  double2* V = nullptr;  // face spectra after the inverse along Q
};

void twiddles(int L, std::vector<double2>& t) {
  const double pi = 3.14159265358979323846264338327950288;
  t.assign(std::max(1, L), make_double2(1.0, 0.0));
  for (int k = 0; k < L; ++k) {
    // exp(-2 pi i k / L) from the FP64 cosine and sine of the angle
    const double ang = 2.0 * pi * (double)k / (double)L;
    t[k] = make_double2(std::cos(ang), -std::sin(ang));
  }
}

size_t smem_rows(const FaceGeom& F) { return sizeof(double2) * 2 * (size_t)F.B1 * F.LP; }
size_t smem_cols(const FaceGeom& F) { return sizeof(double2) * 2 * (size_t)F.B2 * F.LQ; }

}  // namespace

struct BcFft {
  AxisPlan ax[3];
  bool ready = false;  // slice transforms of the current D
};

static int set_smem_limits() {
  static bool done = false;
  if (done) return PICARD_OK;
  const int big = 2 * 16 * kRowElems;  // 64 KB
  PICARD_CUDA(cudaFuncSetAttribute(bcfft_rows_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  PICARD_CUDA(cudaFuncSetAttribute(bcfft_cols_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  PICARD_CUDA(cudaFuncSetAttribute(bcfft_invq_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  PICARD_CUDA(cudaFuncSetAttribute(bcfft_invp_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  PICARD_CUDA(cudaFuncSetAttribute(bcfft_batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  done = true;
  return PICARD_OK;
}

int bcpot_fft_alloc(picard_ctx* c) {
  if (c->bcfft) return PICARD_OK;
  if (!bcpot_fft_supported(c->K)) return fail(PICARD_ERR_BAD_ARG, "FFT BCpotentials: a face is longer than 1024 cells");
  PICARD_TRY(set_smem_limits());
  BcFft* B = new BcFft();
  c->bcfft = B;
  const KParams& K = c->K;
  const int flows[3] = {K.xflow, K.yflow, K.zflow};
  for (int a = 0; a < 3; ++a) {
    if (!flows[a]) continue;
    AxisPlan& A = B->ax[a];
    A.F = face_geom(K, a);
    const FaceGeom& F = A.F;
    void* p = nullptr;
    PICARD_TRY(dev_alloc(c, &p, sizeof(double) * (size_t)F.nA * F.HP * F.LQ));
    A.Dh = static_cast<double*>(p);
    std::vector<double2> t;
    twiddles(F.LP, t);
    PICARD_TRY(dev_alloc(c, &p, sizeof(double2) * t.size()));
    A.twP = static_cast<double2*>(p);
    // no wait: an asynchronous copy from pageable memory returns once the host
    // data is staged, so the vector may be refilled
    PICARD_CUDA(cudaMemcpyAsync(A.twP, t.data(), sizeof(double2) * t.size(), cudaMemcpyHostToDevice, c->st));
    c->stats.h2d_bytes += (int64_t)(sizeof(double2) * t.size());
    twiddles(F.LQ, t);
    PICARD_TRY(dev_alloc(c, &p, sizeof(double2) * t.size()));
    A.twQ = static_cast<double2*>(p);
    PICARD_CUDA(cudaMemcpyAsync(A.twQ, t.data(), sizeof(double2) * t.size(), cudaMemcpyHostToDevice, c->st));
    c->stats.h2d_bytes += (int64_t)(sizeof(double2) * t.size());
    // at least one kernel slice's rows, for the slice transforms
    const long long w = std::max((long long)F.nA * F.nQ, (long long)F.LQ) * F.HP;
    PICARD_TRY(dev_alloc(c, &p, sizeof(double2) * (size_t)w));
    A.W = static_cast<double2*>(p);
    A.w_elems = w;
    PICARD_TRY(dev_alloc(c, &p, sizeof(double2) * (size_t)F.G * 2 * F.HP * F.LQ));
    A.S = static_cast<double2*>(p);
    PICARD_TRY(dev_alloc(c, &p, sizeof(double2) * 2 * (size_t)F.nQ * F.HP));
    A.V = static_cast<double2*>(p);
  }
  return PICARD_OK;
}

void bcpot_fft_free(picard_ctx* c) {
  delete c->bcfft;
  c->bcfft = nullptr;
}

void bcpot_fft_invalidate(picard_ctx* c) {
  if (c->bcfft) c->bcfft->ready = false;
}

// Slice transforms of D for every face axis: chunks of slices through the
// row and column stages (mode 1).
static int prepare(picard_ctx* c) {
  BcFft* B = c->bcfft;
  const double K0 = 1.0 / (2.0 * kTau * kEps0);
  for (int a = 0; a < 3; ++a) {
    AxisPlan& A = B->ax[a];
    if (!A.Dh) continue;
    const FaceGeom& F = A.F;
    const double scale = K0 / ((double)F.LP * (double)F.LQ);
    const int chunk = int(std::max<long long>(1, A.w_elems / ((long long)F.LQ * F.HP)));
    for (int s0 = 0; s0 < F.nA; s0 += chunk) {
      const int cnt = std::min(chunk, F.nA - s0);
      dim3 g1((cnt + F.B1 - 1) / F.B1, F.LQ);
      note_launch();
      // slice index a <-> normal offset s0 + a + 1 (the D table at offset a + 1 along A)
      bcfft_rows_kernel<<<g1, kFftThreads, smem_rows(F), c->st>>>(F, 1, c->D + F.dA, s0, cnt, A.twP, A.W);
      PICARD_CUDA(cudaGetLastError());
      dim3 g2((F.HP + F.B2 - 1) / F.B2, cnt);
      note_launch();
      bcfft_cols_kernel<<<g2, kFftThreads, smem_cols(F), c->st>>>(F, 1, A.W, s0, cnt, scale, A.twQ, A.Dh, nullptr);
      PICARD_CUDA(cudaGetLastError());
    }
  }
  B->ready = true;
  return PICARD_OK;
}

int bc_potentials_fft(picard_ctx* c) {
  PICARD_TRY(bcpot_fft_alloc(c));
  BcFft* B = c->bcfft;
  if (!B->ready) PICARD_TRY(prepare(c));
  PICARD_CUDA(cudaMemsetAsync(c->U, 0, sizeof(double) * c->K.nodes, c->st));  // BCpotentials.f90:36
  for (int a = 0; a < 3; ++a) {
    AxisPlan& A = B->ax[a];
    if (!A.Dh) continue;
    const FaceGeom& F = A.F;
    dim3 g1((F.nA + F.B1 - 1) / F.B1, F.nQ);
    note_launch();
    bcfft_rows_kernel<<<g1, kFftThreads, smem_rows(F), c->st>>>(F, 0, c->C, 0, F.nA, A.twP, A.W);
    PICARD_CUDA(cudaGetLastError());
    dim3 g2((F.HP + F.B2 - 1) / F.B2, F.G);
    note_launch();
    bcfft_cols_kernel<<<g2, kFftThreads, smem_cols(F), c->st>>>(F, 0, A.W, 0, 0, 0.0, A.twQ, A.Dh, A.S);
    PICARD_CUDA(cudaGetLastError());
    dim3 g3((F.HP + F.B2 - 1) / F.B2, 2);
    note_launch();
    bcfft_invq_kernel<<<g3, kFftThreads, smem_cols(F), c->st>>>(F, A.S, A.twQ, A.V);
    PICARD_CUDA(cudaGetLastError());
    dim3 g4((F.nQ + F.B1 - 1) / F.B1, 2);
    note_launch();
    bcfft_invp_kernel<<<g4, kFftThreads, smem_rows(F), c->st>>>(F, A.V, A.twP, c->U);
    PICARD_CUDA(cudaGetLastError());
  }
  return PICARD_OK;
}

// BCpotentials of many runs: the FFT runs' face pairs advance stage by stage,
// each stage one launch over all of them on the batch stream (after every
// such run's U is zeroed and its slice transforms exist, on its own stream);
// the other runs take their own method on their own streams.
int bc_potentials_batch(picard_ctx** ctxs, int n, cudaStream_t bst, cudaEvent_t* rev, cudaEvent_t bev) {
  std::vector<FftJob> jobs;
  std::vector<int> fft_runs;
  long long total[4] = {0, 0, 0, 0};
  size_t smem[4] = {0, 0, 0, 0};
  for (int r = 0; r < n; ++r) {
    picard_ctx* c = ctxs[r];
    if (c->bcpot_tensor != PICARD_BCPOT_FFT) {
      PICARD_TRY(bc_potentials_async(c));
      continue;
    }
    PICARD_TRY(bcpot_fft_alloc(c));
    BcFft* B = c->bcfft;
    if (!B->ready) PICARD_TRY(prepare(c));
    PICARD_CUDA(cudaMemsetAsync(c->U, 0, sizeof(double) * c->K.nodes, c->st));  // BCpotentials.f90:36
    PICARD_CUDA(cudaEventRecord(rev[r], c->st));
    PICARD_CUDA(cudaStreamWaitEvent(bst, rev[r], 0));
    fft_runs.push_back(r);
    for (int a = 0; a < 3; ++a) {
      AxisPlan& A = B->ax[a];
      if (!A.Dh) continue;
      FftJob J;
      J.F = A.F;
      J.C = c->C;
      J.W = A.W;
      J.twP = A.twP;
      J.twQ = A.twQ;
      J.Dh = A.Dh;
      J.S = A.S;
      J.V = A.V;
      J.U = c->U;
      const FaceGeom& F = A.F;
      const int bxs[4] = {(F.nA + F.B1 - 1) / F.B1, (F.HP + F.B2 - 1) / F.B2, (F.HP + F.B2 - 1) / F.B2,
                          (F.nQ + F.B1 - 1) / F.B1};
      const int bys[4] = {F.nQ, F.G, 2, 2};
      const size_t sm[4] = {smem_rows(F), smem_cols(F), smem_cols(F), smem_rows(F)};
      for (int t = 0; t < 4; ++t) {
        J.start[t] = total[t];
        J.bx[t] = bxs[t];
        total[t] += (long long)bxs[t] * bys[t];
        smem[t] = std::max(smem[t], sm[t]);
      }
      jobs.push_back(J);
    }
  }
  if (jobs.empty()) return PICARD_OK;
  // the job table lives on the batch stream until its last launch
  void* dj = nullptr;
  PICARD_CUDA(cudaMallocAsync(&dj, sizeof(FftJob) * jobs.size(), bst));
  PICARD_CUDA(cudaMemcpyAsync(dj, jobs.data(), sizeof(FftJob) * jobs.size(), cudaMemcpyHostToDevice, bst));
  for (int t = 0; t < 4; ++t) {
    note_launch();
    bcfft_batch_kernel<<<(unsigned)total[t], kFftThreads, smem[t], bst>>>(static_cast<const FftJob*>(dj),
                                                                            (int)jobs.size(), t);
    PICARD_CUDA(cudaGetLastError());
  }
  PICARD_CUDA(cudaFreeAsync(dj, bst));
  PICARD_CUDA(cudaEventRecord(bev, bst));
  for (int r : fft_runs) PICARD_CUDA(cudaStreamWaitEvent(ctxs[r]->st, bev, 0));
  return PICARD_OK;
}

}  // namespace picard
