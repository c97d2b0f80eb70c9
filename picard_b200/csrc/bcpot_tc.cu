// bcpot_tc.cu -- BCpotentials (BCpotentials.f90:51-139) on the 5th-generation
// tensor cores.
//
// For one face axis, with (p1, p2) the in-plane coordinates of a face node and
// q the coordinate along the normal,
//   U_f(p1, p2) = sum_q sum_q1 sum_q2 C(q, q1, q2) D_f(q, q1 - p1, q2 - p2),
// where f = 0, 1 are the two faces of the axis (they differ only in the normal
// offset of D).  For a fixed plane q and row shift d = q1 - p1 this is a GEMM
//   U_f(p1, :) += C(q, p1 + d, :) . T_{q,d,f},  T[q2, p2] = D_f(q, d, q2 - p2)
// (T is Toeplitz).  A CTA owns a 128 x 256 output tile -- 128 rows p1, and
// 128 columns p2 of each face side by side -- and accumulates it in tensor
// memory over a slice of the (q, d) pairs (split-K over all SMs).
//
// Precision: every FP64 operand is split into three BF16 parts
// (x = x1 + x2 + x3, 24 significant bits) and each K-step issues the six
// products x_i y_j with i + j <= 4.  The FP32 accumulator in TMEM is folded
// into an FP64 partial of the CTA every kFlushChunks K-chunks, so FP32
// rounding only accumulates over short runs.  A reduction kernel sums the
// per-CTA partials in a fixed order.
//
// Operands sit in shared memory in the canonical K-major no-swizzle layout of
// tcgen05 (8-row x 16-byte core matrices) with rows 16 bytes apart
// throughout: element (r, k) of an operand whose K blocks are L bytes apart
// lives at byte (k / 8) * L + r * 16 + (k % 8) * 2, i.e. leading-byte offset L
// between the two K core matrices of an instruction and stride-byte offset
// 128 between 8-row groups.  Uniform 16-byte rows let a row shift be a plain
// change of the descriptor's start address (see the kernel).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>

#include "common.cuh"
#include "grid.cuh"

namespace picard {

namespace {

constexpr int kTcM = 128;          // rows p1 per tile
constexpr int kTcHalfN = 128;      // columns p2 per face
constexpr int kTcN = 2 * kTcHalfN; // both faces
constexpr int kTcKC = 64;          // K (q2) per chunk
constexpr int kTcThreads = 128;
constexpr int kFlushChunks = 8;    // K-chunks between FP64 folds of the accumulator
constexpr long long kTcSpin = 1LL << 26;

struct TcAxis {
  int axis;        // normal axis
  int n1, n2, nn;  // in-plane extents (p1, p2) and normal extent
  int n2pad;       // n2 rounded up to kTcKC
  int mtiles, ntiles, splits;
};

__device__ inline uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46);
}

__device__ inline void split3(float x, __nv_bfloat16& a, __nv_bfloat16& b, __nv_bfloat16& c) {
  a = __float2bfloat16_rn(x);
  float r = x - __bfloat162float(a);
  b = __float2bfloat16_rn(r);
  r = r - __bfloat162float(b);
  c = __float2bfloat16_rn(r);
}

__device__ inline bool mbar_wait_tc(uint32_t mbar, uint32_t phase) {
  for (long long it = 0; it < kTcSpin; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(mbar), "r"(phase)
        : "memory");
    if (done) return true;
  }
  return false;
}

// C (FP64 node array) -> three BF16 planes per face axis,
// Cs[s][q][row][q2] with row = p1 - 1 in [0, n1), q2 - 1 in [0, n2pad).
__global__ void split_charge_kernel(KParams P, TcAxis X, const double* __restrict__ C, __nv_bfloat16* Cs) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  long long per = (long long)X.nn * X.n1 * X.n2pad;
  if (t >= per) return;
  int q2 = int(t % X.n2pad);
  int row = int((t / X.n2pad) % X.n1);
  int q = int(t / ((long long)X.n2pad * X.n1));
  float v = 0.0f;
  if (q2 < X.n2) {
    int ci, cj, ck;
    if (X.axis == 0) ci = q + 1, cj = row + 1, ck = q2 + 1;
    else if (X.axis == 1) ci = row + 1, cj = q + 1, ck = q2 + 1;
    else ci = row + 1, cj = q2 + 1, ck = q + 1;
    v = (float)C[node_index(P, ci, cj, ck)];
  }
  __nv_bfloat16 a, b, c;
  split3(v, a, b, c);
  Cs[t] = a;
  Cs[per + t] = b;
  Cs[2 * per + t] = c;
}

// D index (1-based) of face f for plane q, shift d (along p1), offset o2 (along p2).
__device__ inline long long d_index(const KParams& P, const TcAxis& X, int f, int q, int d, int o2) {
  int on = f == 0 ? q : q - (X.nn + 1);
  int a, b, c;
  if (X.axis == 0) a = P.nx + 1 + on, b = P.ny + 1 + d, c = P.nz + 1 + o2;
  else if (X.axis == 1) a = P.nx + 1 + d, b = P.ny + 1 + on, c = P.nz + 1 + o2;
  else a = P.nx + 1 + d, b = P.ny + 1 + o2, c = P.nz + 1 + on;
  long long DX = 2LL * P.nx + 1, DY = 2LL * P.ny + 1;
  return (long long)(a - 1) + DX * ((long long)(b - 1) + DY * (long long)(c - 1));
}

// ----------------------------------------------------------------- kernel
//
// Per step (q, d, K-chunk kc) the CTA issues, for each face f, the six split
// products of
//   Acc_f[r][n'] += sum_k A[r][k] B_f[n'][k],   k = q2 - 1 - k0 in [0, 64),
// with A[r][k] = C(q, m0 + r + d, q2) and B_f[n'][k] = W_f(q2 - p2), where the
// output columns are stored reversed, n' = 127 - (p2 - 1 - n0).  Then
//   q2 - p2 = o_min + k + n',   o_min = k0 - n0 - 127,
// so B_f is a sliding window: with Z[u] = (w[u], ..., w[u+7]) (16 bytes, w[j] =
// W_f(o_min + j)), element (n', k) is Z[n' + 8 floor(k/8)][k mod 8], i.e. a
// K-major no-swizzle operand with rows 16 bytes apart and both core-matrix
// strides 128 bytes.  A is read from a tall buffer T holding rows m0 + dA ..
// m0 + dA + 256 of plane q (K-major, rows 16 bytes apart, the eight K blocks
// kRT * 16 bytes apart): shift d starts (d - dA) * 16 bytes further in.  T is
// loaded (cp.async, zero-filled outside the face) once per run of up to kDB
// consecutive shifts; Z is rebuilt per step from a 191-value window of D,
// double buffered so that the MMAs of one step overlap the build of the next,
// and the D values of the next step are prefetched into registers.
constexpr int kDB = 128;            // shifts served by one T buffer
constexpr int kRT = 257;            // T rows (>= kDB + 127; odd multiple of 16 B keeps cp.async conflict-free)
constexpr int kZN = 184;            // Z entries per (face, split): n' + 8 floor(k/8) <= 127 + 56
constexpr int kWL = 192;            // window values per (face, split) (191 used)
constexpr int kWUsed = 191;
constexpr size_t kTSplit = (size_t)8 * kRT * 16;     // bytes of one split of T
constexpr size_t kZFS = (size_t)kZN * 16;            // bytes of one (face, split) Z array
constexpr size_t kSmemT = 3 * kTSplit;
constexpr size_t kSmemZ = 2 * 2 * 3 * kZFS;          // [buf][face][split]
constexpr size_t kSmemW = (size_t)2 * 3 * kWL * 2;   // [face][split][kWL] bf16
constexpr size_t kSmemX = (size_t)4 * 32 * 33 * 8;   // per-warp 32 x 32 FP64 transpose tiles
constexpr size_t kTcSmem = kSmemT + kSmemZ + kSmemW + kSmemX;
constexpr int kFoldsPerFlush = 16;  // on-chip folds between FP64 flushes
// kind::f16 instruction descriptor: F32 accumulate, BF16 A and B, both
// K-major, M = 128, N = 128 (one face per instruction).
constexpr uint32_t kIdescFace = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kTcHalfN >> 3) << 17) |
                                ((uint32_t)(kTcM >> 4) << 24);
constexpr int kPrefetch = 3;  // D values per thread per step (2 * 191 <= 3 * 128)

__global__ void __launch_bounds__(kTcThreads, 1)
    bcpot_tc_kernel(KParams P, TcAxis X, const __nv_bfloat16* __restrict__ Cs, const double* __restrict__ D,
                    double* partial, int* err) {
  extern __shared__ __align__(1024) unsigned char smem[];
  unsigned char* sT = smem;                   // [3][8][kRT][16 B]
  unsigned char* sZ = smem + kSmemT;          // [2][2][3][kZN][16 B]
  __nv_bfloat16* sWin = reinterpret_cast<__nv_bfloat16*>(smem + kSmemT + kSmemZ);  // [2][3][kWL]
  double* sX = reinterpret_cast<double*>(smem + kSmemT + kSmemZ + kSmemW);         // [4][32][33]
  __shared__ __align__(8) unsigned long long mbar[2];
  __shared__ uint32_t tmem_base;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  const int tile = blockIdx.x / X.splits, split = blockIdx.x % X.splits;
  const int mt = tile / X.ntiles, nt = tile % X.ntiles;
  const int m0 = mt * kTcM, n0 = nt * kTcHalfN;
  const int rows_hi = (m0 + kTcM < X.n1) ? m0 + kTcM : X.n1;
  const int dlo = 1 - rows_hi, dhi = X.n1 - m0 - 1;
  const int nd = dhi - dlo + 1;
  const long long npairs = (long long)X.nn * nd;
  const long long pbeg = npairs * split / X.splits, pend = npairs * (split + 1) / X.splits;
  const int nchunks = X.n2pad / kTcKC;
  const long long per = (long long)X.nn * X.n1 * X.n2pad;  // elements of one split of Cs
  double* part = partial + (long long)blockIdx.x * kTcM * kTcN;

  const uint32_t mb0 = (uint32_t)__cvta_generic_to_shared(&mbar[0]);
  const uint32_t mb1 = (uint32_t)__cvta_generic_to_shared(&mbar[1]);
  if (warp == 0) {
    uint32_t dst = (uint32_t)__cvta_generic_to_shared(&tmem_base);
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dst), "r"(2 * kTcN)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mb0) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mb1) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  for (int e = tid; e < kTcM * kTcN; e += kTcThreads) part[e] = 0.0;
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_base;
  uint32_t phase[2] = {0, 0};
  bool pending[2] = {false, false};
  int since_flush = 0;
  bool ok = true;

  auto wait_buf = [&](int b) -> bool {
    if (!pending[b]) return true;
    bool r = mbar_wait_tc(b ? mb1 : mb0, phase[b]);
    phase[b] ^= 1;
    pending[b] = false;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    return r;
  };
  auto drain = [&]() -> bool {
    bool a = wait_buf(0);
    bool b = wait_buf(1);
    return a && b;
  };
  // Two on-chip levels before FP64.  The MMAs accumulate a segment of
  // kFlushChunks steps in TMEM columns [0, 256); fold() adds it (FP32) into
  // a running sum in columns [256, 512) and is cheap (TMEM loads and stores
  // only); every kFoldsPerFlush folds flush64() adds the running sum into the
  // CTA's FP64 partial, staged through a per-warp shared-memory transpose so
  // that the global read-modify-writes are coalesced.  Thread = TMEM lane =
  // tile row; TMEM column f*128 + n' is partial column f*128 + 127 - n'.
  int folds = 0;
  auto fold = [&]() {
    for (int col = 0; col < kTcN; col += 16) {
      uint32_t a[16], r[16];
      const uint32_t lanebase = tmem + ((uint32_t)(32 * warp) << 16);
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
          : "=r"(a[0]), "=r"(a[1]), "=r"(a[2]), "=r"(a[3]), "=r"(a[4]), "=r"(a[5]), "=r"(a[6]), "=r"(a[7]),
            "=r"(a[8]), "=r"(a[9]), "=r"(a[10]), "=r"(a[11]), "=r"(a[12]), "=r"(a[13]), "=r"(a[14]), "=r"(a[15])
          : "r"(lanebase + (uint32_t)col));
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
          : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
            "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
          : "r"(lanebase + (uint32_t)(kTcN + col)));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        const float sum = folds == 0 ? __uint_as_float(a[j]) : __fadd_rn(__uint_as_float(r[j]), __uint_as_float(a[j]));
        r[j] = __float_as_uint(sum);
      }
      asm volatile(
          "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16};"
          ::"r"(lanebase + (uint32_t)(kTcN + col)), "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]),
            "r"(r[5]), "r"(r[6]), "r"(r[7]), "r"(r[8]), "r"(r[9]), "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]),
            "r"(r[14]), "r"(r[15])
          : "memory");
    }
    asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    ++folds;
  };
  auto flush64 = [&]() {
    double* X = sX + warp * 32 * 33;
    for (int col = 0; col < kTcN; col += 32) {
      uint32_t r[32];
      const uint32_t addr = tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)(kTcN + col);
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
          : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
            "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
          : "r"(addr));
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
          : "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
            "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
          : "r"(addr + 16u));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
      for (int j = 0; j < 32; ++j) X[lane * 33 + j] = (double)__uint_as_float(r[j]);
      __syncwarp();
      // lane = TMEM column col + lane, i.e. partial column f*128 + 127 - n'
      const int f = col / kTcHalfN, nprime = col % kTcHalfN + lane;
      for (int rr = 0; rr < 32; ++rr) {
        double* g = part + (long long)(32 * warp + rr) * kTcN + f * kTcHalfN + (kTcHalfN - 1 - nprime);
        *g += X[rr * 33 + lane];
      }
      __syncwarp();
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    folds = 0;
  };
  auto flush = [&]() {
    fold();
    if (folds == kFoldsPerFlush) flush64();
  };

  // D values of one step into registers: item e = tid + 128 m -> face e / 191,
  // window index e % 191
  double pre[kPrefetch];
  auto prefetch = [&](int q, int d, int kc) {
    const int o_min = kc * kTcKC - n0 - (kTcHalfN - 1);
#pragma unroll
    for (int m = 0; m < kPrefetch; ++m) {
      const int e = tid + kTcThreads * m;
      double v = 0.0;
      if (e < 2 * kWUsed) {
        const int f = e / kWUsed, j = e % kWUsed;
        const int o2 = o_min + j;
        if (o2 >= -(X.n2 - 1) && o2 <= X.n2 - 1) v = __ldg(D + d_index(P, X, f, q, d, o2));
      }
      pre[m] = v;
    }
  };
  auto step_of = [&](int kc, long long pr, int& q, int& d) {
    q = int(pr / nd) + 1;
    d = dlo + int(pr % nd);
    (void)kc;
  };

  int step = 0;
  if (pbeg < pend) {
    int q, d;
    step_of(0, pbeg, q, d);
    prefetch(q, d, 0);
  }
  for (int kc = 0; kc < nchunks && ok; ++kc) {
    const int k0 = kc * kTcKC;
    int Tq = -1, TdA = 0;
    for (long long pr = pbeg; pr < pend && ok; ++pr) {
      int q, d;
      step_of(kc, pr, q, d);
      if (q != Tq || d >= TdA + kDB) {
        // every MMA that reads T is done before T is rewritten
        if (!__syncthreads_and(drain() ? 1 : 0)) { ok = false; break; }
        Tq = q;
        TdA = d;
        const int rho0 = m0 + TdA;
        const uint32_t tbase = (uint32_t)__cvta_generic_to_shared(sT);
        for (int e = tid; e < 3 * kRT * 8; e += kTcThreads) {
          const int kb = e & 7, rest = e >> 3;
          const int t = rest % kRT, sp = rest / kRT;
          const int rho = rho0 + t;
          const bool in = rho >= 0 && rho < X.n1;
          const __nv_bfloat16* g =
              in ? Cs + sp * per + ((long long)(q - 1) * X.n1 + rho) * X.n2pad + k0 + kb * 8 : Cs;
          const uint32_t dst = tbase + (uint32_t)(sp * kTSplit + (size_t)kb * kRT * 16 + (size_t)t * 16);
          asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(g), "r"(in ? 16 : 0)
                       : "memory");
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
        asm volatile("cp.async.wait_group 0;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
      }
      const int b = step & 1;
      // the MMAs of step - 2 read Z[b]
      if (!__syncthreads_and(wait_buf(b) ? 1 : 0)) { ok = false; break; }
      // window of this step from the prefetched D values
#pragma unroll
      for (int m = 0; m < kPrefetch; ++m) {
        const int e = tid + kTcThreads * m;
        if (e < 2 * kWUsed) {
          const int f = e / kWUsed, j = e % kWUsed;
          __nv_bfloat16 a0, a1, a2;
          split3((float)pre[m], a0, a1, a2);
          sWin[(f * 3 + 0) * kWL + j] = a0;
          sWin[(f * 3 + 1) * kWL + j] = a1;
          sWin[(f * 3 + 2) * kWL + j] = a2;
        }
      }
      if (tid < 6) sWin[tid * kWL + kWUsed] = __float2bfloat16_rn(0.0f);
      __syncthreads();
      // Z[b][f][s][u] = w[u .. u+7]
      unsigned char* zb = sZ + (size_t)b * 2 * 3 * kZFS;
      for (int e = tid; e < 6 * kZN; e += kTcThreads) {
        const int fs = e / kZN, u = e % kZN;
        const __nv_bfloat16* w = sWin + fs * kWL + u;
        __align__(16) __nv_bfloat16 v[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) v[j] = w[j];
        *reinterpret_cast<uint4*>(zb + (size_t)fs * kZFS + (size_t)u * 16) = *reinterpret_cast<const uint4*>(v);
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      __syncthreads();
      if (tid == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t tb = (uint32_t)__cvta_generic_to_shared(sT) + (uint32_t)(d - TdA) * 16u;
        const uint32_t zs = (uint32_t)__cvta_generic_to_shared(zb);
        const int pa[6] = {0, 0, 1, 0, 1, 2}, pb[6] = {0, 1, 0, 2, 1, 0};
#pragma unroll
        for (int f = 0; f < 2; ++f) {
#pragma unroll
          for (int ks = 0; ks < kTcKC / 16; ++ks) {
#pragma unroll
            for (int t = 0; t < 6; ++t) {
              const uint32_t a_addr = tb + (uint32_t)(pa[t] * kTSplit + (size_t)(2 * ks) * kRT * 16);
              const uint32_t b_addr = zs + (uint32_t)((f * 3 + pb[t]) * kZFS + ks * 256);
              const uint64_t adesc = smem_desc(a_addr, kRT * 16, 128);
              const uint64_t bdesc = smem_desc(b_addr, 128, 128);
              const uint32_t acc = (since_flush == 0 && ks == 0 && t == 0) ? 0u : 1u;
              asm volatile(
                  "{\n\t.reg .pred p;\n\t"
                  "setp.ne.b32 p, %4, 0;\n\t"
                  "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
                  ::"r"(tmem + (uint32_t)(f * kTcHalfN)), "l"(adesc), "l"(bdesc), "r"(kIdescFace), "r"(acc)
                  : "memory");
            }
          }
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(b ? mb1 : mb0)
                     : "memory");
      }
      pending[b] = true;
      ++step;
      // D values of the next step
      {
        long long npr = pr + 1;
        int nkc = kc;
        if (npr >= pend) {
          npr = pbeg;
          ++nkc;
        }
        if (nkc < nchunks) {
          int nq, ndd;
          step_of(nkc, npr, nq, ndd);
          prefetch(nq, ndd, nkc);
        }
      }
      if (++since_flush == kFlushChunks) {
        if (!__syncthreads_and(drain() ? 1 : 0)) { ok = false; break; }
        flush();
        __syncthreads();
        since_flush = 0;
      }
    }
  }
  if (ok && !__syncthreads_and(drain() ? 1 : 0)) ok = false;
  if (ok && since_flush > 0) fold();
  if (ok && folds > 0) flush64();
  if (!ok) {
    if (tid == 0) atomicCAS(err, 0, int(kDevTimeout));
    drain();  // bounded: let outstanding MMAs finish before TMEM is released
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * kTcN) : "memory");
  }
}


// U on both faces of the axis = (sum over splits of the partial tiles) / (4 pi eps0).
__global__ void bcpot_reduce_kernel(KParams P, TcAxis X, const double* partial, double* U) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  long long total = (long long)X.mtiles * X.ntiles * kTcM * kTcN;
  if (t >= total) return;
  int col = int(t % kTcN);
  int row = int((t / kTcN) % kTcM);
  int tile = int(t / ((long long)kTcN * kTcM));
  int mt = tile / X.ntiles, nt = tile % X.ntiles;
  int f = col / kTcHalfN;
  int p1 = mt * kTcM + row + 1, p2 = nt * kTcHalfN + col % kTcHalfN + 1;
  if (p1 > X.n1 || p2 > X.n2) return;
  double s = 0.0;
  for (int sp = 0; sp < X.splits; ++sp)
    s += partial[((long long)(tile * X.splits + sp) * kTcM + row) * kTcN + col];
  const double scale = 1.0 / (2.0 * kTau * kEps0);
  int fixed = f == 0 ? 0 : (X.axis == 0 ? P.nx + 1 : (X.axis == 1 ? P.ny + 1 : P.nz + 1));
  long long g;
  if (X.axis == 0) g = node_index(P, fixed, p1, p2);
  else if (X.axis == 1) g = node_index(P, p1, fixed, p2);
  else g = node_index(P, p1, p2, fixed);
  U[g] = s * scale;
}

TcAxis tc_axis(const KParams& P, int axis, int sms) {
  TcAxis X;
  X.axis = axis;
  if (axis == 0) X.n1 = P.ny, X.n2 = P.nz, X.nn = P.nx;
  else if (axis == 1) X.n1 = P.nx, X.n2 = P.nz, X.nn = P.ny;
  else X.n1 = P.nx, X.n2 = P.ny, X.nn = P.nz;
  X.n2pad = (X.n2 + kTcKC - 1) / kTcKC * kTcKC;
  X.mtiles = (X.n1 + kTcM - 1) / kTcM;
  X.ntiles = (X.n2 + kTcHalfN - 1) / kTcHalfN;
  int tiles = X.mtiles * X.ntiles;
  X.splits = sms / tiles;
  if (X.splits < 1) X.splits = 1;
  return X;
}

}  // namespace

size_t bcpot_tc_smem_bytes(const KParams& P) {
  (void)P;
  return kTcSmem;
}

void bcpot_tc_scratch(const KParams& P, long long* cs_elems, long long* partial_elems) {
  long long cs = 0, pe = 0;
  for (int axis = 0; axis < 3; ++axis) {
    TcAxis X = tc_axis(P, axis, 148);
    long long c = 3LL * X.nn * X.n1 * X.n2pad;
    long long p = (long long)X.mtiles * X.ntiles * X.splits * kTcM * kTcN;
    cs = c > cs ? c : cs;
    pe = p > pe ? p : pe;
  }
  *cs_elems = cs;
  *partial_elems = pe;
}

cudaError_t launch_bc_potentials_tc(const KParams& P, const double* C, const double* D, double* U, void* cs_buf,
                                    double* partial, int* err, cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(U, 0, sizeof(double) * P.nodes, st);
  if (e != cudaSuccess) return e;
  const size_t smem = bcpot_tc_smem_bytes(P);
  static size_t attr = 0;
  if (attr < smem) {
    e = cudaFuncSetAttribute(bcpot_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    attr = smem;
  }
  const int flows[3] = {P.xflow, P.yflow, P.zflow};
  __nv_bfloat16* Cs = static_cast<__nv_bfloat16*>(cs_buf);
  for (int axis = 0; axis < 3; ++axis) {
    if (!flows[axis]) continue;
    TcAxis X = tc_axis(P, axis, 148);
    long long per = (long long)X.nn * X.n1 * X.n2pad;
    note_launch();
    split_charge_kernel<<<(unsigned)((per + 255) / 256), 256, 0, st>>>(P, X, C, Cs);
    note_launch();
    bcpot_tc_kernel<<<X.mtiles * X.ntiles * X.splits, kTcThreads, smem, st>>>(P, X, Cs, D, partial, err);
    long long outs = (long long)X.mtiles * X.ntiles * kTcM * kTcN;
    note_launch();
    bcpot_reduce_kernel<<<(unsigned)((outs + 255) / 256), 256, 0, st>>>(P, X, partial, U);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

}  // namespace picard
