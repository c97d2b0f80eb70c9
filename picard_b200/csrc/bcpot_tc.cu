// bcpot_tc.cu -- BCpotentials (BCpotentials.f90:51-139) on the 5th-generation
// tensor cores.
//
// For one face axis, with (p1, p2) the in-plane coordinates of a face node and
// q the coordinate along the normal,
//   U_f(p1, p2) = sum_q sum_q1 sum_q2 C(q, q1, q2) D_f(q, q1 - p1, q2 - p2),
// where f = 0, 1 are the two faces of the axis (they differ only in the normal
// offset of D).  For a fixed plane q and row shift d = q1 - p1 this is a GEMM
//   U_f(p1, :) += C(q, p1 + d, :) . T_{q,d,f},  T[q2, p2] = D_f(q, d, q2 - p2)
// (T is Toeplitz).  A CTA owns one face of a 128 x N output tile -- 128
// rows p1 by N columns p2, N = 64, 96 or 128 (the smallest that holds a face
// of up to 128 columns, so that narrow faces are not padded to 128) -- and
// accumulates it in tensor memory over a slice of the (q, d) pairs (split-K
// over all SMs).
//
// Precision: every FP64 operand is split into three BF16 parts
// (x = x1 + x2 + x3, 24 significant bits) and each K-step issues the six
// products x_i y_j with i + j <= 4.  Each FP32 MMA accumulation spans one
// step (N K-values); the steps are summed in tensor memory with Kahan
// compensation, and the CTA's result goes out once as FP64.  A reduction
// kernel sums the per-CTA partials in a fixed order.
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
// Two warpgroups: warps w and w + 4 share TMEM lanes 32 (w % 4) .. + 31 and
// split the accumulator columns, so folding a step and building the next
// B window take half as long between MMA batches.
constexpr int kTcThreads = 256;
constexpr long long kTcSpin = 1LL << 26;

struct TcAxis {
  int axis;        // normal axis
  int n1, n2, nn;  // in-plane extents (p1, p2) and normal extent
  int n2pad;       // n2 rounded up to the K chunk
  int N;           // columns p2 per face of a tile, also the K chunk: 64, 96 or 128
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
// A CTA owns one face f of a 128 x 128 output tile and a slice of the (q, d)
// pairs.  Per step (q, d, K-chunk kc) it issues the six split products of
//   Acc[r][n'] += sum_k A[r][k] B[n'][k],   k = q2 - 1 - k0 in [0, 128),
// with A[r][k] = C(q, m0 + r + d, q2) and B[n'][k] = W_f(q2 - p2), where the
// output columns are stored reversed, n' = 127 - (p2 - 1 - n0).  Then
//   q2 - p2 = o_min + k + n',   o_min = k0 - n0 - 127,
// so B is a sliding window: with Z[u] = (w[u], ..., w[u+7]) (16 bytes, w[j] =
// W_f(o_min + j)), element (n', k) is Z[n' + 8 floor(k/8)][k mod 8], i.e. a
// K-major no-swizzle operand with rows 16 bytes apart and both core-matrix
// strides 128 bytes.  A is read from a tall buffer T holding rows m0 + dA ..
// m0 + dA + 192 of plane q (K-major, rows 16 bytes apart, the 16 K blocks
// kRT * 16 bytes apart): shift d starts (d - dA) * 16 bytes further in.  T is
// loaded (cp.async, zero-filled outside the face) once per run of up to kDB
// consecutive shifts; Z is rebuilt per step from a 255-value window of D,
// double buffered so that the MMAs of one step overlap the build of the next,
// and the D values of the next step are prefetched into registers.
//
// Accumulation.  Tensor memory holds two FP32 accumulators (columns 0-127 and
// 128-255) used by alternate steps, and a Kahan-compensated FP32 running sum
// (sum in 256-383, compensation in 384-511).  While the MMAs of step i run
// into one accumulator, the threads fold step i-1's accumulator into the
// running sum, so each FP32 MMA accumulation spans one step (6 x 128
// K-values) and the sum over steps is compensated.  The CTA writes its FP64
// partial (sum - compensation) once at the end.
constexpr int kDB = 64;             // shifts served by one T buffer
constexpr int kRT = 193;            // T rows (>= kDB + 127; odd multiple of 16 B keeps cp.async conflict-free)
// Tile shape for N columns p2 per face and K chunks of N q2 values (N = 64,
// 96, 128: narrow faces pad less).
template <int N>
struct TcShape {
  static constexpr int kHalfN = N;                  // columns p2 per face
  static constexpr int kFullN = 2 * N;              // both faces (partial row)
  static constexpr int kKC = N;                     // K (q2) per chunk
  static constexpr int kKB = kKC / 8;               // K blocks per chunk
  static constexpr int kZN = N + kKC - 8;           // Z entries per split: n' + 8 floor(k/8) <= N - 1 + kKC - 8
  static constexpr int kWUsed = kZN + 7;            // window values used
  static constexpr int kWL = kWUsed + 1;
  static constexpr size_t kTSplit = (size_t)kKB * kRT * 16;  // bytes of one split of T
  static constexpr size_t kZS = (size_t)kZN * 16;            // bytes of one split of Z
  static constexpr size_t kSmemT = 3 * kTSplit;
  static constexpr size_t kSmemZ = 2 * 3 * kZS;              // [buf][split]
  static constexpr size_t kSmemW = (size_t)3 * kWL * 2;      // [split][kWL] bf16
  static constexpr size_t kSmem = kSmemT + kSmemZ + kSmemW;
  // kind::f16 instruction descriptor: F32 accumulate, BF16 A and B, both
  // K-major, M = 128, N.
  static constexpr uint32_t kIdesc =
      (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(kTcM >> 4) << 24);
  static_assert(N % 16 == 0 && N >= 64 && N <= 128, "MMA shape with M = 128");
  static_assert(kWUsed <= 2 * 128, "window within the prefetch");
};
constexpr uint32_t kColAcc = 0, kColSum = 256, kColComp = 384;
constexpr int kPrefetch = (2 * 128 + kTcThreads - 1) / kTcThreads;  // D values per thread per step (window <= 256)

__device__ inline void tmem_ld16(uint32_t addr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(addr));
}
__device__ inline void tmem_st16(uint32_t addr, const uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16};" ::"r"(
          addr),
      "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]), "r"(r[8]), "r"(r[9]),
      "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]), "r"(r[15])
      : "memory");
}

template <int N>
__global__ void __launch_bounds__(kTcThreads, 1)
    bcpot_tc_kernel(KParams P, TcAxis X, const __nv_bfloat16* __restrict__ Cs, const double* __restrict__ D,
                    double* partial, int* err) {
  using Sh = TcShape<N>;
  constexpr int kTcHalfN = Sh::kHalfN, kTcN = Sh::kFullN, kTcKC = Sh::kKC, kKB = Sh::kKB, kZN = Sh::kZN,
                kWUsed = Sh::kWUsed, kWL = Sh::kWL;
  constexpr size_t kTSplit = Sh::kTSplit, kZS = Sh::kZS, kSmemT = Sh::kSmemT, kSmemZ = Sh::kSmemZ;
  constexpr uint32_t kIdescFace = Sh::kIdesc;
  extern __shared__ __align__(1024) unsigned char smem[];
  unsigned char* sT = smem;                   // [3][kKB][kRT][16 B]
  unsigned char* sZ = smem + kSmemT;          // [2][3][kZN][16 B]
  __nv_bfloat16* sWin = reinterpret_cast<__nv_bfloat16*>(smem + kSmemT + kSmemZ);  // [3][kWL]
  __shared__ __align__(8) unsigned long long mbar[2];
  __shared__ uint32_t tmem_base;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int quad = warp & 3;                        // TMEM lane quadrant of this warp
  const int c0 = (warp >> 2) * (N / 2), c1 = c0 + N / 2;  // this warpgroup's accumulator columns

  // CTA -> (tile, face, split)
  const int split = blockIdx.x % X.splits;
  const int tf = blockIdx.x / X.splits;
  const int f = tf % 2, tile = tf / 2;
  const int mt = tile / X.ntiles, nt = tile % X.ntiles;
  const int m0 = mt * kTcM, n0 = nt * kTcHalfN;
  const int rows_hi = (m0 + kTcM < X.n1) ? m0 + kTcM : X.n1;
  const int dlo = 1 - rows_hi, dhi = X.n1 - m0 - 1;
  const int nd = dhi - dlo + 1;
  const long long npairs = (long long)X.nn * nd;
  const long long pbeg = npairs * split / X.splits, pend = npairs * (split + 1) / X.splits;
  const int nchunks = X.n2pad / kTcKC;
  const long long per = (long long)X.nn * X.n1 * X.n2pad;  // elements of one split of Cs
  // partial block of (tile, split): [128 rows][256 columns], this face's half
  double* part = partial + ((long long)tile * X.splits + split) * kTcM * kTcN + f * kTcHalfN;

  const uint32_t mb0 = (uint32_t)__cvta_generic_to_shared(&mbar[0]);
  const uint32_t mb1 = (uint32_t)__cvta_generic_to_shared(&mbar[1]);
  if (warp == 0) {
    uint32_t dst = (uint32_t)__cvta_generic_to_shared(&tmem_base);
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dst), "r"(512)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mb0) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mb1) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_base;
  const uint32_t lanebase = tmem + ((uint32_t)(32 * quad) << 16);  // this warp's 32 TMEM lanes
  uint32_t phase[2] = {0, 0};
  bool pending[2] = {false, false};  // MMAs committed on mbar[b], not yet waited for
  bool unfolded[2] = {false, false};  // accumulator b holds a step not yet folded
  bool ok = true;

  // running sum and compensation start at zero
  {
    uint32_t z[16];
#pragma unroll
    for (int j = 0; j < 16; ++j) z[j] = 0u;
    for (int col = c0; col < c1; col += 16) {
      tmem_st16(lanebase + kColSum + col, z);
      tmem_st16(lanebase + kColComp + col, z);
    }
    asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
  }

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
  // Kahan: y = a - c; t = s + y; c = (t - s) - y; s = t
  auto fold = [&](int b) {
    if (!unfolded[b]) return;
    for (int col = c0; col < c1; col += 16) {
      uint32_t a[16], sm[16], cp[16];
      tmem_ld16(lanebase + kColAcc + (uint32_t)(b * kTcHalfN + col), a);
      tmem_ld16(lanebase + kColSum + col, sm);
      tmem_ld16(lanebase + kColComp + col, cp);
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        const float y = __fsub_rn(__uint_as_float(a[j]), __uint_as_float(cp[j]));
        const float t = __fadd_rn(__uint_as_float(sm[j]), y);
        cp[j] = __float_as_uint(__fsub_rn(__fsub_rn(t, __uint_as_float(sm[j])), y));
        sm[j] = __float_as_uint(t);
      }
      tmem_st16(lanebase + kColSum + col, sm);
      tmem_st16(lanebase + kColComp + col, cp);
    }
    asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    unfolded[b] = false;
  };

  // D values of one step into registers: item e = tid + 128 m -> window index e
  double pre[kPrefetch];
  auto prefetch = [&](int q, int d, int kc) {
    const int o_min = kc * kTcKC - n0 - (kTcHalfN - 1);
#pragma unroll
    for (int m = 0; m < kPrefetch; ++m) {
      const int j = tid + kTcThreads * m;
      double v = 0.0;
      if (j < kWUsed) {
        const int o2 = o_min + j;
        if (o2 >= -(X.n2 - 1) && o2 <= X.n2 - 1) v = __ldg(D + d_index(P, X, f, q, d, o2));
      }
      pre[m] = v;
    }
  };

  int step = 0;
  if (pbeg < pend) prefetch(int(pbeg / nd) + 1, dlo + int(pbeg % nd), 0);
  for (int kc = 0; kc < nchunks && ok; ++kc) {
    const int k0 = kc * kTcKC;
    int Tq = -1, TdA = 0;
    for (long long pr = pbeg; pr < pend && ok; ++pr) {
      const int q = int(pr / nd) + 1;
      const int d = dlo + int(pr % nd);
      if (q != Tq || d >= TdA + kDB) {
        // every MMA that reads T is done before T is rewritten
        if (!__syncthreads_and(drain() ? 1 : 0)) { ok = false; break; }
        Tq = q;
        TdA = d;
        const int rho0 = m0 + TdA;
        const uint32_t tbase = (uint32_t)__cvta_generic_to_shared(sT);
        for (int e = tid; e < 3 * kRT * kKB; e += kTcThreads) {
          const int kb = e % kKB, rest = e / kKB;
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
      // the MMAs of step - 2 (accumulator b, Z[b]) are done: fold them
      if (!__syncthreads_and(wait_buf(b) ? 1 : 0)) { ok = false; break; }
      fold(b);
      // window of this step from the prefetched D values
#pragma unroll
      for (int m = 0; m < kPrefetch; ++m) {
        const int j = tid + kTcThreads * m;
        if (j < kWUsed) {
          __nv_bfloat16 a0, a1, a2;
          split3((float)pre[m], a0, a1, a2);
          sWin[0 * kWL + j] = a0;
          sWin[1 * kWL + j] = a1;
          sWin[2 * kWL + j] = a2;
        }
      }
      if (tid < 3) sWin[tid * kWL + kWUsed] = __float2bfloat16_rn(0.0f);
      // D values of the next step: issued now, so that their latency overlaps
      // the Z build and the MMA issue of this step
      {
        long long npr = pr + 1;
        int nkc = kc;
        if (npr >= pend) {
          npr = pbeg;
          ++nkc;
        }
        if (nkc < nchunks) prefetch(int(npr / nd) + 1, dlo + int(npr % nd), nkc);
      }
      __syncthreads();
      // Z[b][s][u] = w_s[u .. u+7]
      unsigned char* zb = sZ + (size_t)b * 3 * kZS;
      for (int e = tid; e < 3 * kZN; e += kTcThreads) {
        const int sp = e / kZN, u = e % kZN;
        const __nv_bfloat16* w = sWin + sp * kWL + u;
        __align__(16) __nv_bfloat16 v[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) v[j] = w[j];
        *reinterpret_cast<uint4*>(zb + (size_t)sp * kZS + (size_t)u * 16) = *reinterpret_cast<const uint4*>(v);
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      __syncthreads();
      if (tid == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t tb = (uint32_t)__cvta_generic_to_shared(sT) + (uint32_t)(d - TdA) * 16u;
        const uint32_t zs = (uint32_t)__cvta_generic_to_shared(zb);
        const uint32_t acc_cols = tmem + kColAcc + (uint32_t)(b * kTcHalfN);
        // the five correction products first, the leading product x1 y1
        // last: an FP32 MMA accumulation loses up to an ulp of the running
        // sum per update, so the 5 (K / 16) updates of the small products
        // happen while the sum is small, and only the K / 16 updates of the
        // leading product see it at full size
        const int pa[6] = {2, 1, 0, 1, 0, 0}, pb[6] = {0, 1, 2, 0, 1, 0};
        // descriptors of this step's first A and B blocks; every other block
        // is a multiple of 16 bytes further in, which adds to the start
        // address field (address / 16, below 2^14 for any shared-memory
        // address) without carrying into the offset fields
        const uint64_t adesc0 = smem_desc(tb, kRT * 16, 128);
        const uint64_t bdesc0 = smem_desc(zs, 128, 128);
#pragma unroll
        for (int t = 0; t < 6; ++t) {
#pragma unroll
          for (int ks = 0; ks < kTcKC / 16; ++ks) {
            const uint64_t adesc = adesc0 + (uint64_t)((pa[t] * kTSplit + (size_t)(2 * ks) * kRT * 16) >> 4);
            const uint64_t bdesc = bdesc0 + (uint64_t)((pb[t] * kZS + (size_t)ks * 256) >> 4);
            const uint32_t acc = (ks == 0 && t == 0) ? 0u : 1u;
            asm volatile(
                "{\n\t.reg .pred p;\n\t"
                "setp.ne.b32 p, %4, 0;\n\t"
                "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
                ::"r"(acc_cols), "l"(adesc), "l"(bdesc), "r"(kIdescFace), "r"(acc)
                : "memory");
          }
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(b ? mb1 : mb0)
                     : "memory");
      }
      pending[b] = true;
      unfolded[b] = true;
      ++step;
    }
  }
  if (ok && !__syncthreads_and(drain() ? 1 : 0)) ok = false;
  if (ok) {
    fold(step & 1);        // the older of the two outstanding steps first
    fold((step + 1) & 1);
    // partial = sum - compensation, this thread's row
    double* row = part + (long long)(32 * quad + lane) * kTcN;
    for (int col = c0; col < c1; col += 16) {
      uint32_t sm[16], cp[16];
      tmem_ld16(lanebase + kColSum + col, sm);
      tmem_ld16(lanebase + kColComp + col, cp);
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
      for (int j = 0; j < 16; ++j)
        row[kTcHalfN - 1 - (col + j)] = (double)__uint_as_float(sm[j]) - (double)__uint_as_float(cp[j]);
    }
  } else {
    if (tid == 0) atomicCAS(err, 0, int(kDevTimeout));
    drain();  // bounded: let outstanding MMAs finish before TMEM is released
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512) : "memory");
  }
}

// U on both faces of the axis = (sum over splits of the partial tiles) / (4 pi eps0).
__global__ void bcpot_reduce_kernel(KParams P, TcAxis X, const double* partial, double* U) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int kTcHalfN = X.N, kTcN = 2 * X.N;
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
  X.N = X.n2 <= 64 ? 64 : (X.n2 <= 96 ? 96 : 128);
  X.n2pad = (X.n2 + X.N - 1) / X.N * X.N;
  X.mtiles = (X.n1 + kTcM - 1) / kTcM;
  X.ntiles = (X.n2 + X.N - 1) / X.N;
  int tiles = X.mtiles * X.ntiles * 2;  // one CTA per face of a tile
  X.splits = sms / tiles;
  if (X.splits < 1) X.splits = 1;
  return X;
}

}  // namespace

size_t bcpot_tc_smem_bytes(const KParams& P) {
  size_t m = 0;
  for (int axis = 0; axis < 3; ++axis) {
    const int N = tc_axis(P, axis, 148).N;
    const size_t b = N == 64 ? TcShape<64>::kSmem : (N == 96 ? TcShape<96>::kSmem : TcShape<128>::kSmem);
    m = b > m ? b : m;
  }
  return m;
}

void bcpot_tc_scratch(const KParams& P, long long* cs_elems, long long* partial_elems) {
  long long cs = 0, pe = 0;
  for (int axis = 0; axis < 3; ++axis) {
    TcAxis X = tc_axis(P, axis, 148);
    long long c = 3LL * X.nn * X.n1 * X.n2pad;
    long long p = (long long)X.mtiles * X.ntiles * X.splits * kTcM * (2LL * X.N);
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
  static bool attr = false;
  if (!attr) {
    e = cudaFuncSetAttribute(bcpot_tc_kernel<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TcShape<64>::kSmem);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(bcpot_tc_kernel<96>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)TcShape<96>::kSmem);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(bcpot_tc_kernel<128>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)TcShape<128>::kSmem);
    if (e != cudaSuccess) return e;
    attr = true;
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
    const unsigned grid = (unsigned)(X.mtiles * X.ntiles * 2 * X.splits);
    if (X.N == 64)
      bcpot_tc_kernel<64><<<grid, kTcThreads, TcShape<64>::kSmem, st>>>(P, X, Cs, D, partial, err);
    else if (X.N == 96)
      bcpot_tc_kernel<96><<<grid, kTcThreads, TcShape<96>::kSmem, st>>>(P, X, Cs, D, partial, err);
    else
      bcpot_tc_kernel<128><<<grid, kTcThreads, TcShape<128>::kSmem, st>>>(P, X, Cs, D, partial, err);
    long long outs = (long long)X.mtiles * X.ntiles * kTcM * (2LL * X.N);
    note_launch();
    bcpot_reduce_kernel<<<(unsigned)((outs + 255) / 256), 256, 0, st>>>(P, X, partial, U);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

}  // namespace picard
