// jacobi_resident.cu -- FP32 Jacobi sweeps of the increment with the state
// resident on chip for a whole batch of sweeps (CalcEpotential.f90:50-56 on
// the increment w of the F32_REFINE solver; open boundaries).
//
// One cooperative launch runs m consecutive sweeps.  The interior is cut into
// blocks of 32 (x) x BY (y) x NZ (z) nodes, one CTA each, all co-resident.
// Thread (tx, ty) keeps its NZ-node column of w in registers and the CTA keeps
// r (constant between anchors) in shared memory, so a sweep reads and writes
// no array in global memory: x neighbours come from warp shuffles, y
// neighbours through shared-memory plane groups, z neighbours from the
// thread's own registers.  Across CTA boundaries only the faces move: after a
// sweep each CTA writes its six faces of w to an exchange buffer (double
// buffered by sweep parity), every CTA meets at a grid barrier, and the next
// sweep stages its neighbours' faces as halos.  Ghost nodes of the open
// boundary (and halos beyond the domain) are zero.
//
// Each sweep writes the same per-tile partial sums of squared residuals as
// the TMA sweep kernel -- tiles of 32 x 8 x ZC nodes, the same per-thread
// accumulation in z order, the same warp tree and the same in-order sum over
// the tile's eight warps -- and every node update uses jacobi_res_f32 /
// jacobi_next_f32, so the two kernels agree bit for bit and the host's batch
// logic (stop test, replay from the anchor) is shared.
//
// The grid barrier is a counter in global memory (zeroed before the launch)
// that each CTA's elected thread increments and then polls with acquire
// loads.  The poll is bounded: past the limit the CTA records kDevTimeout in
// *err and returns; the other CTAs then give up at their own next barrier.
// The wait test (PICARD_OPT_WAIT_TEST) makes every CTA's first wait run out
// on purpose, with a short limit, so that the timeout path can be tested.
// All CTAs are co-resident by construction of the cooperative launch.
#include <cuda_runtime.h>

#include <algorithm>

#include "common.cuh"
#include "grid.cuh"
#include "stencil.cuh"

namespace picard {

namespace {

constexpr int kResG = 4;                 // planes per shared-memory exchange group
constexpr long long kBarSpin = 1LL << 22;
// Poll limit of the wait test (PICARD_OPT_WAIT_TEST): the barrier then waits
// for one arrival more than the grid makes, so every CTA gives up after this
// many polls and returns.
constexpr long long kBarSpinTest = 1LL << 14;

template <int BY, int NZ, int ZC>
struct ResLayout {
  static constexpr int kThreads = 32 * BY;
  static constexpr int kTilesZ = NZ / ZC;          // z tiles per CTA
  static constexpr int kR = NZ * BY * 32;          // r of the CTA's nodes [z][ty][tx]
  static constexpr int kPB = 2 * kResG * (BY + 2) * 32;  // plane groups [2][G][BY+2][32]
  static constexpr int kXH = 2 * BY * NZ;          // x halos [lo/hi][ty][z]
  static constexpr int kYH = 2 * NZ * 32;          // y halos [lo/hi][z][tx]
  static constexpr int kRed = BY * kTilesZ;        // doubles: warp sums [ty][z tile]
  static constexpr size_t kBytes = sizeof(float) * (kR + kPB + kXH + kYH) + sizeof(double) * (size_t)kRed;
  // exchange faces of one CTA (floats): x [lo/hi][ty][z], y [lo/hi][z][tx], z [lo/hi][ty][tx]
  static constexpr int kFX = 2 * BY * NZ, kFY = 2 * NZ * 32, kFZ = 2 * BY * 32;
  static constexpr int kFace = kFX + kFY + kFZ;
  static_assert(NZ % kResG == 0 && NZ % ZC == 0 && BY % 8 == 0, "block shape");
  static_assert((kR + kPB + kXH + kYH) % 2 == 0, "double alignment of the reduction scratch");
};

struct ResArgs {
  Stencil S;
  JacobiCoefF J;
  const float* r;      // padded scaled residual of the live anchor
  const float* win;    // padded increment before the first sweep (unused when w_zero)
  float* wout;         // padded increment after the last sweep
  float* faces;        // [2][nctas][kFace]
  unsigned int* bar;   // grid barrier counter, zero at launch
  double* partial;     // [m][ntiles]
  int* err;
  unsigned int bar_extra;  // arrivals the barrier waits for beyond the grid's (0; 1 only in the wait test)
  long long spin;          // poll limit of one barrier wait
  int m, w_zero;
  int gx, gy, gz, ntiles;  // tile grid of the TMA sweep kernel
  int cgx, cgy, cgz;       // CTA grid
};

__device__ __forceinline__ unsigned int ld_acquire(const unsigned int* p) {
  unsigned int v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Every CTA of the grid arrives; returns false (uniformly over the CTA) when
// the wait gave up.
__device__ bool grid_barrier(unsigned int* bar, unsigned int target, long long spin, int* err, int* s_abort) {
  __syncthreads();
  if (threadIdx.x == 0 && threadIdx.y == 0) {
    __threadfence();
    atomicAdd(bar, 1u);
    bool ok = false;
    for (long long it = 0; it < spin; ++it) {
      if (ld_acquire(bar) >= target) {
        ok = true;
        break;
      }
      __nanosleep(32);
    }
    __threadfence();
    if (!ok) {
      *s_abort = 1;
      atomicCAS(err, 0, int(kDevTimeout));
    }
  }
  __syncthreads();
  return *s_abort == 0;
}

// w of the padded array at node (i, j, k), zero outside the ghost layer.
__device__ __forceinline__ float w_at(const Stencil& S, const float* w, int i, int j, int k) {
  if (i < 0 || i > S.nx + 1 || j < 0 || j > S.ny + 1 || k < 0 || k > S.nz + 1) return 0.0f;
  return __ldcg(w + fidx(S, i, j, k));
}

// Stages the halos of sweep s+1 (s >= 0) from the faces the neighbouring
// CTAs wrote after sweep s; returns this thread's z halos in zlo, zhi.
template <int BY, int NZ, int ZC>
__device__ __forceinline__ void stage_from_faces(const ResArgs& a, int s, float* xh, float* yh, float& zlo,
                                                 float& zhi) {
  using L = ResLayout<BY, NZ, ZC>;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = tx + 32 * ty;
  const int cta = blockIdx.x;
  const int cx = cta % a.cgx, cy = (cta / a.cgx) % a.cgy, cz = cta / (a.cgx * a.cgy);
  const float* F = a.faces + (size_t)((s + 1) & 1) * gridDim.x * L::kFace;
  const int plane = a.cgx * a.cgy;
  const float* fxlo = cx > 0 ? F + (size_t)(cta - 1) * L::kFace + BY * NZ : nullptr;  // its hi x face
  const float* fxhi = cx + 1 < a.cgx ? F + (size_t)(cta + 1) * L::kFace : nullptr;    // its lo x face
  const float* fylo = cy > 0 ? F + (size_t)(cta - a.cgx) * L::kFace + L::kFX + NZ * 32 : nullptr;
  const float* fyhi = cy + 1 < a.cgy ? F + (size_t)(cta + a.cgx) * L::kFace + L::kFX : nullptr;
  for (int q = tid; q < BY * NZ; q += L::kThreads) {
    xh[q] = fxlo ? __ldcg(fxlo + q) : 0.0f;
    xh[BY * NZ + q] = fxhi ? __ldcg(fxhi + q) : 0.0f;
  }
  for (int q = tid; q < NZ * 32; q += L::kThreads) {
    yh[q] = fylo ? __ldcg(fylo + q) : 0.0f;
    yh[NZ * 32 + q] = fyhi ? __ldcg(fyhi + q) : 0.0f;
  }
  zlo = cz > 0 ? __ldcg(F + (size_t)(cta - plane) * L::kFace + L::kFX + L::kFY + BY * 32 + ty * 32 + tx) : 0.0f;
  zhi = cz + 1 < a.cgz ? __ldcg(F + (size_t)(cta + plane) * L::kFace + L::kFX + L::kFY + ty * 32 + tx) : 0.0f;
}

template <int BY, int NZ, int ZC>
__global__ void __launch_bounds__(32 * BY, 1) jacobi_resident_kernel(ResArgs a) {
  using L = ResLayout<BY, NZ, ZC>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float* rs = reinterpret_cast<float*>(smem_raw);  // [NZ][BY][32]
  float* pb = rs + L::kR;                           // [2][G][BY+2][32]
  float* xh = pb + L::kPB;                          // [2][BY][NZ]
  float* yh = xh + L::kXH;                          // [2][NZ][32]
  double* red = reinterpret_cast<double*>(yh + L::kYH);
  __shared__ int s_abort;

  const Stencil& S = a.S;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = tx + 32 * ty;
  // this thread's column: nodes (i, j, k0 .. k0 + kact - 1) are interior
  int kact;
  float w[NZ];
  float zlo = 0.0f, zhi = 0.0f;
  {
    const int cta = blockIdx.x;
    const int cx = cta % a.cgx, cy = (cta / a.cgx) % a.cgy, cz = cta / (a.cgx * a.cgy);
    const int i = 32 * cx + tx + 1, j = BY * cy + ty + 1, k0 = NZ * cz + 1;
    kact = (i <= S.nx && j <= S.ny) ? min(NZ, S.nz - k0 + 1) : 0;
    if (tid == 0) s_abort = 0;
#pragma unroll
    for (int z = 0; z < NZ; ++z) {
      float rv = 0.0f, wv = 0.0f;
      if (z < kact) {
        const long long c = fidx(S, i, j, k0 + z);
        rv = __ldg(a.r + c);
        if (!a.w_zero) wv = __ldcg(a.win + c);
      }
      rs[(z * BY + ty) * 32 + tx] = rv;
      w[z] = wv;
    }
    // halos of the first sweep: the global increment itself (zero when w_zero)
    if (!a.w_zero) {
      for (int q = tid; q < BY * NZ; q += L::kThreads) {
        const int y = q / NZ, z = q % NZ;
        xh[q] = w_at(S, a.win, 32 * cx, BY * cy + y + 1, k0 + z);
        xh[BY * NZ + q] = w_at(S, a.win, 32 * cx + 33, BY * cy + y + 1, k0 + z);
      }
      for (int q = tid; q < NZ * 32; q += L::kThreads) {
        const int z = q / 32, x = q % 32;
        yh[q] = w_at(S, a.win, 32 * cx + x + 1, BY * cy, k0 + z);
        yh[NZ * 32 + q] = w_at(S, a.win, 32 * cx + x + 1, BY * cy + BY + 1, k0 + z);
      }
      zlo = w_at(S, a.win, i, j, k0 - 1);
      zhi = w_at(S, a.win, i, j, k0 + NZ);
    } else {
      for (int q = tid; q < 2 * BY * NZ; q += L::kThreads) xh[q] = 0.0f;
      for (int q = tid; q < 2 * NZ * 32; q += L::kThreads) yh[q] = 0.0f;
    }
  }

  for (int s = 0; s < a.m; ++s) {
    // ---- plane groups through shared memory, the update in registers
    auto stage = [&](int g) {
      float* P = pb + (g & 1) * kResG * (BY + 2) * 32;
#pragma unroll
      for (int zz = 0; zz < kResG; ++zz) {
        const int z = g * kResG + zz;
        float* Q = P + zz * (BY + 2) * 32;
        Q[(ty + 1) * 32 + tx] = w[z];
        if (ty == 0) Q[tx] = yh[z * 32 + tx];
        if (ty == BY - 1) Q[(BY + 1) * 32 + tx] = yh[NZ * 32 + z * 32 + tx];
      }
    };
    __syncthreads();  // halos staged; the previous sweep is done with pb and red
    stage(0);
    __syncthreads();
    float r2 = 0.0f;
    float wm = zlo;
#pragma unroll
    for (int g = 0; g < NZ / kResG; ++g) {
      if (g + 1 < NZ / kResG) stage(g + 1);
      const float* P = pb + (g & 1) * kResG * (BY + 2) * 32;
#pragma unroll
      for (int zz = 0; zz < kResG; ++zz) {
        const int z = g * kResG + zz;
        const float wc = w[z];
        const float wp = z + 1 < NZ ? w[z + 1] : zhi;
        float xm = __shfl_up_sync(0xffffffffu, wc, 1);
        float xp = __shfl_down_sync(0xffffffffu, wc, 1);
        if (tx == 0) xm = xh[ty * NZ + z];
        if (tx == 31) xp = xh[BY * NZ + ty * NZ + z];
        const float* Q = P + zz * (BY + 2) * 32;
        const float res = jacobi_res_f32(a.J, wc, xm, xp, Q[ty * 32 + tx], Q[(ty + 2) * 32 + tx], wm, wp,
                                         rs[(z * BY + ty) * 32 + tx]);
        if (z < kact) {
          r2 = acc_r2_f32(r2, res);
          w[z] = jacobi_next_f32(a.J, wc, res);
        }
        wm = wc;
        if ((z + 1) % ZC == 0) {
          // the tile's z range ends here: its warp sum, as the TMA kernel forms it
          double v = (double)r2;
          for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
          if (tx == 0) red[ty * L::kTilesZ + z / ZC] = v;
          r2 = 0.0f;
        }
      }
      __syncthreads();
    }

    // ---- per-tile partials: the in-order sum over each tile's eight warps
    {
      const int cta = blockIdx.x;
      const int cx = cta % a.cgx, cy = (cta / a.cgx) % a.cgy, cz = cta / (a.cgx * a.cgy);
      if (tid < (BY / 8) * L::kTilesZ) {
        const int byl = tid / L::kTilesZ, bzl = tid % L::kTilesZ;
        const int by = cy * (BY / 8) + byl, bz = cz * L::kTilesZ + bzl;
        if (by < a.gy && bz < a.gz) {
          double sum = 0.0;
          for (int q = 0; q < 8; ++q) sum += red[(byl * 8 + q) * L::kTilesZ + bzl];
          a.partial[(size_t)s * a.ntiles + cx + (size_t)a.gx * (by + (size_t)a.gy * bz)] = sum;
        }
      }
    }

    // ---- faces of the new iterate for the next sweep's halos
    if (s + 1 < a.m) {
      float* F = a.faces + ((size_t)((s + 1) & 1) * gridDim.x + blockIdx.x) * L::kFace;
      if (tx == 0 || tx == 31) {
        float* X = F + (tx == 0 ? 0 : BY * NZ) + ty * NZ;
#pragma unroll
        for (int z = 0; z < NZ; ++z) __stcg(X + z, w[z]);
      }
      if (ty == 0 || ty == BY - 1) {
        float* Y = F + L::kFX + (ty == 0 ? 0 : NZ * 32) + tx;
#pragma unroll
        for (int z = 0; z < NZ; ++z) __stcg(Y + z * 32, w[z]);
      }
      __stcg(F + L::kFX + L::kFY + ty * 32 + tx, w[0]);
      __stcg(F + L::kFX + L::kFY + BY * 32 + ty * 32 + tx, w[NZ - 1]);
    }

    // ---- every CTA finished this sweep (after the last one too: the final
    // store below may overwrite the array the first sweep read halos from)
    if (!grid_barrier(a.bar, (unsigned int)(s + 1) * gridDim.x + a.bar_extra, a.spin, a.err, &s_abort)) return;
    if (s + 1 < a.m) stage_from_faces<BY, NZ, ZC>(a, s, xh, yh, zlo, zhi);
  }

  {
    const int cta = blockIdx.x;
    const int cx = cta % a.cgx, cy = (cta / a.cgx) % a.cgy, cz = cta / (a.cgx * a.cgy);
    const int i = 32 * cx + tx + 1, j = BY * cy + ty + 1, k0 = NZ * cz + 1;
#pragma unroll
    for (int z = 0; z < NZ; ++z)
      if (z < kact) __stcg(a.wout + fidx(S, i, j, k0 + z), w[z]);
  }
}

struct ResKernel {
  const void* fn = nullptr;
  size_t smem = 0;
};

template <int BY, int NZ, int ZC>
ResKernel res_kernel() {
  return {reinterpret_cast<const void*>(&jacobi_resident_kernel<BY, NZ, ZC>), ResLayout<BY, NZ, ZC>::kBytes};
}

// The CTA shapes the resident sweep offers, smallest first.
struct ResShape {
  int by, nz;
};
constexpr ResShape kResShapes[] = {{8, 8}, {8, 16}, {16, 16}, {16, 32}, {32, 32}};

ResKernel pick_kernel(int by, int nz, int zc) {
#define PICARD_RES_CASE(BY_, NZ_) \
  if (by == BY_ && nz == NZ_) return zc == 8 ? res_kernel<BY_, NZ_, 8>() : res_kernel<BY_, NZ_, 4>();
  PICARD_RES_CASE(8, 8)
  PICARD_RES_CASE(8, 16)
  PICARD_RES_CASE(16, 16)
  PICARD_RES_CASE(16, 32)
  PICARD_RES_CASE(32, 32)
#undef PICARD_RES_CASE
  return {};
}

int face_floats(int by, int nz) { return 2 * by * nz + 2 * nz * 32 + 2 * by * 32; }

}  // namespace

int resident_plan(const KParams& P, JacobiGeom& G, int shape_index) {
  G.res = 0;
  if (!G.tma) return 0;
  static_assert(sizeof(kResShapes) / sizeof(kResShapes[0]) == kResidentShapes, "shape table");
  if (shape_index < 0 || shape_index >= kResidentShapes) return 0;
  const ResShape sh = kResShapes[shape_index];
  int dev = 0, sms = 0, coop = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
  if (cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev) != cudaSuccess || !coop) return 0;
  const ResKernel k = pick_kernel(sh.by, sh.nz, G.zc);
  if (!k.fn) return 0;
  if (cudaFuncSetAttribute(k.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)k.smem) != cudaSuccess) return 0;
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k.fn, 32 * sh.by, k.smem) != cudaSuccess || per_sm < 1)
    return 0;
  const int cgx = (P.nx + 31) / 32, cgy = (P.ny + sh.by - 1) / sh.by, cgz = (P.nz + sh.nz - 1) / sh.nz;
  const long long nctas = (long long)cgx * cgy * cgz;
  if (nctas > (long long)per_sm * sms) return 0;
  G.res = 1;
  G.res_by = sh.by;
  G.res_nz = sh.nz;
  G.res_cgx = cgx;
  G.res_cgy = cgy;
  G.res_cgz = cgz;
  G.res_ctas = int(nctas);
  return 1;
}

long long resident_face_floats(const JacobiGeom& G) {
  return G.res ? 2LL * G.res_ctas * face_floats(G.res_by, G.res_nz) : 0;
}

cudaError_t launch_sweeps_resident(const KParams& P, const JacobiGeom& G, const float* r, const float* win,
                                   float* wout, float* faces, unsigned int* bar, double* partial, int m, int w_zero,
                                   int* err, cudaStream_t st, int wait_test) {
  if (!G.res || m < 1) return cudaErrorInvalidValue;
  const ResKernel k = pick_kernel(G.res_by, G.res_nz, G.zc);
  if (!k.fn) return cudaErrorInvalidValue;
  cudaError_t e = cudaMemsetAsync(bar, 0, sizeof(unsigned int), st);
  if (e != cudaSuccess) return e;
  ResArgs a;
  a.S = make_stencil(P);
  a.J = jacobi_coef_f(P);
  a.r = r;
  a.win = win;
  a.wout = wout;
  a.faces = faces;
  a.bar = bar;
  a.partial = partial;
  a.err = err;
  a.bar_extra = wait_test ? 1u : 0u;
  a.spin = wait_test ? kBarSpinTest : kBarSpin;
  a.m = m;
  a.w_zero = w_zero;
  a.gx = (int)G.grid.x;
  a.gy = (int)G.grid.y;
  a.gz = (int)G.grid.z;
  a.ntiles = G.nblocks;
  a.cgx = G.res_cgx;
  a.cgy = G.res_cgy;
  a.cgz = G.res_cgz;
  void* args[] = {&a};
  note_launch();
  return cudaLaunchCooperativeKernel(k.fn, dim3(G.res_ctas), dim3(32, G.res_by), args, k.smem, st);
}

}  // namespace picard
