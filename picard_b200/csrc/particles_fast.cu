// particles_fast.cu -- CELL32 particle kernels (the performance layout) and
// the integer scan used by compaction and production.
//
// A CELL32 particle is its CIC base node (i, j, k), packed in one uint32, the
// in-cell fractions f = (x - Lx_min)/dx + 1/2 - i in [0, 1) as 32-bit fixed
// point (f 2^32), and the velocity as FP32: 28 bytes plus one species byte.
// Node i sits at x = Lx_min + (i - 1/2) dx, so the CIC weights are (1 - f, f)
// directly and the position advance is one integer add per axis.
#include <cuda_runtime.h>

#include <climits>

#include <cmath>

#include "common.cuh"
#include "kernels.cuh"
#include "outflow.cuh"

namespace picard {

namespace {

constexpr int kThreads = 256;

inline int persistent_grid(long long n) {
  long long b = (n + kThreads - 1) / kThreads;
  if (b > 148LL * 16) b = 148LL * 16;
  return b < 1 ? 1 : int(b);
}

// ------------------------------------------------------------------ scan

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

__device__ inline int block_scan_excl(int v, int& total) {
  __shared__ int warp_sums[32];
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_sums[warp] = x;
  __syncthreads();
  if (warp == 0) {
    int w = (lane < int(blockDim.x >> 5)) ? warp_sums[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    warp_sums[lane] = w;
  }
  __syncthreads();
  int prefix = (warp > 0 ? warp_sums[warp - 1] : 0) + x - v;
  total = warp_sums[(blockDim.x >> 5) - 1];
  __syncthreads();
  return prefix;
}

__global__ void scan_tiles_kernel(const int* in, int* out, int n, int* tile_sums) {
  long long base = (long long)blockIdx.x * kScanTile + (long long)threadIdx.x * kScanItems;
  int v[kScanItems];
  int s = 0;
#pragma unroll
  for (int q = 0; q < kScanItems; ++q) {
    long long i = base + q;
    v[q] = i < n ? in[i] : 0;
    s += v[q];
  }
  int total;
  int run = block_scan_excl(s, total);
#pragma unroll
  for (int q = 0; q < kScanItems; ++q) {
    long long i = base + q;
    if (i < n) out[i] = run;
    run += v[q];
  }
  if (threadIdx.x == 0) tile_sums[blockIdx.x] = total;
}

__global__ void scan_add_kernel(int* out, int n, const int* tile_offsets) {
  long long base = (long long)blockIdx.x * kScanTile;
  int add = tile_offsets[blockIdx.x];
  for (int q = threadIdx.x; q < kScanTile; q += blockDim.x) {
    long long i = base + q;
    if (i < n) out[i] += add;
  }
}

// ------------------------------------------------------------ CELL32 ops

struct C32 {
  int i, j, k;
  uint32_t f[3];  // in-cell offsets, 32-bit fixed point
};

__device__ inline C32 load_pos(const PartC32& a, long long p) {
  C32 r;
  unpack_cell(a.cell[p], r.i, r.j, r.k);
  r.f[0] = a.fx[p];
  r.f[1] = a.fy[p];
  r.f[2] = a.fz[p];
  return r;
}

// The same with streaming (evict-first) loads: for the passes that read every
// particle once, so that the 7.8 GB particle stream does not push the E table
// or the density accumulators out of L2.
__device__ inline C32 load_pos_cs(const PartC32& a, long long p) {
  C32 r;
  unpack_cell(__ldcs(a.cell + p), r.i, r.j, r.k);
  r.f[0] = __ldcs(a.fx + p);
  r.f[1] = __ldcs(a.fy + p);
  r.f[2] = __ldcs(a.fz + p);
  return r;
}

// Move one axis by d cells (FP32, in cell units) in 32-bit fixed point: d is
// scaled to 2^-32 cells (exact when |d| >= 2^-9, else rounded to the nearest
// 2^-32), added to the offset, and the whole cells of the sum move the index.
// Open axes pin far-out particles at the outer guard node (they are outside
// the domain and BCoutflow removes them); periodic axes shift by whole
// periods so the index stays representable.
__device__ inline void move_axis(int& i, uint32_t& f, float d, int n, int open) {
  d = fminf(fmaxf(d, -1073741824.0f), 1073741824.0f);  // |d| <= 2^30 cells (NaN: -2^30)
  const long long t = (long long)f + __float2ll_rn(d * 4294967296.0f);
  f = uint32_t(t);             // t modulo 2^32: the offset in [0, 1)
  i += int(t >> 32);           // floor(t / 2^32): whole cells
  if (open) {
    if (i < -1) i = -1, f = 0u;
    if (i > n + 1) i = n + 1, f = kOffHalf;
  } else if (i < -1) {  // whole periods up to the first index >= -1
    i = int((long long)i + (long long)n * ((-1LL - i + n - 1) / n));
  } else if (i > n + 1) {  // whole periods down to the first index <= n + 1
    i = int((long long)i - (long long)n * (((long long)i - n - 1 + n - 1) / n));
  }
}

// x < min  <=>  i + f < 1/2;  x > max  <=>  i + f > n + 1/2.
__device__ inline bool below(int i, uint32_t f) { return i < 0 || (i == 0 && f < kOffHalf); }
__device__ inline bool above(int i, uint32_t f, int n) { return i > n || (i == n && f > kOffHalf); }

// BCoutflow.f90:28-53 in cell coordinates (true = keep).
__device__ inline bool keep_c32(const KParams& P, const C32& c) {
  if (P.xflow && (below(c.i, c.f[0]) || above(c.i, c.f[0], P.nx))) return false;
  if (P.yflow && (below(c.j, c.f[1]) || above(c.j, c.f[1], P.ny))) return false;
  if (P.zflow && (below(c.k, c.f[2]) || above(c.k, c.f[2], P.nz))) return false;
  return true;
}

// ParticlesTransfer.f90:494-519 in cell coordinates: whole-period shifts.
__device__ inline void wrap_c32(const KParams& P, C32& c) {
  if (below(c.k, c.f[2])) c.k += P.nz;
  if (above(c.k, c.f[2], P.nz)) c.k -= P.nz;
  if (below(c.j, c.f[1])) c.j += P.ny;
  if (above(c.j, c.f[1], P.ny)) c.j -= P.ny;
  if (below(c.i, c.f[0])) c.i += P.nx;
  if (above(c.i, c.f[0], P.nx)) c.i -= P.nx;
}

__device__ __forceinline__ void advance_one(const KParams& P, uint32_t& cell, uint32_t& fx, uint32_t& fy, uint32_t& fz,
                                            float vx, float vy, float vz, float dtdx, float dtdy, float dtdz) {
  int i, j, k;
  unpack_cell(cell, i, j, k);
  move_axis(i, fx, vx * dtdx, P.nx, P.xflow);
  move_axis(j, fy, vy * dtdy, P.ny, P.yflow);
  move_axis(k, fz, vz * dtdz, P.nz, P.zflow);
  cell = pack_cell(i, j, k);
}

// Four particles per thread and pass with 16-byte loads and stores (the
// particle arrays are 256-byte aligned): seven loads of 16 bytes in flight per
// thread instead of seven of 4.  The remainder n % 4 goes one by one.
__global__ void advance_position_c32_kernel(KParams P, PartC32 a, long long n, float dtdx, float dtdy, float dtdz) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  const long long n4 = n >> 2;
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n4; q += stride) {
    uint4 c = reinterpret_cast<const uint4*>(a.cell)[q];
    uint4 x = reinterpret_cast<const uint4*>(a.fx)[q];
    uint4 y = reinterpret_cast<const uint4*>(a.fy)[q];
    uint4 z = reinterpret_cast<const uint4*>(a.fz)[q];
    const float4 u = reinterpret_cast<const float4*>(a.vx)[q];
    const float4 v = reinterpret_cast<const float4*>(a.vy)[q];
    const float4 w = reinterpret_cast<const float4*>(a.vz)[q];
    advance_one(P, c.x, x.x, y.x, z.x, u.x, v.x, w.x, dtdx, dtdy, dtdz);
    advance_one(P, c.y, x.y, y.y, z.y, u.y, v.y, w.y, dtdx, dtdy, dtdz);
    advance_one(P, c.z, x.z, y.z, z.z, u.z, v.z, w.z, dtdx, dtdy, dtdz);
    advance_one(P, c.w, x.w, y.w, z.w, u.w, v.w, w.w, dtdx, dtdy, dtdz);
    reinterpret_cast<uint4*>(a.cell)[q] = c;
    reinterpret_cast<uint4*>(a.fx)[q] = x;
    reinterpret_cast<uint4*>(a.fy)[q] = y;
    reinterpret_cast<uint4*>(a.fz)[q] = z;
  }
  for (long long p = 4 * n4 + (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += stride) {
    uint32_t c = a.cell[p], x = a.fx[p], y = a.fy[p], z = a.fz[p];
    advance_one(P, c, x, y, z, a.vx[p], a.vy[p], a.vz[p], dtdx, dtdy, dtdz);
    a.cell[p] = c;
    a.fx[p] = x;
    a.fy[p] = y;
    a.fz[p] = z;
  }
}

// Only a particle whose cell index is 0 or n on some axis (or beyond) can
// wrap, so interior cells are decided from the cell word alone, the in-cell
// offsets are read only for the rest, and a cell word is written only when it
// changes.
__device__ __forceinline__ void transfer_one(const KParams& P, const PartC32& a, long long p, uint32_t cell) {
  const uint32_t cx = cell & kCellMaskX, cy = (cell >> kCellBitsX) & kCellMaskY, cz = cell >> (kCellBitsX + kCellBitsY);
  if (cx - 2u < uint32_t(P.nx - 1) && cy - 2u < uint32_t(P.ny - 1) && cz - 2u < uint32_t(P.nz - 1)) return;
  C32 c = load_pos(a, p);
  wrap_c32(P, c);
  const uint32_t moved = pack_cell(c.i, c.j, c.k);
  if (moved != cell) a.cell[p] = moved;
}

// Cell words four at a time (16-byte loads), the remainder one by one.
__global__ void transfer_c32_kernel(KParams P, PartC32 a, long long n) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  const long long n4 = n >> 2;
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n4; q += stride) {
    const uint4 c = reinterpret_cast<const uint4*>(a.cell)[q];
    transfer_one(P, a, 4 * q, c.x);
    transfer_one(P, a, 4 * q + 1, c.y);
    transfer_one(P, a, 4 * q + 2, c.z);
    transfer_one(P, a, 4 * q + 3, c.w);
  }
  for (long long p = 4 * n4 + (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += stride)
    transfer_one(P, a, p, a.cell[p]);
}

// BCoutflow.f90:28-53 and ParticlesTransfer.f90:494-519 on the CELL32
// layout, for the in-place removal of outflow.cuh.  An in-cell offset decides
// an axis only when the cell index is 0 or n there (below / above), so the
// offsets are read only for those particles.
struct OutflowC32 {
  KParams P;
  PartC32 a;
  using Key = uint32_t;
  __device__ Key load_key(long long p) const { return a.cell[p]; }
  __device__ bool keep_wrap(long long p, uint32_t cell, int wrap) const {
    // interior cells 1 .. n-1 on every axis (packed as 2 .. n): kept, no wrap
    const uint32_t cx = cell & kCellMaskX, cy = (cell >> kCellBitsX) & kCellMaskY,
                   cz = cell >> (kCellBitsX + kCellBitsY);
    if (cx - 2u < uint32_t(P.nx - 1) && cy - 2u < uint32_t(P.ny - 1) && cz - 2u < uint32_t(P.nz - 1)) return true;
    C32 c;
    unpack_cell(cell, c.i, c.j, c.k);
    c.f[0] = (c.i == 0 || c.i == P.nx) ? a.fx[p] : kOffHalf;
    c.f[1] = (c.j == 0 || c.j == P.ny) ? a.fy[p] : kOffHalf;
    c.f[2] = (c.k == 0 || c.k == P.nz) ? a.fz[p] : kOffHalf;
    if (!keep_c32(P, c)) return false;
    if (wrap) {
      wrap_c32(P, c);
      const uint32_t moved = pack_cell(c.i, c.j, c.k);
      if (moved != cell) a.cell[p] = moved;
    }
    return true;
  }
  __device__ void move(long long d, long long s) const {
    a.cell[d] = a.cell[s];
    a.fx[d] = a.fx[s];
    a.fy[d] = a.fy[s];
    a.fz[d] = a.fz[s];
    a.vx[d] = a.vx[s];
    a.vy[d] = a.vy[s];
    a.vz[d] = a.vz[s];
    a.sp[d] = a.sp[s];
  }
};

// Per-species push constants in FP32.
struct SpeciesF32 {
  float etadt2[8];
  float tB[8][3];
  float sB[8][3];
};

__device__ inline void gather_c32(const KParams& P, const C32& c, const float4* __restrict__ E, float Ep[3]) {
  const float fx = off_f32(c.f[0]), fy = off_f32(c.f[1]), fz = off_f32(c.f[2]);
  float wx[2] = {1.0f - fx, fx}, wy[2] = {1.0f - fy, fy}, wz[2] = {1.0f - fz, fz};
  int i0 = min(max(c.i, 0), P.nx + 1), j0 = min(max(c.j, 0), P.ny + 1), k0 = min(max(c.k, 0), P.nz + 1);
  int i1 = min(max(c.i + 1, 0), P.nx + 1), j1 = min(max(c.j + 1, 0), P.ny + 1), k1 = min(max(c.k + 1, 0), P.nz + 1);
  Ep[0] = Ep[1] = Ep[2] = 0.0f;
  const int ii[2] = {i0, i1}, jj[2] = {j0, j1}, kk[2] = {k0, k1};
#pragma unroll
  for (int dk = 0; dk < 2; ++dk)
#pragma unroll
    for (int dj = 0; dj < 2; ++dj) {
      // node indices fit 32 bits: the packed cell word bounds nxp*nyp*nzp below 2^32
      const uint32_t row = uint32_t(P.nxp) * (uint32_t(jj[dj]) + uint32_t(P.nyp) * uint32_t(kk[dk]));
      float4 e0 = __ldg(E + row + ii[0]);
      float4 e1 = __ldg(E + row + ii[1]);
      float w = wy[dj] * wz[dk];
      float a0 = wx[0] * w, a1 = wx[1] * w;
      Ep[0] += e0.x * a0 + e1.x * a1;
      Ep[1] += e0.y * a0 + e1.y * a1;
      Ep[2] += e0.z * a0 + e1.z * a1;
    }
}

// AdvanceVelocity.f90:85-119 in FP32 (mode 0); Exp / Imp half steps
// (modes 1 / 2, AdvanceVelocity.f90:201-230, 311-340).
__device__ inline void boris_c32(const KParams& P, const SpeciesF32& S, int s, int mode, const float Ep[3], float v[3]) {
  if (P.fluid[s]) {
    if (P.gyration[s]) {
      float B[3] = {float(P.B0[0]), float(P.B0[1]), float(P.B0[2])};
      float vb = v[0] * B[0] + v[1] * B[1] + v[2] * B[2];
      float ib = 1.0f / (B[0] * B[0] + B[1] * B[1] + B[2] * B[2]);
      float vd0 = vb * B[0] + (Ep[1] * B[2] - Ep[2] * B[1]);
      float vd1 = vb * B[1] + (Ep[2] * B[0] - Ep[0] * B[2]);
      float vd2 = vb * B[2] + (Ep[0] * B[1] - Ep[1] * B[0]);
      v[0] = vd0 * ib;
      v[1] = vd1 * ib;
      v[2] = vd2 * ib;
    }
    return;
  }
  const float ve0 = float(P.ve[0]), ve1 = float(P.ve[1]), ve2 = float(P.ve[2]);
  const float e = S.etadt2[s];
  const float* tB = S.tB[s];
  float vmin[3], vmid[3];
  if (mode == 1) {
    vmin[0] = v[0] - ve0;
    vmin[1] = v[1] - ve1;
    vmin[2] = v[2] - ve2;
  } else {
    vmin[0] = v[0] - ve0 + e * Ep[0];
    vmin[1] = v[1] - ve1 + e * Ep[1];
    vmin[2] = v[2] - ve2 + e * Ep[2];
  }
  vmid[0] = vmin[0] + vmin[1] * tB[2] - vmin[2] * tB[1];
  vmid[1] = vmin[1] + vmin[2] * tB[0] - vmin[0] * tB[2];
  vmid[2] = vmin[2] + vmin[0] * tB[1] - vmin[1] * tB[0];
  if (mode == 0) {
    const float* sB = S.sB[s];
    v[0] = vmin[0] + vmid[1] * sB[2] - vmid[2] * sB[1] + ve0 + e * Ep[0];
    v[1] = vmin[1] + vmid[2] * sB[0] - vmid[0] * sB[2] + ve1 + e * Ep[1];
    v[2] = vmin[2] + vmid[0] * sB[1] - vmid[1] * sB[0] + ve2 + e * Ep[2];
    return;
  }
  float smid = vmid[0] * vmid[0] + vmid[1] * vmid[1] + vmid[2] * vmid[2];
  if (smid > 0.0f) {
    float smin = vmin[0] * vmin[0] + vmin[1] * vmin[1] + vmin[2] * vmin[2];
    float f = sqrtf(smin / smid);
    vmid[0] *= f;
    vmid[1] *= f;
    vmid[2] *= f;
  }
  if (mode == 1) {
    v[0] = vmid[0] + ve0 + e * Ep[0];
    v[1] = vmid[1] + ve1 + e * Ep[1];
    v[2] = vmid[2] + ve2 + e * Ep[2];
  } else {
    v[0] = vmid[0] + ve0;
    v[1] = vmid[1] + ve1;
    v[2] = vmid[2] + ve2;
  }
}

__device__ __forceinline__ void advance_velocity_one(const KParams& P, const SpeciesF32& S, const float4* E,
                                                     int mode, uint32_t cell, uint32_t fx, uint32_t fy, uint32_t fz,
                                                     float& vx, float& vy, float& vz, int sp) {
  C32 c;
  unpack_cell(cell, c.i, c.j, c.k);
  c.f[0] = fx;
  c.f[1] = fy;
  c.f[2] = fz;
  float Ep[3];
  gather_c32(P, c, E, Ep);
  float v[3] = {vx, vy, vz};
  boris_c32(P, S, sp, mode, Ep, v);
  vx = v[0];
  vy = v[1];
  vz = v[2];
}

// Streaming loads and stores for the particles, so that they leave the E
// table in L2 (as in push_advance_c32_kernel); thread q takes particles
// 4q .. 4q + 3 with 16-byte accesses, the tail of a count that is not a
// multiple of 4 one by one.
__global__ void __launch_bounds__(256, 3) advance_velocity_c32_kernel(KParams P, SpeciesF32 S, PartC32 a, long long n,
                                                                      const float4* E, int mode) {
  const long long nquad = n >> 2;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < nquad; q += stride) {
    const uint4 cell = __ldcs(reinterpret_cast<const uint4*>(a.cell) + q);
    const uint4 fx = __ldcs(reinterpret_cast<const uint4*>(a.fx) + q);
    const uint4 fy = __ldcs(reinterpret_cast<const uint4*>(a.fy) + q);
    const uint4 fz = __ldcs(reinterpret_cast<const uint4*>(a.fz) + q);
    float4 vx = __ldcs(reinterpret_cast<const float4*>(a.vx) + q);
    float4 vy = __ldcs(reinterpret_cast<const float4*>(a.vy) + q);
    float4 vz = __ldcs(reinterpret_cast<const float4*>(a.vz) + q);
    const char4 sp = __ldcs(reinterpret_cast<const char4*>(a.sp) + q);
    advance_velocity_one(P, S, E, mode, cell.x, fx.x, fy.x, fz.x, vx.x, vy.x, vz.x, sp.x);
    advance_velocity_one(P, S, E, mode, cell.y, fx.y, fy.y, fz.y, vx.y, vy.y, vz.y, sp.y);
    advance_velocity_one(P, S, E, mode, cell.z, fx.z, fy.z, fz.z, vx.z, vy.z, vz.z, sp.z);
    advance_velocity_one(P, S, E, mode, cell.w, fx.w, fy.w, fz.w, vx.w, vy.w, vz.w, sp.w);
    __stcs(reinterpret_cast<float4*>(a.vx) + q, vx);
    __stcs(reinterpret_cast<float4*>(a.vy) + q, vy);
    __stcs(reinterpret_cast<float4*>(a.vz) + q, vz);
  }
  for (long long p = 4 * nquad + (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += stride) {
    float vx = __ldcs(a.vx + p), vy = __ldcs(a.vy + p), vz = __ldcs(a.vz + p);
    advance_velocity_one(P, S, E, mode, __ldcs(a.cell + p), __ldcs(a.fx + p), __ldcs(a.fy + p), __ldcs(a.fz + p), vx,
                         vy, vz, __ldcs(a.sp + p));
    __stcs(a.vx + p, vx);
    __stcs(a.vy + p, vy);
    __stcs(a.vz + p, vz);
  }
}

// AdvanceVelocity of one step followed by AdvancePosition of the next, in one
// pass over the particles: the same operations as advance_velocity_c32_kernel
// (mode 0) then advance_position_c32_kernel, so the same bits, with one read
// and one write of each particle instead of two.  Thread q takes particles
// 4q .. 4q + 3 with 16-byte loads and stores, so four particles' bytes are in
// flight per thread before the E gathers that depend on them: 80 registers
// (no spills), 3 blocks of 256 per SM, and the E-field + push phase takes
// 3.05 ms at 268 M particles, against 3.56 ms for particle pairs (8-byte
// accesses, 80 registers), 3.40 ms for quads at 126 registers (2 blocks per
// SM) and 4.6 ms for one particle per thread (64 registers, 4 blocks per SM).
__device__ __forceinline__ void push_advance_one(const KParams& P, const SpeciesF32& S, const float4* E, float dtdx,
                                                 float dtdy, float dtdz, uint32_t& cell, uint32_t& fx, uint32_t& fy,
                                                 uint32_t& fz, float& vx, float& vy, float& vz, int sp) {
  C32 c;
  unpack_cell(cell, c.i, c.j, c.k);
  c.f[0] = fx;
  c.f[1] = fy;
  c.f[2] = fz;
  float Ep[3];
  gather_c32(P, c, E, Ep);
  float v[3] = {vx, vy, vz};
  boris_c32(P, S, sp, 0, Ep, v);
  vx = v[0];
  vy = v[1];
  vz = v[2];
  move_axis(c.i, c.f[0], v[0] * dtdx, P.nx, P.xflow);
  move_axis(c.j, c.f[1], v[1] * dtdy, P.ny, P.yflow);
  move_axis(c.k, c.f[2], v[2] * dtdz, P.nz, P.zflow);
  cell = pack_cell(c.i, c.j, c.k);
  fx = c.f[0];
  fy = c.f[1];
  fz = c.f[2];
}

__global__ void __launch_bounds__(256, 3) push_advance_c32_kernel(KParams P, SpeciesF32 S, PartC32 a, long long n,
                                                                   const float4* E, float dtdx, float dtdy,
                                                                   float dtdz) {
  const long long nquad = n >> 2;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < nquad; q += stride) {
    uint4 cell = __ldcs(reinterpret_cast<const uint4*>(a.cell) + q);
    uint4 fx = __ldcs(reinterpret_cast<const uint4*>(a.fx) + q);
    uint4 fy = __ldcs(reinterpret_cast<const uint4*>(a.fy) + q);
    uint4 fz = __ldcs(reinterpret_cast<const uint4*>(a.fz) + q);
    float4 vx = __ldcs(reinterpret_cast<const float4*>(a.vx) + q);
    float4 vy = __ldcs(reinterpret_cast<const float4*>(a.vy) + q);
    float4 vz = __ldcs(reinterpret_cast<const float4*>(a.vz) + q);
    const char4 sp = __ldcs(reinterpret_cast<const char4*>(a.sp) + q);
    push_advance_one(P, S, E, dtdx, dtdy, dtdz, cell.x, fx.x, fy.x, fz.x, vx.x, vy.x, vz.x, sp.x);
    push_advance_one(P, S, E, dtdx, dtdy, dtdz, cell.y, fx.y, fy.y, fz.y, vx.y, vy.y, vz.y, sp.y);
    push_advance_one(P, S, E, dtdx, dtdy, dtdz, cell.z, fx.z, fy.z, fz.z, vx.z, vy.z, vz.z, sp.z);
    push_advance_one(P, S, E, dtdx, dtdy, dtdz, cell.w, fx.w, fy.w, fz.w, vx.w, vy.w, vz.w, sp.w);
    __stcs(reinterpret_cast<float4*>(a.vx) + q, vx);
    __stcs(reinterpret_cast<float4*>(a.vy) + q, vy);
    __stcs(reinterpret_cast<float4*>(a.vz) + q, vz);
    __stcs(reinterpret_cast<uint4*>(a.cell) + q, cell);
    __stcs(reinterpret_cast<uint4*>(a.fx) + q, fx);
    __stcs(reinterpret_cast<uint4*>(a.fy) + q, fy);
    __stcs(reinterpret_cast<uint4*>(a.fz) + q, fz);
  }
  for (long long p = 4 * nquad + (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += stride) {
    uint32_t cell = __ldcs(a.cell + p), fx = __ldcs(a.fx + p), fy = __ldcs(a.fy + p), fz = __ldcs(a.fz + p);
    float vx = __ldcs(a.vx + p), vy = __ldcs(a.vy + p), vz = __ldcs(a.vz + p);
    push_advance_one(P, S, E, dtdx, dtdy, dtdz, cell, fx, fy, fz, vx, vy, vz, __ldcs(a.sp + p));
    __stcs(a.vx + p, vx);
    __stcs(a.vy + p, vy);
    __stcs(a.vz + p, vz);
    __stcs(a.cell + p, cell);
    __stcs(a.fx + p, fx);
    __stcs(a.fy + p, fy);
    __stcs(a.fz + p, fz);
  }
}

__device__ inline int fold_index(int i, int n, int open) {
  if (open) return i < 1 ? 1 : (i > n ? n : i);
  // periodic: the interior node congruent to i modulo n -- one period for
  // the ghost layers, a closed-form remainder for anything farther out
  if (i < 1)
    i += n;
  else if (i > n)
    i -= n;
  if (i >= 1 && i <= n) return i;
  long long r = ((long long)i - 1) % n;
  return int(r < 0 ? r + n : r) + 1;
}

__device__ inline unsigned long long stencil_key(int i, int j, int k, int s) {
  auto c = [](int v) { v += 2; return (unsigned long long)(v < 0 ? 0 : (v > 0xFFFFF ? 0xFFFFF : v)); };
  return (c(i) | (c(j) << 20) | (c(k) << 40)) << 4 | (unsigned long long)s;
}

// Offset (0 or 1) along axis a of corner q of the CIC stencil, in the order
// of ParticlesGridify.f90:70-88 (F1..F8: 000, 100, 010, 001, 110, 011, 101,
// 111).  A function rather than a table: with q and a known at compile time
// it folds to a constant (a __constant__ table made the tiled deposit 36 %
// slower).
__device__ __forceinline__ int corner(int q, int a) {
  return a == 0 ? (q == 1 || q == 4 || q == 6 || q == 7)
                : a == 1 ? (q == 2 || q == 4 || q == 5 || q == 7) : (q == 3 || q == 5 || q == 6 || q == 7);
}

// CIC weights of a CELL32 particle: products in FP64 of the offsets (exact in
// FP64), each rounded once to the deposit's 2^-40 fixed point.  Every CELL32
// deposit kernel takes its weights from here, so their sums agree bit for bit.
__device__ inline void cic_fixed_c32(const C32& c, long long w[8], double F[8]) {
  const double x = off_one_plus(c.f[0]), y = off_one_plus(c.f[1]), z = off_one_plus(c.f[2]);
  const double wx[2] = {2.0 - x, x - 1.0}, wy[2] = {2.0 - y, y - 1.0}, wz[2] = {2.0 - z, z - 1.0};
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    F[q] = (wx[corner(q, 0)] * wy[corner(q, 1)]) * wz[corner(q, 2)];
    w[q] = fixed40_rn(F[q]);
  }
}

// Warp-aggregated fixed-point deposit (see particles_exact.cu deposit8).
__device__ inline void deposit8(unsigned long long key, bool active, const long long w[8], const long long nodes[8],
                                unsigned long long* plane) {
  unsigned act = __ballot_sync(0xffffffffu, active);
  if (!active) return;
  unsigned grp = __match_any_sync(act, key);
  int lane = threadIdx.x & 31;
  int leader = __ffs(grp) - 1;
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    unsigned long long u = (unsigned long long)(w[q] + (1LL << kDepositShift));
    unsigned lo = unsigned(u & 0x3FFFFu), hi = unsigned(u >> 18);
    unsigned slo = __reduce_add_sync(grp, lo);
    unsigned shi = __reduce_add_sync(grp, hi);
    if (lane == leader) {
      long long cnt = __popc(grp);
      long long sum = (long long)(((unsigned long long)shi << 18) + (unsigned long long)slo) - cnt * (1LL << kDepositShift);
      atomicAdd(plane + nodes[q], (unsigned long long)sum);
    }
  }
}

// ParticlesGridify.f90:65-123 with FP64 weights rounded to 2^-40 and ghost
// folds applied to the node indices.
__global__ void deposit_c32_kernel(KParams P, PartC32 a, long long n, unsigned long long* Nacc,
                                   unsigned long long* Facc) {
  long long stride = (long long)gridDim.x * blockDim.x;
  long long n_round = ((n + 31) / 32) * 32;
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n_round; p += stride) {
    bool active = p < n;
    long long w[8] = {0, 0, 0, 0, 0, 0, 0, 0}, nodes[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    double Fw[8];
    int s = 0;
    unsigned long long key = ~0ull;
    if (active) {
      C32 c = load_pos(a, p);
      s = a.sp[p];
      cic_fixed_c32(c, w, Fw);
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        int i = fold_index(c.i + corner(q, 0), P.nx, P.xflow), j = fold_index(c.j + corner(q, 1), P.ny, P.yflow),
            k = fold_index(c.k + corner(q, 2), P.nz, P.zflow);
        nodes[q] = node_index(P, i, j, k);
      }
      key = stencil_key(c.i, c.j, c.k, s);
    }
    deposit8(key, active, w, nodes, Nacc + (long long)s * P.nodes);
    if (Facc && active) {
      double vel[3] = {a.vx[p], a.vy[p], a.vz[p]};
      for (int c = 0; c < 3; ++c)
        for (int q = 0; q < 8; ++q)
          atomicAdd(Facc + ((long long)s * 3 + c) * P.nodes + nodes[q],
                    (unsigned long long)__double2ll_rn(Fw[q] * vel[c] * kFluxScale));
    }
  }
}

// ParticlesGridify.f90:65-123, shared-memory tiled, one tile per warp.
// Particles are stored in cell order (initialisation and every append go cell
// by cell; compaction keeps the order) and move a small fraction of a cell per
// step, so a warp's kDepWarpChunk consecutive particles (one or two cells
// at 64 per cell) touch a small box of nodes.  Each warp takes the bounding
// box of its particles' CIC stencils (base node + 1 on every axis, by
// species) with warp reductions, accumulates the fixed-point weights in its
// own slice of shared memory with 32-bit atomics -- weights lie in [0, 2^40],
// split into 20-bit halves so neither half-sum can overflow -- and adds every
// touched node to global memory once, with the ghost folds applied.  A warp
// whose box does not fit its slice (a row or plane boundary, or a particle
// far from the rest after BCoutflow filled a hole) falls back to one global
// atomic per particle corner.  Warps synchronise only with themselves: no
// block barrier holds a warp's loads behind another warp's atomics.
// Integer sums are exact and order-independent: N is bit-identical to the
// warp-aggregated kernel's.
constexpr int kDepPer = 2;                       // particles per lane
constexpr int kDepWarpChunk = 32 * kDepPer;      // particles per warp iteration
constexpr int kDepWarpTile = 512;                // tile entries per warp (two u32 halves each: 4 KB)
constexpr int kDepWarps = 8;                     // warps per CTA

__global__ void __launch_bounds__(256, 4) deposit_tile_c32_kernel(KParams P, PartC32 a, long long n,
                                                                  unsigned long long* Nacc) {
  extern __shared__ unsigned int dep_tile[];  // per warp: [2][kDepWarpTile] low and high 20-bit halves
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  unsigned int* lo = dep_tile + warp * 2 * kDepWarpTile;
  unsigned int* hi = lo + kDepWarpTile;
  const long long warps = (long long)gridDim.x * kDepWarps;
  for (long long base = ((long long)blockIdx.x * kDepWarps + warp) * kDepWarpChunk; base < n;
       base += warps * kDepWarpChunk) {
    C32 c[kDepPer];
    int sp[kDepPer];
    bool act[kDepPer];
    int imin = INT_MAX, imax = INT_MIN, jmin = INT_MAX, jmax = INT_MIN, kmin = INT_MAX, kmax = INT_MIN;
    int smin = INT_MAX, smax = INT_MIN;
#pragma unroll
    for (int m = 0; m < kDepPer; ++m) {
      const long long p = base + lane + 32 * m;
      act[m] = p < n;
      if (act[m]) {
        c[m] = load_pos_cs(a, p);
        sp[m] = __ldcs(a.sp + p);
        imin = min(imin, c[m].i), imax = max(imax, c[m].i);
        jmin = min(jmin, c[m].j), jmax = max(jmax, c[m].j);
        kmin = min(kmin, c[m].k), kmax = max(kmax, c[m].k);
        smin = min(smin, sp[m]), smax = max(smax, sp[m]);
      }
    }
    // the warp's bounding box (lane 0 always holds a particle: base < n)
    imin = __reduce_min_sync(0xffffffffu, imin), imax = __reduce_max_sync(0xffffffffu, imax);
    jmin = __reduce_min_sync(0xffffffffu, jmin), jmax = __reduce_max_sync(0xffffffffu, jmax);
    kmin = __reduce_min_sync(0xffffffffu, kmin), kmax = __reduce_max_sync(0xffffffffu, kmax);
    smin = __reduce_min_sync(0xffffffffu, smin), smax = __reduce_max_sync(0xffffffffu, smax);
    const long long bi = (long long)imax - imin + 2, bj = (long long)jmax - jmin + 2, bk = (long long)kmax - kmin + 2,
                    bs = (long long)smax - smin + 1;
    const long long vol = bi * bj * bk * bs;
    if (vol <= kDepWarpTile) {
      const int vi = int(vol);
      for (int e = lane; e < vi; e += 32) lo[e] = 0u, hi[e] = 0u;
      __syncwarp();
#pragma unroll
      for (int m = 0; m < kDepPer; ++m) {
        if (!act[m]) continue;
        long long w[8];
        double F[8];
        cic_fixed_c32(c[m], w, F);
        const int b0 = (((sp[m] - smin) * int(bk) + (c[m].k - kmin)) * int(bj) + (c[m].j - jmin)) * int(bi) +
                       (c[m].i - imin);
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const unsigned long long wq = (unsigned long long)w[q];
          const int e = b0 + (corner(q, 2) * int(bj) + corner(q, 1)) * int(bi) + corner(q, 0);
          atomicAdd(lo + e, unsigned(wq & 0xFFFFFu));
          atomicAdd(hi + e, unsigned(wq >> 20));
        }
      }
      __syncwarp();
      for (int e = lane; e < vi; e += 32) {
        const unsigned l = lo[e], h = hi[e];
        if ((l | h) == 0u) continue;
        int r = e;
        const int ii = r % int(bi) + imin;
        r /= int(bi);
        const int jj = r % int(bj) + jmin;
        r /= int(bj);
        const int kk = r % int(bk) + kmin;
        const int ss = r / int(bk) + smin;
        const int i = fold_index(ii, P.nx, P.xflow), j = fold_index(jj, P.ny, P.yflow),
                  k = fold_index(kk, P.nz, P.zflow);
        const unsigned long long v = ((unsigned long long)h << 20) + (unsigned long long)l;
        atomicAdd(Nacc + (long long)ss * P.nodes + node_index(P, i, j, k), v);
      }
      __syncwarp();
    } else {
#pragma unroll
      for (int m = 0; m < kDepPer; ++m) {
        if (!act[m]) continue;
        long long w[8];
        double F[8];
        cic_fixed_c32(c[m], w, F);
        unsigned long long* plane = Nacc + (long long)sp[m] * P.nodes;
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const int i = fold_index(c[m].i + corner(q, 0), P.nx, P.xflow),
                    j = fold_index(c[m].j + corner(q, 1), P.ny, P.yflow),
                    k = fold_index(c[m].k + corner(q, 2), P.nz, P.zflow);
          atomicAdd(plane + node_index(P, i, j, k), (unsigned long long)w[q]);
        }
      }
    }
  }
}

__global__ void energy_particles_c32_kernel(KParams P, PartC32 a, long long n, double* partial) {
  __shared__ double sh[32];
  double acc = 0.0;
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
    int s = a.sp[p];
    double vx = a.vx[p], vy = a.vy[p], vz = a.vz[p];
    acc += P.n2p[s] * P.mass[s] * (vx * vx + vy * vy + vz * vz);
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < int(blockDim.x >> 5); ++w) t += sh[w];
    partial[blockIdx.x] = t;
  }
}

__global__ void finish_sum_kernel(const double* partial, int nb, double scale, double* out) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    double t = 0.0;
    for (int b = 0; b < nb; ++b) t += partial[b];
    *out = t * scale;
  }
}

SpeciesF32 species_f32(const KParams& P, double dt, double deltat, int mode) {
  SpeciesF32 S;
  for (int s = 0; s < 8; ++s) {
    double e = mode == 0 ? 0.5 * dt * P.eta[s] : 0.5 * dt * P.eta[s] * 2.0 * deltat / dt;
    S.etadt2[s] = float(e);
    for (int c = 0; c < 3; ++c) {
      S.tB[s][c] = float(mode == 0 ? P.tB[s][c] : P.tB[s][c] * 2.0 * deltat / dt);
      S.sB[s][c] = float(P.sB[s][c]);
    }
  }
  return S;
}

}  // namespace

int scan_scratch_ints(int n) {
  if (n <= kScanTile) return 0;
  int nb = (n + kScanTile - 1) / kScanTile;
  return 2 * nb + 2 + scan_scratch_ints(nb);
}

cudaError_t launch_scan_int(const int* in, int* out, int n, int* total, int* scratch, cudaStream_t st) {
  if (n <= 0) return cudaMemsetAsync(total, 0, sizeof(int), st);
  if (n <= kScanTile) {
    note_launch();
    scan_tiles_kernel<<<1, kScanThreads, 0, st>>>(in, out, n, total);
    return cudaGetLastError();
  }
  int nb = (n + kScanTile - 1) / kScanTile;
  int* sums = scratch;
  int* offs = scratch + nb + 1;
  note_launch();
  scan_tiles_kernel<<<nb, kScanThreads, 0, st>>>(in, out, n, sums);
  cudaError_t e = launch_scan_int(sums, offs, nb, total, offs + nb + 1, st);
  if (e != cudaSuccess) return e;
  note_launch();
  scan_add_kernel<<<nb, kScanThreads, 0, st>>>(out, n, offs);
  return cudaGetLastError();
}

cudaError_t launch_advance_position_c32(const KParams& P, PartC32 a, long long n, double dt, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  note_launch();
  advance_position_c32_kernel<<<persistent_grid(n), kThreads, 0, st>>>(P, a, n, float(dt / P.dx), float(dt / P.dy),
                                                                       float(dt / P.dz));
  return cudaGetLastError();
}

cudaError_t launch_transfer_c32(const KParams& P, PartC32 a, long long n, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  note_launch();
  transfer_c32_kernel<<<persistent_grid(n), kThreads, 0, st>>>(P, a, n);
  return cudaGetLastError();
}

cudaError_t launch_outflow_c32(const KParams& P, PartC32 a, long long n, uint2* words, int* block_counts,
                               int* block_offsets, int* count, int wrap, int* err, cudaStream_t st,
                               const OutflowSplit* split) {
  return launch_outflow_inplace(OutflowC32{P, a}, n, words, block_counts, block_offsets, count, wrap, err, st, split);
}

cudaError_t launch_advance_velocity_c32(const KParams& P, PartC32 a, long long n, const float4* E, double dt,
                                        double deltat, int mode, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  SpeciesF32 S = species_f32(P, dt, deltat, mode);
  note_launch();
  advance_velocity_c32_kernel<<<persistent_grid((n + 3) / 4), kThreads, 0, st>>>(P, S, a, n, E, mode);
  return cudaGetLastError();
}

cudaError_t launch_push_advance_c32(const KParams& P, PartC32 a, long long n, const float4* E, double dt,
                                    cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  SpeciesF32 S = species_f32(P, dt, 0.0, 0);
  note_launch();
  push_advance_c32_kernel<<<persistent_grid((n + 3) / 4), kThreads, 0, st>>>(P, S, a, n, E, float(dt / P.dx),
                                                                            float(dt / P.dy), float(dt / P.dz));
  return cudaGetLastError();
}

cudaError_t launch_deposit_c32(const KParams& P, PartC32 a, long long n, unsigned long long* Nacc,
                               unsigned long long* Facc, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  if (!Facc) {
    const size_t smem = size_t(kDepWarps) * 2 * sizeof(unsigned int) * kDepWarpTile;
    static bool attr = false;
    if (!attr) {
      cudaError_t e = cudaFuncSetAttribute(deposit_tile_c32_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)smem);
      if (e != cudaSuccess) return e;
      attr = true;
    }
    static int per_sm = 0;
    if (!per_sm) {
      cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, deposit_tile_c32_kernel, 256, smem);
      if (e != cudaSuccess) return e;
      if (per_sm < 1) per_sm = 1;
    }
    const long long chunks = (n + kDepWarps * kDepWarpChunk - 1) / (kDepWarps * kDepWarpChunk),
                    full = 148LL * per_sm;
    const int grid = int(chunks < full ? chunks : full);
    note_launch();
    deposit_tile_c32_kernel<<<grid, 256, smem, st>>>(P, a, n, Nacc);
    return cudaGetLastError();
  }
  note_launch();
  deposit_c32_kernel<<<persistent_grid(n), kThreads, 0, st>>>(P, a, n, Nacc, Facc);
  return cudaGetLastError();
}

cudaError_t launch_energy_particles_c32(const KParams& P, PartC32 a, long long n, ReduceBuf rb, cudaStream_t st) {
  int nb = persistent_grid(n > 0 ? n : 1);
  if (nb > rb.max_blocks) nb = rb.max_blocks;
  note_launch();
  energy_particles_c32_kernel<<<nb, kThreads, 0, st>>>(P, a, n, rb.partial);
  note_launch();
  finish_sum_kernel<<<1, 32, 0, st>>>(rb.partial, nb, 0.5, rb.result);
  return cudaGetLastError();
}

}  // namespace picard
