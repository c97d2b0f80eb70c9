// common.cuh -- device-side definitions shared by every kernel of libpicard_gpu.
//
// Grid layout in HBM: every node array is the reference's (Nx+2, Ny+2, Nz+2)
// column-major box (x fastest) with a one-node ghost layer, 0-based here:
// node (i, j, k), i in [0, Nx+1], sits at x = Lx_min + (i - 0.5) dx.
// Per-species and per-component arrays are stored plane by plane
// (species-major), so every deposit and stencil touches one contiguous box.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "picard_gpu.h"

namespace picard {

// physical constants, picard.f90:56-66
constexpr double kTau = 6.2831853071795864769252867665590;
constexpr double kEc = 1.60217646e-19;
constexpr double kMp = 1.6726216e-27;
constexpr double kMe = 9.1093819e-31;
constexpr double kEps0 = 8.854187817e-12;
constexpr double kKb = 1.380650e-23;
constexpr double kMu0 = 1.25663706143591729538505735331180e-6;

// Fixed-point scale of the deposit accumulators: one macro-particle's CIC
// weight (in [0, 1]) is stored as round(w * 2^40) in an int64, so the sum is
// exact and order-independent and a node holds up to 2^23 particle weights
// per species.
constexpr int kDepositShift = 40;
constexpr double kDepositScale = 1099511627776.0;  // 2^40
// Flux accumulators hold round(w * v * 2^20) (v in m/s).
constexpr int kFluxShift = 20;
constexpr double kFluxScale = 1048576.0;  // 2^20

// Packed CELL32 base-node index: (i+1) | (j+1) << 11 | (k+1) << 22, where
// (i, j, k) is the 0-based CIC lower node, in [-1, N+1] per axis.
constexpr uint32_t kCellBitsX = 11, kCellBitsY = 11, kCellBitsZ = 10;
constexpr uint32_t kCellMaskX = (1u << kCellBitsX) - 1u;
constexpr uint32_t kCellMaskY = (1u << kCellBitsY) - 1u;
constexpr uint32_t kCellMaskZ = (1u << kCellBitsZ) - 1u;

__host__ __device__ inline uint32_t pack_cell(int i, int j, int k) {
  return uint32_t(i + 1) | (uint32_t(j + 1) << kCellBitsX) | (uint32_t(k + 1) << (kCellBitsX + kCellBitsY));
}
__host__ __device__ inline void unpack_cell(uint32_t c, int& i, int& j, int& k) {
  i = int(c & kCellMaskX) - 1;
  j = int((c >> kCellBitsX) & kCellMaskY) - 1;
  k = int(c >> (kCellBitsX + kCellBitsY)) - 1;
}

// Kernel-argument copy of the run parameters (passed by value).
struct KParams {
  int nx, ny, nz;
  int nxp, nyp, nzp;  // nx + 2 ...
  long long nodes;    // nxp * nyp * nzp
  int species;
  int xflow, yflow, zflow;
  int produce_dt_scaled;
  double xmin, xmax, ymin, ymax, zmin, zmax;
  double Lx_min, Lx_max, Ly_min, Ly_max, Lz_min, Lz_max;
  double dx, dy, dz, dV;
  double dt;
  double ve[3], E0[3], B0[3];
  int gyration[8], fluid[8];
  int ipp[8], epp[8], hpp[8];
  double mass[8], charge[8], kelvin[8], n2p[8], eta[8];
  double v0[8][3];
  double tB[8][3], sB[8][3];
  double vn[8], Qn[8], nu_i[8], nu_d[8], Ek[8];
  double ue[8], uh[8], ui[8];  // ParticlesProduce.f90:26-36
  uint64_t seed;
};

__host__ __device__ inline long long node_index(const KParams& P, int i, int j, int k) {
  return (long long)i + (long long)P.nxp * ((long long)j + (long long)P.nyp * (long long)k);
}

// ------------------------------------------------------------------ Philox
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11), written from the paper.
__host__ __device__ inline void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    uint64_t p0 = (uint64_t)0xD2511F53u * c[0];
    uint64_t p1 = (uint64_t)0xCD9E8D57u * c[2];
    uint32_t hi0 = uint32_t(p0 >> 32), lo0 = uint32_t(p0);
    uint32_t hi1 = uint32_t(p1 >> 32), lo1 = uint32_t(p1);
    uint32_t n0 = hi1 ^ c[1] ^ k0;
    uint32_t n2 = hi0 ^ c[3] ^ k1;
    c[0] = n0;
    c[1] = lo1;
    c[2] = n2;
    c[3] = lo0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
}

// One draw site: counter (a, b, iteration, tag << 24 | block), key = seed.
// Uniform n uses block n/2, words 2(n%2) and 2(n%2)+1, as a 53-bit double.
struct Site {
  uint32_t a, b, it, tag;
  uint32_t k0, k1;
  uint32_t blk;
  uint32_t w[4];
  __host__ __device__ Site(uint64_t seed, uint32_t a_, uint32_t b_, uint32_t it_, uint32_t tag_)
      : a(a_), b(b_), it(it_), tag(tag_), k0(uint32_t(seed)), k1(uint32_t(seed >> 32)), blk(0xFFFFFFFFu) {}
  __host__ __device__ double u(uint32_t n) {
    uint32_t bk = n >> 1;
    if (bk != blk) {
      w[0] = a;
      w[1] = b;
      w[2] = it;
      w[3] = (tag << 24) | bk;
      philox4x32_10(w, k0, k1);
      blk = bk;
    }
    // selects, not an index: a draw number known only at run time keeps w in registers
    const uint32_t w0 = (n & 1) ? w[2] : w[0], w1 = (n & 1) ? w[3] : w[1];
    return ((double)(w0 >> 5) * 67108864.0 + (double)(w1 >> 6)) * (1.0 / 9007199254740992.0);
  }
};

constexpr uint32_t kTagInit = 1, kTagInflow = 2, kTagProduceCount = 3, kTagProduceParticle = 4;

// ------------------------------------------------------------ particle sets

struct PartF64 {
  double *x, *y, *z, *vx, *vy, *vz;
  int8_t* sp;
};
// CELL32 particles: packed base node, in-cell offsets as 32-bit fixed point
// (f / 2^32 in [0, 1) of a cell), FP32 velocities, species.
struct PartC32 {
  uint32_t* cell;
  uint32_t *fx, *fy, *fz;
  float *vx, *vy, *vz;
  int8_t* sp;
};

// In-cell offset 1/2 (the cell centre of the reference's node spacing).
constexpr uint32_t kOffHalf = 0x80000000u;

// An in-cell offset as FP64 (exact) and as FP32 (its leading 23 bits).
__host__ __device__ inline double off_f64(uint32_t f) { return (double)f * (1.0 / 4294967296.0); }
__device__ inline float off_f32(uint32_t f) { return __uint_as_float((f >> 9) | 0x3F800000u) - 1.0f; }
// 1 + f / 2^32 as FP64, exactly, built from the bits (the 32 offset bits are
// the top of the 52-bit mantissa): no conversion instruction.  For x in
// [1, 2), 2 - x and x - 1 are exact.
__device__ inline double off_one_plus(uint32_t f) {
  return __hiloint2double(int(0x3FF00000u | (f >> 12)), int(f << 20));
}
// round(F * 2^40) to nearest, ties to even (the rounding of __double2ll_rn),
// for F in [0, 2^11): one FMA against 1.5 * 2^52 leaves the integer in the
// low mantissa bits.
__device__ inline long long fixed40_rn(double F) {
  return __double_as_longlong(fma(F, 1099511627776.0, 6755399441055744.0)) - 0x4338000000000000LL;
}

// Process-wide count of kernels launched by this library (every launch
// wrapper calls it once per launch); reported by picard_gpu_get_stats.
void note_launch();
long long launches_so_far();

// Status word written by kernels (first error wins).
enum DevError : int { kDevOk = 0, kDevCapacity = 1, kDevRange = 2, kDevTimeout = 3 };

}  // namespace picard
