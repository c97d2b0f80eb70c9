// particles_exact.cu -- FP64 particle kernels with the reference's arithmetic.
//
// Compiled with --fmad=false: every multiply and add is rounded separately,
// in the order the reference writes its expressions, so positions, cell
// indices and the removed / wrapped particle sets equal the FP64 oracle's.
// This unit also holds the stochastic generators (init, inflow, produce),
// which both particle layouts share: particles are generated in FP64 and
// converted to the CELL32 layout only when stored.
#include <cuda_runtime.h>

#include <cmath>

#include "common.cuh"
#include "kernels.cuh"
#include "outflow.cuh"

namespace picard {

namespace {

constexpr int kThreads = 256;

inline int grid_for(long long n, int threads = kThreads) {
  long long b = (n + threads - 1) / threads;
  if (b < 1) b = 1;
  if (b > 2147483647LL) b = 2147483647LL;
  return int(b);
}

// ------------------------------------------------------------ generation

// Tools.f90:30-48 normal(): r1 for the angle, r2 = 1 - u in (0, 1].
__device__ double normal_from(Site& s, uint32_t n) {
  double r1 = s.u(n);
  double r2 = 1.0 - s.u(n + 1);
  return sqrt(-2.0 * log(r2)) * sin(kTau * r1);
}

// Tools.f90:2-28 Gaussian()
__device__ void gaussian_from(Site& s, uint32_t n, double u[3], const double v[3], double t, double m) {
  if (t > 0.0 && m > 0.0) {
    double a = m / (2.0 * kKb * t);
    double pw = sqrt(1.0 / a);
    for (int c = 0; c < 3; ++c) u[c] = normal_from(s, n + 2 * c);
    double r2 = sqrt(2.0);
    for (int c = 0; c < 3; ++c) u[c] = u[c] * pw / r2;
    for (int c = 0; c < 3; ++c) u[c] = u[c] + v[c];
  } else {
    for (int c = 0; c < 3; ++c) u[c] = v[c];
  }
}

// -dt/2 rotation with |v - ve| restored (ParticlesInitialize.f90:73-80).
__device__ void half_rotate(double v[3], const double ve[3], const double tB[3]) {
  double vmin[3], vmid[3];
  for (int c = 0; c < 3; ++c) vmin[c] = v[c] - ve[c];
  vmid[0] = vmin[0] + vmin[1] * tB[2] - vmin[2] * tB[1];
  vmid[1] = vmin[1] + vmin[2] * tB[0] - vmin[0] * tB[2];
  vmid[2] = vmin[2] + vmin[0] * tB[1] - vmin[1] * tB[0];
  double smid = vmid[0] * vmid[0] + vmid[1] * vmid[1] + vmid[2] * vmid[2];
  if (smid > 0.0) {
    double smin = vmin[0] * vmin[0] + vmin[1] * vmin[1] + vmin[2] * vmin[2];
    double f = sqrt(smin / smid);
    for (int c = 0; c < 3; ++c) vmid[c] = vmid[c] * f;
  }
  for (int c = 0; c < 3; ++c) v[c] = vmid[c] + ve[c];
}

// Member `m` of the group (ss, pp) at cell `a`: m = 0 is the ion,
// 1..epp its electrons, epp+1.. its protons.  ParticlesInitialize.f90:65-113,
// BCinflow.f90:66-114.
__device__ void gen_member(const KParams& P, uint32_t tag, uint32_t it, uint32_t a, int ss, int pp, int m, double x0,
                           double y0, double z0, double x[3], double v[3], int& sp) {
  int s0 = ss - 1;
  Site ion(P.seed, a, (uint32_t(ss) << 24) | (uint32_t(pp) << 8), it, tag);
  x[0] = x0 + P.dx * ion.u(0);
  x[1] = y0 + P.dy * ion.u(1);
  x[2] = z0 + P.dz * ion.u(2);
  // The ion draws its velocity from its own site after the position (from
  // u(3)); an electron or proton from a site of its own (from u(0)).  One
  // code path for both, so that a warp holding ions and their members runs
  // the Gaussian draws and the rotation once, not once per kind.
  const bool is_ion = m == 0;
  const int t = is_ion ? s0 : (m <= P.epp[s0] ? 0 : 1);  // member: 0 = electron, 1 = proton
  Site src = is_ion ? ion : Site(P.seed, a, (uint32_t(ss) << 24) | (uint32_t(pp) << 8) | uint32_t(m), it, tag);
  gaussian_from(src, is_ion ? 3u : 0u, v, P.v0[s0], P.kelvin[t], P.mass[t]);
  half_rotate(v, P.ve, P.tB[t]);
  sp = t;
}

// Slot of (ss, pp, member) inside one cell's block of created particles.
__device__ inline void decode_group(const KParams& P, const int* prefix, int local, int& ss, int& pp, int& m) {
  int s0 = 0;
  while (s0 < P.species - 1 && local >= prefix[s0 + 1]) ++s0;
  int g = 1 + P.epp[s0] + P.hpp[s0];
  int r = local - prefix[s0];
  ss = s0 + 1;
  pp = r / g + 1;
  m = r % g;
}

// Stores one FP64 particle in either layout.
__device__ inline void store_f64(PartF64 o, long long slot, const double x[3], const double v[3], int sp) {
  o.x[slot] = x[0];
  o.y[slot] = x[1];
  o.z[slot] = x[2];
  o.vx[slot] = v[0];
  o.vy[slot] = v[1];
  o.vz[slot] = v[2];
  o.sp[slot] = int8_t(sp);
}

// Base node (floor) and in-cell fraction of one coordinate, for CELL32.
// Position x on an axis -> CIC base node i and the 32-bit fixed-point offset
// f = round((t - floor t) 2^32) of t = (x - lmin)/d + 1/2 (a carry moves to
// the next node).  Far-out positions are pinned one node beyond the guard
// layer, where BCoutflow removes them.
__device__ inline void to_cell(double x, double lmin, double d, int nmax, int& i, uint32_t& f) {
  double t = (x - lmin) / d + 0.5;
  if (!(t > -2.0)) t = -2.0;  // NaN too
  if (t > nmax + 3.0) t = nmax + 3.0;
  double fl = floor(t);
  i = int(fl);
  unsigned long long q = (unsigned long long)__double2ull_rn((t - fl) * 4294967296.0);
  if (q >> 32) {
    q = 0;
    i += 1;
  }
  f = uint32_t(q);
  if (i < -1) {
    i = -1;
    f = 0u;
  }
  if (i > nmax + 1) {
    i = nmax + 1;
    f = 0xFFFFFFFFu;
  }
}

__device__ inline void store_c32(const KParams& P, PartC32 o, long long slot, const double x[3], const double v[3],
                                 int sp) {
  int i, j, k;
  uint32_t fx, fy, fz;
  to_cell(x[0], P.Lx_min, P.dx, P.nx, i, fx);
  to_cell(x[1], P.Ly_min, P.dy, P.ny, j, fy);
  to_cell(x[2], P.Lz_min, P.dz, P.nz, k, fz);
  o.cell[slot] = pack_cell(i, j, k);
  o.fx[slot] = fx;
  o.fy[slot] = fy;
  o.fz[slot] = fz;
  o.vx[slot] = float(v[0]);
  o.vy[slot] = float(v[1]);
  o.vz[slot] = float(v[2]);
  o.sp[slot] = int8_t(sp);
}

struct GroupPrefix {
  int p[9];
};

__host__ inline GroupPrefix group_prefix(const KParams& P) {
  GroupPrefix g;
  g.p[0] = 0;
  for (int s = 0; s < 8; ++s) g.p[s + 1] = g.p[s] + (s < P.species ? P.ipp[s] * (1 + P.epp[s] + P.hpp[s]) : 0);
  return g;
}

// ParticlesInitialize.f90:54-119: one thread per created particle, slot =
// start + (interior cell in k, j, i order) * per_cell + slot inside the cell.
template <class Store>
__global__ void init_kernel(KParams P, GroupPrefix G, long long start, long long total, Store store) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= total) return;
  int per_cell = G.p[P.species];
  long long c = t / per_cell;
  int local = int(t - c * per_cell);
  int ii = int(c % P.nx) + 2;
  int jj = int((c / P.nx) % P.ny) + 2;
  int kk = int(c / ((long long)P.nx * P.ny)) + 2;
  double x0 = P.Lx_min + P.dx * (ii - 2);
  double y0 = P.Ly_min + P.dy * (jj - 2);
  double z0 = P.Lz_min + P.dz * (kk - 2);
  uint32_t a = uint32_t(node_index(P, ii - 1, jj - 1, kk - 1));
  int ss, pp, m, sp;
  decode_group(P, G.p, local, ss, pp, m);
  double x[3], v[3];
  gen_member(P, kTagInit, 0u, a, ss, pp, m, x0, y0, z0, x, v, sp);
  store(start + t, x, v, sp);
}

struct StoreF64 {
  PartF64 o;
  __device__ void operator()(long long slot, const double x[3], const double v[3], int sp) const {
    store_f64(o, slot, x, v, sp);
  }
};
struct StoreC32 {
  KParams P;
  PartC32 o;
  __device__ void operator()(long long slot, const double x[3], const double v[3], int sp) const {
    store_c32(P, o, slot, x, v, sp);
  }
};

// Guard cell number g of the enumeration -> 1-based (ii, jj, kk) and the
// lower-edge coordinates of the cell (BCinflow.f90:56-61, 127-132, ...).
// Candidate indices of one BCinflow call are decoded in 32-bit arithmetic.
constexpr long long kMaxInflowCandidates = 0xFFFFFFFFLL;

// Guard cell g of the inflow enumeration; the launchers keep every candidate
// index (and so g) below 2^32, so the decode divides in 32 bits.
__device__ inline void inflow_cell(const KParams& P, const InflowTable& T, uint32_t g, int& ii, int& jj, int& kk,
                                   double& x0, double& y0, double& z0) {
  int f = 0;
  while (f < T.nfaces - 1 && (long long)g >= T.f[f + 1].first) ++f;
  const InflowFace& F = T.f[f];
  const uint32_t l = g - uint32_t(F.first), inner = uint32_t(F.i_n);
  const uint32_t lo = l / inner;
  int o = F.o_lo + int(lo);
  int in = F.i_lo + int(l - lo * inner);
  if (F.axis == 0) {  // outer kk, inner jj
    ii = F.fixed;
    kk = o;
    jj = in;
    x0 = F.edge;
    y0 = P.Ly_min + P.dy * (jj - 2);
    z0 = P.Lz_min + P.dz * (kk - 2);
  } else if (F.axis == 1) {  // outer kk, inner ii
    jj = F.fixed;
    kk = o;
    ii = in;
    x0 = P.Lx_min + P.dx * (ii - 2);
    y0 = F.edge;
    z0 = P.Lz_min + P.dz * (kk - 2);
  } else {  // outer jj, inner ii
    kk = F.fixed;
    jj = o;
    ii = in;
    x0 = P.Lx_min + P.dx * (ii - 2);
    y0 = P.Ly_min + P.dy * (jj - 2);
    z0 = F.edge;
  }
}

// BCinflow.f90:23-476 (append every candidate, reference order).
template <class Store>
__global__ void inflow_kernel(KParams P, InflowTable T, int iteration, long long start, long long total, Store store) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= total) return;
  const uint32_t tu = uint32_t(t), pc = uint32_t(T.per_cell), g = tu / pc;
  const int local = int(tu - g * pc);
  int ii, jj, kk;
  double x0, y0, z0;
  inflow_cell(P, T, g, ii, jj, kk, x0, y0, z0);
  uint32_t a = uint32_t(node_index(P, ii - 1, jj - 1, kk - 1));
  int ss, pp, m, sp;
  decode_group(P, T.group_prefix, local, ss, pp, m);
  double x[3], v[3];
  gen_member(P, kTagInflow, uint32_t(iteration), a, ss, pp, m, x0, y0, z0, x, v, sp);
  store(start + t, x, v, sp);
}

// BCoutflow.f90:28-66 predicate (true = keep).
__device__ inline bool outflow_keep(const KParams& P, double x, double y, double z) {
  bool del = false;
  if (P.xflow && (x < P.xmin || x > P.xmax)) del = true;
  if (P.yflow && (y < P.ymin || y > P.ymax)) del = true;
  if (P.zflow && (z < P.zmin || z > P.zmax)) del = true;
  if (x < 2.0 * P.Lx_min - P.Lx_max || x > 2.0 * P.Lx_max - P.Lx_min) del = true;
  if (y < 2.0 * P.Ly_min - P.Ly_max || y > 2.0 * P.Ly_max - P.Ly_min) del = true;
  if (z < 2.0 * P.Lz_min - P.Lz_max || z > 2.0 * P.Lz_max - P.Lz_min) del = true;
  return !del;
}

// ParticlesTransfer.f90:494-519
__device__ inline void transfer_wrap(const KParams& P, double& x, double& y, double& z) {
  const double Lx = P.xmax - P.xmin, Ly = P.ymax - P.ymin, Lz = P.zmax - P.zmin;
  if (z < P.zmin) z = z + Lz;
  if (z > P.zmax) z = z - Lz;
  if (y < P.ymin) y = y + Ly;
  if (y > P.ymax) y = y - Ly;
  if (x < P.xmin) x = x + Lx;
  if (x > P.xmax) x = x - Lx;
}

// Fast-path inflow: BCinflow + AdvancePosition + BCoutflow + ParticlesTransfer
// for the new candidates only.  Candidate t is generated, advanced by dt,
// tested and wrapped; true = it survives.
__device__ inline bool inflow_candidate(const KParams& P, const InflowTable& T, int iteration, long long t,
                                        double x[3], double v[3], int& sp) {
  const uint32_t tu = uint32_t(t), pc = uint32_t(T.per_cell), g = tu / pc;
  const int local = int(tu - g * pc);
  int ii, jj, kk;
  double x0, y0, z0;
  inflow_cell(P, T, g, ii, jj, kk, x0, y0, z0);
  uint32_t a = uint32_t(node_index(P, ii - 1, jj - 1, kk - 1));
  int ss, pp, m;
  decode_group(P, T.group_prefix, local, ss, pp, m);
  gen_member(P, kTagInflow, uint32_t(iteration), a, ss, pp, m, x0, y0, z0, x, v, sp);
  x[0] = x[0] + v[0] * P.dt;
  x[1] = x[1] + v[1] * P.dt;
  x[2] = x[2] + v[2] * P.dt;
  if (!outflow_keep(P, x[0], x[1], x[2])) return false;
  transfer_wrap(P, x[0], x[1], x[2]);
  return true;
}

// ------------------------------------------------------------- produce

// ParticlesProduce.f90:46-58: distance of the cell centre from the source,
// averaged over 8 sub-points when the cell is close to it.
__device__ void haser_radius(const KParams& P, double x0, double y0, double z0, double& r1, double& r2) {
  double xc = x0 + 0.5 * P.dx, yc = y0 + 0.5 * P.dy, zc = z0 + 0.5 * P.dz;
  r2 = xc * xc + yc * yc + zc * zc;
  r1 = sqrt(r2);
  double q = 4.0 * r1;
  if (q * q * q < P.dV) {
    const double fa[8][3] = {{0.25, 0.25, 0.25}, {0.25, 0.25, 0.75}, {0.25, 0.75, 0.25}, {0.75, 0.25, 0.25},
                             {0.25, 0.75, 0.75}, {0.75, 0.25, 0.75}, {0.75, 0.75, 0.25}, {0.75, 0.75, 0.75}};
    double s = 0.0;
    for (int t = 0; t < 8; ++t) {
      double a = x0 + fa[t][0] * P.dx, b = y0 + fa[t][1] * P.dy, c = z0 + fa[t][2] * P.dz;
      s = s + sqrt(a * a + b * b + c * c);
    }
    r1 = s * 0.125;
    r2 = r1 * r1;
  }
}

// ParticlesProduce.f90:62-73: number of ions of species ss created in cell a.
__device__ int produce_number(const KParams& P, int iteration, uint32_t a, int ss, double r1, double r2) {
  int s0 = ss - 1;
  double nden = 0.0;
  if (P.vn[s0] > 0.0) nden = P.Qn[s0] / (2.0 * kTau * r2 * P.vn[s0]) * exp(-P.nu_d[s0] * r1 / P.vn[s0]);
  if (!(P.n2p[s0] > 0.0)) return 0;
  Site r(P.seed, a, uint32_t(ss), uint32_t(iteration), kTagProduceCount);
  double rate = P.nu_i[s0] * nden * P.dV / P.n2p[s0];
  if (P.produce_dt_scaled) rate = rate * P.dt;
  return int(rate + r.u(0));
}

__device__ inline void interior_cell(const KParams& P, long long c, int& ii, int& jj, int& kk, double& x0,
                                     double& y0, double& z0) {
  ii = int(c % P.nx) + 2;
  jj = int((c / P.nx) % P.ny) + 2;
  kk = int(c / ((long long)P.nx * P.ny)) + 2;
  x0 = P.Lx_min + P.dx * (ii - 2);
  y0 = P.Ly_min + P.dy * (jj - 2);
  z0 = P.Lz_min + P.dz * (kk - 2);
}

__global__ void produce_count_kernel(KParams P, int iteration, int* counts) {
  long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  long long cells = (long long)P.nx * P.ny * P.nz;
  if (c >= cells) return;
  int ii, jj, kk;
  double x0, y0, z0, r1, r2;
  interior_cell(P, c, ii, jj, kk, x0, y0, z0);
  haser_radius(P, x0, y0, z0, r1, r2);
  uint32_t a = uint32_t(node_index(P, ii - 1, jj - 1, kk - 1));
  int total = 0;
  for (int ss = 1; ss <= P.species; ++ss) {
    int k = produce_number(P, iteration, a, ss, r1, r2);
    if (k > 0) total += k * (1 + P.epp[ss - 1] + P.hpp[ss - 1]);
  }
  counts[c] = total;
}

// ParticlesProduce.f90:75-103 for every ion of one cell, in (ss, pp) order.
template <class Store>
__global__ void produce_emit_kernel(KParams P, int iteration, const int* offsets, const int* count, long long capacity,
                                    int* err, Store store) {
  long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  long long cells = (long long)P.nx * P.ny * P.nz;
  if (c >= cells) return;
  const long long start = *count;
  int next = (c + 1 < cells) ? offsets[c + 1] : -1;
  int mine = offsets[c];
  if (next == mine) return;
  int ii, jj, kk;
  double x0, y0, z0, r1, r2;
  interior_cell(P, c, ii, jj, kk, x0, y0, z0);
  haser_radius(P, x0, y0, z0, r1, r2);
  uint32_t a = uint32_t(node_index(P, ii - 1, jj - 1, kk - 1));
  long long slot = start + mine;
  if (slot + ((next >= 0 ? next : offsets[cells]) - mine) > capacity) {
    atomicCAS(err, 0, int(kDevCapacity));
    return;
  }
  for (int ss = 1; ss <= P.species; ++ss) {
    int s0 = ss - 1;
    int k = produce_number(P, iteration, a, ss, r1, r2);
    for (int pp = 1; pp <= k; ++pp) {
      Site r(P.seed, a, (uint32_t(ss) << 24) | uint32_t(pp), uint32_t(iteration), kTagProduceParticle);
      double rnd[7];
      for (int q = 0; q < 7; ++q) rnd[q] = r.u(uint32_t(q));
      double xi[3], vi[3];
      xi[0] = x0 + P.dx * rnd[0];
      xi[1] = y0 + P.dy * rnd[1];
      xi[2] = z0 + P.dz * rnd[2];
      double rn = sqrt(xi[0] * xi[0] + xi[1] * xi[1] + xi[2] * xi[2]);
      double un = sqrt(rnd[3] * rnd[3] + rnd[4] * rnd[4] + rnd[5] * rnd[5]);
      for (int q = 0; q < 3; ++q) vi[q] = P.vn[s0] * xi[q] / rn + P.ui[s0] * rnd[3 + q] / un;
      for (int q = 0; q < 3; ++q) xi[q] = xi[q] + vi[q] * P.dt * rnd[6];
      store(slot++, xi, vi, s0);
      for (int ee = 1; ee <= P.epp[s0] + P.hpp[s0]; ++ee) {
        bool el = ee <= P.epp[s0];
        double u = el ? P.ue[s0] : P.uh[s0];
        double xe[3], vv[3];
        for (int q = 0; q < 3; ++q) vv[q] = vi[q] - (u + P.ui[s0]) * rnd[3 + q] / un;
        for (int q = 0; q < 3; ++q) xe[q] = xi[q] - vi[q] * P.dt * rnd[6] + vv[q] * P.dt * rnd[6];
        store(slot++, xe, vv, el ? 0 : 1);
      }
    }
  }
}

// ------------------------------------------------------ FP64 layout kernels

__global__ void advance_position_f64_kernel(PartF64 a, long long n, double dt) {
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
    a.x[p] = a.x[p] + a.vx[p] * dt;
    a.y[p] = a.y[p] + a.vy[p] * dt;
    a.z[p] = a.z[p] + a.vz[p] * dt;
  }
}

__global__ void transfer_f64_kernel(KParams P, PartF64 a, long long n) {
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
    double x = a.x[p], y = a.y[p], z = a.z[p];
    transfer_wrap(P, x, y, z);
    a.x[p] = x;
    a.y[p] = y;
    a.z[p] = z;
  }
}

// Exclusive scan of one int per thread over the block; total = the block's sum.
__device__ inline int block_exclusive_scan(int v, int* smem_warp, int& total) {
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) smem_warp[warp] = x;
  __syncthreads();
  if (warp == 0) {
    int w = (lane < (blockDim.x >> 5)) ? smem_warp[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    smem_warp[lane] = w;
  }
  __syncthreads();
  int warp_prefix = warp > 0 ? smem_warp[warp - 1] : 0;
  total = smem_warp[(blockDim.x >> 5) - 1];
  __syncthreads();
  return warp_prefix + x - v;
}

// BCoutflow.f90:28-66 and ParticlesTransfer.f90:494-519 on the FP64 layout,
// for the in-place removal of outflow.cuh.
struct OutflowF64 {
  KParams P;
  PartF64 a;
  using Key = double3;
  __device__ Key load_key(long long p) const { return make_double3(a.x[p], a.y[p], a.z[p]); }
  __device__ bool keep_wrap(long long p, double3 key, int wrap) const {
    const double x = key.x, y = key.y, z = key.z;
    if (!outflow_keep(P, x, y, z)) return false;
    if (wrap) {
      double wx = x, wy = y, wz = z;
      transfer_wrap(P, wx, wy, wz);
      if (wx != x || wy != y || wz != z) {
        a.x[p] = wx;
        a.y[p] = wy;
        a.z[p] = wz;
      }
    }
    return true;
  }
  __device__ void move(long long d, long long s) const {
    a.x[d] = a.x[s];
    a.y[d] = a.y[s];
    a.z[d] = a.z[s];
    a.vx[d] = a.vx[s];
    a.vy[d] = a.vy[s];
    a.vz[d] = a.vz[s];
    a.sp[d] = a.sp[s];
  }
};

// The fused inflow in two passes, so that survivors land in candidate order
// (deterministic): per-block survivor counts, an exclusive scan, then every
// block regenerates its candidates and stores the survivors at *count + its
// offset + their rank in the block.
__global__ void __launch_bounds__(kThreads) inflow_count_kernel(KParams P, InflowTable T, int iteration,
                                                                long long total, int* block_counts) {
  __shared__ int warp_sums[32];
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  double x[3], v[3];
  int sp = 0;
  const bool keep = t < total && inflow_candidate(P, T, iteration, t, x, v, sp);
  int sum;
  block_exclusive_scan(keep ? 1 : 0, warp_sums, sum);
  if (threadIdx.x == 0) block_counts[blockIdx.x] = sum;
}

template <class Store>
__global__ void __launch_bounds__(kThreads) inflow_emit_kernel(KParams P, InflowTable T, int iteration,
                                                               long long total, const int* offsets, const int* count,
                                                               long long capacity, int* err, Store store) {
  __shared__ int warp_sums[32];
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  double x[3], v[3];
  int sp = 0;
  const bool keep = t < total && inflow_candidate(P, T, iteration, t, x, v, sp);
  int sum;
  const int rank = block_exclusive_scan(keep ? 1 : 0, warp_sums, sum);
  if (keep) {
    const long long slot = (long long)*count + offsets[blockIdx.x] + rank;
    if (slot < capacity)
      store(slot, x, v, sp);
    else
      atomicCAS(err, 0, int(kDevCapacity));
  }
}

// The fused inflow in one generation: every block generates its candidates
// once and writes its survivors, in candidate order, to its own stretch of a
// staging area (FP64 position and velocity, species); after the scan of the
// block counts, the place pass stores them at *count + the block's offset +
// their rank -- the same slots and values as count + emit.
__global__ void __launch_bounds__(kThreads) inflow_stage_kernel(KParams P, InflowTable T, int iteration,
                                                                long long total, int* block_counts, double* stage,
                                                                int8_t* stage_sp, long long stride) {
  __shared__ int warp_sums[32];
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  double x[3], v[3];
  int sp = 0;
  const bool keep = t < total && inflow_candidate(P, T, iteration, t, x, v, sp);
  int sum;
  const int rank = block_exclusive_scan(keep ? 1 : 0, warp_sums, sum);
  if (keep) {
    const long long q = (long long)blockIdx.x * blockDim.x + rank;
    stage[q] = x[0];
    stage[q + stride] = x[1];
    stage[q + 2 * stride] = x[2];
    stage[q + 3 * stride] = v[0];
    stage[q + 4 * stride] = v[1];
    stage[q + 5 * stride] = v[2];
    stage_sp[q] = int8_t(sp);
  }
  if (threadIdx.x == 0) block_counts[blockIdx.x] = sum;
}

template <class Store>
__global__ void __launch_bounds__(kThreads) inflow_place_kernel(const int* block_counts, const int* offsets,
                                                                const int* count, long long capacity, int* err,
                                                                const double* stage, const int8_t* stage_sp,
                                                                long long stride, Store store) {
  const int r = threadIdx.x;
  if (r >= block_counts[blockIdx.x]) return;
  const long long q = (long long)blockIdx.x * blockDim.x + r;
  const double x[3] = {stage[q], stage[q + stride], stage[q + 2 * stride]};
  const double v[3] = {stage[q + 3 * stride], stage[q + 4 * stride], stage[q + 5 * stride]};
  const long long slot = (long long)*count + offsets[blockIdx.x] + r;
  if (slot < capacity)
    store(slot, x, v, int(stage_sp[q]));
  else
    atomicCAS(err, 0, int(kDevCapacity));
}

// CIC weights of ParticlesGridify.f90:70-88 (F1..F8 before the 1/dV).
struct Cic64 {
  int i, j, k;  // 0-based base node
  double F[8];
};

__device__ inline void cic64(const KParams& P, double x, double y, double z, Cic64& w) {
  double rest0 = fmod(x - P.Lx_min + 0.5 * P.dx, P.dx);
  double rest1 = fmod(y - P.Ly_min + 0.5 * P.dy, P.dy);
  double rest2 = fmod(z - P.Lz_min + 0.5 * P.dz, P.dz);
  double d0 = P.dx - rest0, d1 = P.dy - rest1, d2 = P.dz - rest2;
  w.i = int((x - P.Lx_min) / P.dx + 0.5);
  w.j = int((y - P.Ly_min) / P.dy + 0.5);
  w.k = int((z - P.Lz_min) / P.dz + 0.5);
  w.F[0] = d0 * d1 * d2;
  w.F[1] = rest0 * d1 * d2;
  w.F[2] = d0 * rest1 * d2;
  w.F[3] = d0 * d1 * rest2;
  w.F[4] = rest0 * rest1 * d2;
  w.F[5] = d0 * rest1 * rest2;
  w.F[6] = rest0 * d1 * rest2;
  w.F[7] = rest0 * rest1 * rest2;
}

__constant__ int kOff[8][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {1, 1, 0}, {0, 1, 1}, {1, 0, 1}, {1, 1, 1}};

__device__ inline int clamp_gather(int i, int n) { return i < 0 ? 0 : (i > n + 1 ? n + 1 : i); }

// AdvanceVelocity.f90:39-121 (mode 0), AdvanceVelocityExp (mode 1),
// AdvanceVelocityImp (mode 2).  E is three planes (Ex, Ey, Ez) of nodes.
__global__ void advance_velocity_f64_kernel(KParams P, PartF64 a, long long n, const double* __restrict__ E,
                                            double dt, double deltat, int mode) {
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
    Cic64 w;
    cic64(P, a.x[p], a.y[p], a.z[p], w);
    double Ep[3];
    for (int c = 0; c < 3; ++c) {
      const double* Ec = E + (long long)c * P.nodes;
      double s = 0.0;
      for (int q = 0; q < 8; ++q) {
        int i = clamp_gather(w.i + kOff[q][0], P.nx), j = clamp_gather(w.j + kOff[q][1], P.ny),
            k = clamp_gather(w.k + kOff[q][2], P.nz);
        double e = Ec[node_index(P, i, j, k)];
        s = (q == 0) ? e * w.F[0] : s + e * w.F[q];
      }
      Ep[c] = s / P.dV;
    }
    int s = a.sp[p];
    double v[3] = {a.vx[p], a.vy[p], a.vz[p]};
    if (P.fluid[s]) {
      if (P.gyration[s]) {
        const double* B = P.B0;
        double vb = v[0] * B[0] + v[1] * B[1] + v[2] * B[2];
        double vm[3], vd[3];
        for (int c = 0; c < 3; ++c) vm[c] = vb * B[c];
        vd[0] = vm[0] + (Ep[1] * B[2] - Ep[2] * B[1]);
        vd[1] = vm[1] + (Ep[2] * B[0] - Ep[0] * B[2]);
        vd[2] = vm[2] + (Ep[0] * B[1] - Ep[1] * B[0]);
        double ib = 1.0 / (B[0] * B[0] + B[1] * B[1] + B[2] * B[2]);
        a.vx[p] = vd[0] * ib;
        a.vy[p] = vd[1] * ib;
        a.vz[p] = vd[2] * ib;
      }
      continue;
    }
    double etadt2, tB[3];
    if (mode == 0) {
      etadt2 = 0.5 * dt * P.eta[s];
      for (int c = 0; c < 3; ++c) tB[c] = P.tB[s][c];
    } else {
      etadt2 = 0.5 * dt * P.eta[s] * 2.0 * deltat / dt;
      for (int c = 0; c < 3; ++c) tB[c] = P.tB[s][c] * 2.0 * deltat / dt;
    }
    double vmin[3], vmid[3];
    if (mode == 0) {
      const double* sB = P.sB[s];
      double vplus[3];
      for (int c = 0; c < 3; ++c) vmin[c] = v[c] - P.ve[c] + etadt2 * Ep[c];
      vmid[0] = vmin[0] + vmin[1] * tB[2] - vmin[2] * tB[1];
      vmid[1] = vmin[1] + vmin[2] * tB[0] - vmin[0] * tB[2];
      vmid[2] = vmin[2] + vmin[0] * tB[1] - vmin[1] * tB[0];
      vplus[0] = vmin[0] + vmid[1] * sB[2] - vmid[2] * sB[1];
      vplus[1] = vmin[1] + vmid[2] * sB[0] - vmid[0] * sB[2];
      vplus[2] = vmin[2] + vmid[0] * sB[1] - vmid[1] * sB[0];
      for (int c = 0; c < 3; ++c) v[c] = vplus[c] + P.ve[c] + etadt2 * Ep[c];
    } else {
      if (mode == 1)
        for (int c = 0; c < 3; ++c) vmin[c] = v[c] - P.ve[c];
      else
        for (int c = 0; c < 3; ++c) vmin[c] = v[c] - P.ve[c] + etadt2 * Ep[c];
      vmid[0] = vmin[0] + vmin[1] * tB[2] - vmin[2] * tB[1];
      vmid[1] = vmin[1] + vmin[2] * tB[0] - vmin[0] * tB[2];
      vmid[2] = vmin[2] + vmin[0] * tB[1] - vmin[1] * tB[0];
      double smid = vmid[0] * vmid[0] + vmid[1] * vmid[1] + vmid[2] * vmid[2];
      if (smid > 0.0) {
        double smin = vmin[0] * vmin[0] + vmin[1] * vmin[1] + vmin[2] * vmin[2];
        double f = sqrt(smin / smid);
        for (int c = 0; c < 3; ++c) vmid[c] = vmid[c] * f;
      }
      if (mode == 1)
        for (int c = 0; c < 3; ++c) v[c] = vmid[c] + P.ve[c] + etadt2 * Ep[c];
      else
        for (int c = 0; c < 3; ++c) v[c] = vmid[c] + P.ve[c];
    }
    a.vx[p] = v[0];
    a.vy[p] = v[1];
    a.vz[p] = v[2];
  }
}

// Deposit index of node i on an axis of n cells: open axes fold the ghost
// layers onto the first / last interior node (ParticlesGridify.f90:149-171),
// periodic axes fold them onto the opposite interior node (ibid. 167-170).
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

// Warp-aggregated fixed-point deposit of 8 weights (each in [0, 2^40]) at
// the nodes of `key`'s stencil.  Lanes with equal keys are summed with
// 32-bit warp reductions of the weights split at bit 18, then one lane per
// group issues the 8 atomics.
__device__ inline void deposit8(unsigned long long key, bool active, const long long w[8], const long long nodes[8],
                                unsigned long long* plane) {
  unsigned act = __ballot_sync(0xffffffffu, active);
  if (!active) return;
  unsigned grp = __match_any_sync(act, key);
  int lane = threadIdx.x & 31;
  int leader = __ffs(grp) - 1;
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    long long v = w[q];
    // Weights are in [-2^40, 2^40]; bias them into [0, 2^41] for the split.
    unsigned long long u = (unsigned long long)(v + (1LL << kDepositShift));
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

// Grouping key of a particle's stencil: base node (offset by 2, 20 bits per
// axis) and species.
__device__ inline unsigned long long stencil_key(int i, int j, int k, int s) {
  auto c = [](int v) { v += 2; return (unsigned long long)(v < 0 ? 0 : (v > 0xFFFFF ? 0xFFFFF : v)); };
  return (c(i) | (c(j) << 20) | (c(k) << 40)) << 4 | (unsigned long long)s;
}

__global__ void deposit_f64_kernel(KParams P, PartF64 a, long long n, unsigned long long* Nacc,
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
      Cic64 c;
      cic64(P, a.x[p], a.y[p], a.z[p], c);
      s = a.sp[p];
      for (int q = 0; q < 8; ++q) {
        Fw[q] = c.F[q] / P.dV;
        w[q] = __double2ll_rn(Fw[q] * kDepositScale);
        int i = fold_index(c.i + kOff[q][0], P.nx, P.xflow), j = fold_index(c.j + kOff[q][1], P.ny, P.yflow),
            k = fold_index(c.k + kOff[q][2], P.nz, P.zflow);
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

// Block partial sums of sum(n2p*mass*|v|^2) (picard.f90:661-664).
__global__ void energy_particles_f64_kernel(KParams P, PartF64 a, long long n, double* partial) {
  __shared__ double sh[32];
  double acc = 0.0;
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
    int s = a.sp[p];
    double v2 = a.vx[p] * a.vx[p] + a.vy[p] * a.vy[p] + a.vz[p] * a.vz[p];
    acc += P.n2p[s] * P.mass[s] * v2;
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

__global__ void cell_indices_f64_kernel(KParams P, PartF64 a, long long n, int* ijk) {
  long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  ijk[3 * p + 0] = 1 + int((a.x[p] - P.Lx_min) / P.dx + 0.5);
  ijk[3 * p + 1] = 1 + int((a.y[p] - P.Ly_min) / P.dy + 0.5);
  ijk[3 * p + 2] = 1 + int((a.z[p] - P.Lz_min) / P.dz + 0.5);
}

// CalcDistance.f90:28-87 (one thread per (ii, jj, kk) of the positive octant).
__global__ void calc_distance_kernel(KParams P, double* D) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int Nx = P.nx, Ny = P.ny, Nz = P.nz;
  long long total = (long long)(Nx + 1) * (Ny + 1) * (Nz + 1);
  if (t >= total) return;
  int ii = int(t % (Nx + 1)) + 1, jj = int((t / (Nx + 1)) % (Ny + 1)) + 1, kk = int(t / ((long long)(Nx + 1) * (Ny + 1))) + 1;
  const long long DX = 2 * Nx + 1, DY = 2 * Ny + 1;
  double di = double(ii - 1), dj = double(jj - 1), dk = double(kk - 1);
  double a = di * P.dx, b = dj * P.dy, c = dk * P.dz;
  double an = (Nx - di) * P.dx, bn = (Ny - dj) * P.dy, cn = (Nz - dk) * P.dz;
  auto inv = [](double x, double y, double z) { return 1.0 / sqrt(x * x + y * y + z * z); };
  double t0 = (ii == 1 && jj == 1 && kk == 1) ? 0.0 : inv(a, b, c);
  const int xf = P.xflow != 0, yf = P.yflow != 0, zf = P.zflow != 0;
  if (xf) {
    if (!yf && !zf) {
      t0 = t0 + inv(a, bn, c);
      t0 = t0 + inv(a, b, cn);
      t0 = t0 + inv(a, bn, cn);
    } else if (!yf) {
      t0 = t0 + inv(a, bn, c);
    } else if (!zf) {
      t0 = t0 + inv(a, b, cn);
    }
  } else if (yf) {
    if (!zf) {
      t0 = t0 + inv(an, b, c);
      t0 = t0 + inv(a, b, cn);
      t0 = t0 + inv(an, b, cn);
    } else {
      t0 = t0 + inv(an, b, c);
    }
  } else if (zf) {
    t0 = t0 + inv(an, b, c);
    t0 = t0 + inv(a, bn, c);
    t0 = t0 + inv(an, bn, c);
  } else {
    t0 = t0 + inv(an, b, c);
    t0 = t0 + inv(a, bn, c);
    t0 = t0 + inv(a, b, cn);
    t0 = t0 + inv(an, bn, c);
    t0 = t0 + inv(a, bn, cn);
    t0 = t0 + inv(an, b, cn);
    t0 = t0 + inv(an, bn, cn);
  }
  int pi = Nx + 1 + (ii - 1), pj = Ny + 1 + (jj - 1), pk = Nz + 1 + (kk - 1);
  int ni = Nx + 1 - (ii - 1), nj = Ny + 1 - (jj - 1), nk = Nz + 1 - (kk - 1);
  auto at = [&](int i, int j, int k) { return (long long)(i - 1) + DX * ((long long)(j - 1) + DY * (long long)(k - 1)); };
  D[at(pi, pj, pk)] = t0;
  D[at(ni, pj, pk)] = t0;
  D[at(pi, nj, pk)] = t0;
  D[at(pi, pj, nk)] = t0;
  D[at(ni, nj, pk)] = t0;
  D[at(pi, nj, nk)] = t0;
  D[at(ni, pj, nk)] = t0;
  D[at(ni, nj, nk)] = t0;
}

// CELL32 -> FP64 positions: x = Lx_min + (i + f/2^32 - 0.5) dx.
__global__ void c32_to_f64_kernel(KParams P, PartC32 a, long long n, PartF64 o) {
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    unpack_cell(a.cell[p], i, j, k);
    o.x[p] = P.Lx_min + ((double)i + off_f64(a.fx[p]) - 0.5) * P.dx;
    o.y[p] = P.Ly_min + ((double)j + off_f64(a.fy[p]) - 0.5) * P.dy;
    o.z[p] = P.Lz_min + ((double)k + off_f64(a.fz[p]) - 0.5) * P.dz;
    o.vx[p] = a.vx[p];
    o.vy[p] = a.vy[p];
    o.vz[p] = a.vz[p];
    o.sp[p] = a.sp[p];
  }
}

__global__ void f64_to_c32_kernel(KParams P, PartF64 a, long long n, PartC32 o) {
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
    double x[3] = {a.x[p], a.y[p], a.z[p]};
    double v[3] = {a.vx[p], a.vy[p], a.vz[p]};
    store_c32(P, o, p, x, v, a.sp[p]);
  }
}

}  // namespace

int compact_blocks(long long n) { return int((n + kOutflowTile - 1) / kOutflowTile); }

int inflow_blocks(long long candidates) { return grid_for(candidates); }

cudaError_t launch_calc_distance(const KParams& P, double* D, cudaStream_t st) {
  long long total = (long long)(P.nx + 1) * (P.ny + 1) * (P.nz + 1);
  note_launch();
  calc_distance_kernel<<<grid_for(total), kThreads, 0, st>>>(P, D);
  return cudaGetLastError();
}

cudaError_t launch_init_f64(const KParams& P, PartF64 out, long long start, cudaStream_t st) {
  GroupPrefix G = group_prefix(P);
  long long total = (long long)P.nx * P.ny * P.nz * G.p[P.species];
  if (total == 0) return cudaSuccess;
  note_launch();
  init_kernel<<<grid_for(total), kThreads, 0, st>>>(P, G, start, total, StoreF64{out});
  return cudaGetLastError();
}

cudaError_t launch_init_c32(const KParams& P, PartC32 out, long long start, cudaStream_t st) {
  GroupPrefix G = group_prefix(P);
  long long total = (long long)P.nx * P.ny * P.nz * G.p[P.species];
  if (total == 0) return cudaSuccess;
  note_launch();
  init_kernel<<<grid_for(total), kThreads, 0, st>>>(P, G, start, total, StoreC32{P, out});
  return cudaGetLastError();
}

cudaError_t launch_inflow_f64(const KParams& P, const InflowTable& T, int iteration, PartF64 out, long long start,
                              cudaStream_t st) {
  long long total = T.cells * T.per_cell;
  if (total == 0) return cudaSuccess;
  if (total > kMaxInflowCandidates) return cudaErrorInvalidValue;
  note_launch();
  inflow_kernel<<<grid_for(total), kThreads, 0, st>>>(P, T, iteration, start, total, StoreF64{out});
  return cudaGetLastError();
}

cudaError_t launch_inflow_c32(const KParams& P, const InflowTable& T, int iteration, PartC32 out, long long start,
                              cudaStream_t st) {
  long long total = T.cells * T.per_cell;
  if (total == 0) return cudaSuccess;
  if (total > kMaxInflowCandidates) return cudaErrorInvalidValue;
  note_launch();
  inflow_kernel<<<grid_for(total), kThreads, 0, st>>>(P, T, iteration, start, total, StoreC32{P, out});
  return cudaGetLastError();
}

cudaError_t launch_produce_count(const KParams& P, int iteration, int* counts, cudaStream_t st) {
  long long cells = (long long)P.nx * P.ny * P.nz;
  note_launch();
  produce_count_kernel<<<grid_for(cells), kThreads, 0, st>>>(P, iteration, counts);
  return cudaGetLastError();
}

__global__ void add_count_kernel(int* count, const int* add, long long capacity) {
  long long v = (long long)*count + *add;
  *count = int(v < capacity ? v : capacity);
}

template <class Store>
static cudaError_t inflow_fused(const KParams& P, const InflowTable& T, int iteration, Store store, int* count,
                                long long capacity, int* block_counts, int* block_offsets, int* err,
                                const InflowStage& S, cudaStream_t st) {
  const long long total = T.cells * T.per_cell;
  if (total == 0) return cudaSuccess;
  if (total > kMaxInflowCandidates) return cudaErrorInvalidValue;
  const int nb = inflow_blocks(total);
  cudaError_t e;
  if (S.x) {
    const long long stride = (long long)nb * kThreads;
    note_launch();
    inflow_stage_kernel<<<nb, kThreads, 0, st>>>(P, T, iteration, total, block_counts, S.x, S.sp, stride);
    e = launch_scan_int(block_counts, block_offsets, nb, block_offsets + nb, block_offsets + nb + 1, st);
    if (e != cudaSuccess) return e;
    note_launch();
    inflow_place_kernel<<<nb, kThreads, 0, st>>>(block_counts, block_offsets, count, capacity, err, S.x, S.sp, stride,
                                                 store);
    note_launch();
    add_count_kernel<<<1, 1, 0, st>>>(count, block_offsets + nb, capacity);
    return cudaGetLastError();
  }
  note_launch();
  inflow_count_kernel<<<nb, kThreads, 0, st>>>(P, T, iteration, total, block_counts);
  e = launch_scan_int(block_counts, block_offsets, nb, block_offsets + nb, block_offsets + nb + 1, st);
  if (e != cudaSuccess) return e;
  note_launch();
  inflow_emit_kernel<<<nb, kThreads, 0, st>>>(P, T, iteration, total, block_offsets, count, capacity, err, store);
  note_launch();
  add_count_kernel<<<1, 1, 0, st>>>(count, block_offsets + nb, capacity);
  return cudaGetLastError();
}

cudaError_t launch_inflow_fused_c32(const KParams& P, const InflowTable& T, int iteration, PartC32 out, int* count,
                                    long long capacity, int* block_counts, int* block_offsets, int* err,
                                    const InflowStage& stage, cudaStream_t st) {
  return inflow_fused(P, T, iteration, StoreC32{P, out}, count, capacity, block_counts, block_offsets, err, stage,
                      st);
}

cudaError_t launch_inflow_fused_f64(const KParams& P, const InflowTable& T, int iteration, PartF64 out, int* count,
                                    long long capacity, int* block_counts, int* block_offsets, int* err,
                                    const InflowStage& stage, cudaStream_t st) {
  return inflow_fused(P, T, iteration, StoreF64{out}, count, capacity, block_counts, block_offsets, err, stage, st);
}

long long inflow_stage_slots(long long candidates) { return (long long)inflow_blocks(candidates) * kThreads; }

cudaError_t launch_produce_emit_f64(const KParams& P, int iteration, const int* offsets, PartF64 out, int* count,
                                    long long capacity, int* err, cudaStream_t st) {
  long long cells = (long long)P.nx * P.ny * P.nz;
  note_launch();
  produce_emit_kernel<<<grid_for(cells), kThreads, 0, st>>>(P, iteration, offsets, count, capacity, err,
                                                            StoreF64{out});
  note_launch();
  add_count_kernel<<<1, 1, 0, st>>>(count, offsets + cells, capacity);
  return cudaGetLastError();
}

cudaError_t launch_produce_emit_c32(const KParams& P, int iteration, const int* offsets, PartC32 out, int* count,
                                    long long capacity, int* err, cudaStream_t st) {
  long long cells = (long long)P.nx * P.ny * P.nz;
  note_launch();
  produce_emit_kernel<<<grid_for(cells), kThreads, 0, st>>>(P, iteration, offsets, count, capacity, err,
                                                            StoreC32{P, out});
  note_launch();
  add_count_kernel<<<1, 1, 0, st>>>(count, offsets + cells, capacity);
  return cudaGetLastError();
}

static int persistent_grid(long long n) {
  long long b = (n + kThreads - 1) / kThreads;
  if (b > 148LL * 16) b = 148LL * 16;
  return b < 1 ? 1 : int(b);
}

cudaError_t launch_advance_position_f64(const KParams& P, PartF64 a, long long n, double dt, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  note_launch();
  advance_position_f64_kernel<<<persistent_grid(n), kThreads, 0, st>>>(a, n, dt);
  return cudaGetLastError();
}

cudaError_t launch_transfer_f64(const KParams& P, PartF64 a, long long n, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  note_launch();
  transfer_f64_kernel<<<persistent_grid(n), kThreads, 0, st>>>(P, a, n);
  return cudaGetLastError();
}

cudaError_t launch_outflow_f64(const KParams& P, PartF64 a, long long n, uint2* words, int* block_counts,
                               int* block_offsets, int* count, int wrap, int* err, cudaStream_t st,
                               const OutflowSplit* split) {
  return launch_outflow_inplace(OutflowF64{P, a}, n, words, block_counts, block_offsets, count, wrap, err, st, split);
}

cudaError_t launch_advance_velocity_f64(const KParams& P, PartF64 a, long long n, const double* E, double dt,
                                        double deltat, int mode, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  note_launch();
  advance_velocity_f64_kernel<<<persistent_grid(n), kThreads, 0, st>>>(P, a, n, E, dt, deltat, mode);
  return cudaGetLastError();
}

cudaError_t launch_deposit_f64(const KParams& P, PartF64 a, long long n, unsigned long long* Nacc,
                               unsigned long long* Facc, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  note_launch();
  deposit_f64_kernel<<<persistent_grid(n), kThreads, 0, st>>>(P, a, n, Nacc, Facc);
  return cudaGetLastError();
}

cudaError_t launch_energy_particles_f64(const KParams& P, PartF64 a, long long n, ReduceBuf rb, cudaStream_t st) {
  int nb = persistent_grid(n > 0 ? n : 1);
  if (nb > rb.max_blocks) nb = rb.max_blocks;
  note_launch();
  energy_particles_f64_kernel<<<nb, kThreads, 0, st>>>(P, a, n, rb.partial);
  note_launch();
  finish_sum_kernel<<<1, 32, 0, st>>>(rb.partial, nb, 0.5, rb.result);
  return cudaGetLastError();
}

cudaError_t launch_cell_indices_f64(const KParams& P, PartF64 a, long long n, int* ijk, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  note_launch();
  cell_indices_f64_kernel<<<grid_for(n), kThreads, 0, st>>>(P, a, n, ijk);
  return cudaGetLastError();
}

}  // namespace picard

namespace picard {
cudaError_t launch_c32_to_f64(const KParams& P, PartC32 a, long long n, PartF64 out, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  note_launch();
  c32_to_f64_kernel<<<persistent_grid(n), kThreads, 0, st>>>(P, a, n, out);
  return cudaGetLastError();
}
cudaError_t launch_f64_to_c32(const KParams& P, PartF64 a, long long n, PartC32 out, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  note_launch();
  f64_to_c32_kernel<<<persistent_grid(n), kThreads, 0, st>>>(P, a, n, out);
  return cudaGetLastError();
}
}  // namespace picard

// ---------------------------------------------------------------------------
// Allocation-free deposit: picard_gpu_particles_gridify_noalloc.
//
// Some callers cannot allocate device memory at the point where they need a
// charge deposit: a host whose device memory is owned by another runtime's
// fixed pool (a Fortran program that manages its arrays through OpenACC or
// CUDA Fortran data regions), a serving loop that has already promised all of
// the HBM to resident runs, or a pipeline that cannot afford the device-wide
// synchronisation cudaFree implies.  For them this entry point takes the
// particle arrays and the output grids from the caller and keeps its only
// scratch -- the int64 fixed-point accumulators -- in the file-scope array
// below, so it calls no cudaMalloc, cudaFree or allocating library routine.
#include <string>

namespace picard {
KParams make_kparams(const picard_params& p);
int fail(int code, const std::string& msg);

namespace {

// Every device that loads the library holds this array (16 MiB) until the
// process exits.  All calls share it, so calls that overlap on the GPU race.
static __device__ __align__(256) unsigned long long g_noalloc_acc[PICARD_NOALLOC_MAX_WORDS];

// True when x lies within half a cell of [L_min, L_max] (NaN: false).  There
// the CIC base node is 0 .. n and both stencil nodes lie inside the
// ghost-padded box, with non-negative weights.  The reference deposits after
// BCoutflow and ParticlesTransfer, which leave every particle inside
// [min, max], so its particles always pass.
__device__ inline bool within_half_cell(double x, double lo, double hi, double d) {
  return x >= lo - 0.5 * d && x < hi + 0.5 * d;
}

// ParticlesGridify.f90:65-123 for caller-owned FP64 arrays; int_particles
// holds the reference's 1-based species numbers.  Particles of another
// species number, or farther than half a cell outside the domain on some
// axis, are not deposited.
__global__ void deposit_noalloc_kernel(KParams P, const double* __restrict__ x, const double* __restrict__ y,
                                       const double* __restrict__ z, const int32_t* __restrict__ sp1, long long n,
                                       unsigned long long* acc) {
  long long stride = (long long)gridDim.x * blockDim.x;
  long long n_round = ((n + 31) / 32) * 32;
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n_round; p += stride) {
    int s = (p < n) ? sp1[p] - 1 : -1;
    bool active = s >= 0 && s < P.species;
    double xp = 0.0, yp = 0.0, zp = 0.0;
    if (active) {
      xp = x[p];
      yp = y[p];
      zp = z[p];
      active = within_half_cell(xp, P.Lx_min, P.Lx_max, P.dx) && within_half_cell(yp, P.Ly_min, P.Ly_max, P.dy) &&
               within_half_cell(zp, P.Lz_min, P.Lz_max, P.dz);
    }
    long long w[8] = {0, 0, 0, 0, 0, 0, 0, 0}, nodes[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    unsigned long long key = ~0ull;
    if (active) {
      Cic64 c;
      cic64(P, xp, yp, zp, c);
      for (int q = 0; q < 8; ++q) {
        w[q] = __double2ll_rn(c.F[q] / P.dV * kDepositScale);
        int i = fold_index(c.i + kOff[q][0], P.nx, P.xflow), j = fold_index(c.j + kOff[q][1], P.ny, P.yflow),
            k = fold_index(c.k + kOff[q][2], P.nz, P.zflow);
        nodes[q] = node_index(P, i, j, k);
      }
      key = stencil_key(c.i, c.j, c.k, s);
    } else {
      s = 0;
    }
    deposit8(key, active, w, nodes, acc + (long long)s * P.nodes);
  }
}

// N(s, node) = n2p_s * acc * 2^-40 in the reference layout (species fastest),
// with the ghost folds of ParticlesGridify.f90:149-278; C = sum_s q_s N_s.
__global__ void finish_noalloc_kernel(KParams P, const unsigned long long* acc, double* N, double* C) {
  long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= P.nodes) return;
  int i = int(g % P.nxp), j = int((g / P.nxp) % P.nyp), k = int(g / ((long long)P.nxp * P.nyp));
  auto mirror = [](int v, int nn, int open) { return (v >= 1 && v <= nn) ? v : (open ? -1 : (v < 1 ? v + nn : v - nn)); };
  int mi = mirror(i, P.nx, P.xflow), mj = mirror(j, P.ny, P.yflow), mk = mirror(k, P.nz, P.zflow);
  double c = 0.0;
  for (int s = 0; s < P.species; ++s) {
    double v = 0.0;
    if (mi >= 0 && mj >= 0 && mk >= 0) {
      long long a = (long long)acc[(long long)s * P.nodes + node_index(P, mi, mj, mk)];
      v = P.n2p[s] * ((double)a * (1.0 / kDepositScale));
    }
    N[(long long)s + (long long)P.species * g] = v;
    c = c + v * P.charge[s];
  }
  C[g] = c;
}

}  // namespace
}  // namespace picard

extern "C" int picard_gpu_particles_gridify_noalloc(const picard_params* p, const double* x, const double* y,
                                                    const double* z, const int32_t* int_particles, int32_t num_local,
                                                    double* N, double* C, void* stream) {
  using namespace picard;
  if (!p) return fail(PICARD_ERR_BAD_ARG, "params is NULL");
  if (!(p->dxyz[0] > 0.0 && p->dxyz[1] > 0.0 && p->dxyz[2] > 0.0))
    return fail(PICARD_ERR_BAD_ARG, "params not derived (call picard_params_derive first)");
  if (p->species < 2 || p->species > 8) return fail(PICARD_ERR_BAD_ARG, "species must be in 2..8");
  if (p->nx < 1 || p->ny < 1 || p->nz < 1) return fail(PICARD_ERR_BAD_ARG, "grid dimensions must be positive");
  const long long nodes = (long long)(p->nx + 2) * (p->ny + 2) * (p->nz + 2);
  const long long words = nodes * p->species;
  if (words > (long long)PICARD_NOALLOC_MAX_WORDS)
    return fail(PICARD_ERR_BAD_ARG, "the allocation-free deposit needs species*(Nx+2)*(Ny+2)*(Nz+2) = " +
                                        std::to_string(words) + " accumulator words; its fixed scratch holds " +
                                        std::to_string((long long)PICARD_NOALLOC_MAX_WORDS));
  if (num_local < 0) return fail(PICARD_ERR_BAD_ARG, "num_local must be >= 0");
  if (num_local > 0 && (!x || !y || !z || !int_particles)) return fail(PICARD_ERR_BAD_ARG, "particle array is NULL");
  if (!N || !C) return fail(PICARD_ERR_BAD_ARG, "output array is NULL");
  // The array's host-side name is not a device address.  Its address on the
  // current device is looked up on every call (a table lookup once the
  // library's device code is loaded), so nothing cached outlives a
  // cudaDeviceReset.  The first call on a device loads that code: make it
  // before any stream capture.
  void* q = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&q, g_noalloc_acc);
  if (e != cudaSuccess) return fail(PICARD_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
  unsigned long long* acc = static_cast<unsigned long long*>(q);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const KParams K = make_kparams(*p);
  // the array keeps the previous call's sums: clear the part this call uses
  e = cudaMemsetAsync(acc, 0, sizeof(unsigned long long) * (size_t)words, st);
  if (e != cudaSuccess) return fail(PICARD_ERR_CUDA, std::string("cudaMemsetAsync: ") + cudaGetErrorString(e));
  if (num_local > 0) {
    note_launch();
    deposit_noalloc_kernel<<<persistent_grid(num_local), kThreads, 0, st>>>(K, x, y, z, int_particles, num_local,
                                                                             acc);
  }
  note_launch();
  finish_noalloc_kernel<<<grid_for(nodes), kThreads, 0, st>>>(K, acc, N, C);
  e = cudaGetLastError();
  if (e != cudaSuccess) return fail(PICARD_ERR_CUDA, std::string("deposit launch: ") + cudaGetErrorString(e));
  return PICARD_OK;
}
