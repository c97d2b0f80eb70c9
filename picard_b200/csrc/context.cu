// context.cu -- the C ABI of include/picard_gpu.h: context life cycle,
// transfers in the reference layouts, and one entry point per reference
// subroutine (each cites the routine it replaces).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "context.cuh"
#include "picard_gpu.h"

using namespace picard;

#include <atomic>

namespace picard {

static thread_local std::string g_last_error;
static std::atomic<long long> g_launches{0};

void note_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
long long launches_so_far() { return g_launches.load(std::memory_order_relaxed); }

int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

int check_cuda(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return PICARD_OK;
  // reported here: clear the runtime's last-error slot so that a later,
  // unrelated launch check does not report it again (sticky errors stay)
  (void)cudaGetLastError();
  return fail(PICARD_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

KParams make_kparams(const picard_params& p) {
  KParams K;
  std::memset(&K, 0, sizeof(K));
  K.nx = p.nx;
  K.ny = p.ny;
  K.nz = p.nz;
  K.nxp = p.nx + 2;
  K.nyp = p.ny + 2;
  K.nzp = p.nz + 2;
  K.nodes = (long long)K.nxp * K.nyp * K.nzp;
  K.species = p.species;
  K.xflow = p.xflow != 0;
  K.yflow = p.yflow != 0;
  K.zflow = p.zflow != 0;
  K.produce_dt_scaled = p.produce_dt_scaled;
  K.xmin = p.xmin; K.xmax = p.xmax; K.ymin = p.ymin; K.ymax = p.ymax; K.zmin = p.zmin; K.zmax = p.zmax;
  K.Lx_min = p.Lx_min; K.Lx_max = p.Lx_max; K.Ly_min = p.Ly_min; K.Ly_max = p.Ly_max;
  K.Lz_min = p.Lz_min; K.Lz_max = p.Lz_max;
  K.dx = p.dxyz[0];
  K.dy = p.dxyz[1];
  K.dz = p.dxyz[2];
  K.dV = p.dxyz[0] * p.dxyz[1] * p.dxyz[2];
  K.dt = p.dt;
  for (int c = 0; c < 3; ++c) {
    K.ve[c] = p.ve[c];
    K.E0[c] = p.E0[c];
    K.B0[c] = p.B0[c];
  }
  const double* m = p.mass;
  for (int s = 0; s < 8; ++s) {
    K.gyration[s] = p.gyration[s] != 0;
    K.fluid[s] = p.fluid[s] != 0;
    K.ipp[s] = p.ipp[s];
    K.epp[s] = p.epp[s];
    K.hpp[s] = p.hpp[s];
    K.mass[s] = p.mass[s];
    K.charge[s] = p.charge[s];
    K.kelvin[s] = p.kelvin[s];
    K.n2p[s] = p.n2p[s];
    K.eta[s] = p.eta[s];
    for (int c = 0; c < 3; ++c) {
      K.v0[s][c] = p.v0[s][c];
      K.tB[s][c] = p.tB[s][c];
      K.sB[s][c] = p.sB[s][c];
    }
    K.vn[s] = p.vn[s];
    K.Qn[s] = p.Qn[s];
    K.nu_i[s] = p.nu_i[s];
    K.nu_d[s] = p.nu_d[s];
    K.Ek[s] = p.Ek[s];
    K.ue[s] = K.uh[s] = K.ui[s] = 0.0;
  }
  // ParticlesProduce.f90:26-36
  for (int s = 0; s < p.species; ++s) {
    K.ue[s] = std::sqrt(2.0 * m[s] * p.Ek[s] * (1.0 / (m[0] * (m[s] + m[0]))));
    K.uh[s] = std::sqrt(2.0 * m[s] * p.Ek[s] * (1.0 / (m[1] * (m[s] + m[1]))));
    if (p.epp[s] > 0)
      K.ui[s] = std::sqrt(2.0 * m[0] * p.Ek[s] * (1.0 / (m[s] * (m[s] + m[0]))));
    else if (p.hpp[s] > 0)
      K.ui[s] = std::sqrt(2.0 * m[1] * p.Ek[s] * (1.0 / (m[s] * (m[s] + m[1]))));
  }
  K.seed = p.seed;
  return K;
}

// The guard shell BCinflow.f90 fills on one rank, in its loop order.
InflowTable make_inflow_table(const picard_params& p) {
  InflowTable T;
  std::memset(&T, 0, sizeof(T));
  const double dx = p.dxyz[0], dy = p.dxyz[1], dz = p.dxyz[2];
  const int Nx = p.nx, Ny = p.ny, Nz = p.nz;
  int ypos = (p.yflow && (p.Ly_max + 0.5 * dy > p.ymax)) ? 1 : 0;
  int yneg = (p.yflow && (p.Ly_min - 0.5 * dy < p.ymin)) ? 1 : 0;
  int zpos = (p.zflow && (p.Lz_max + 0.5 * dz > p.zmax)) ? 1 : 0;
  int zneg = (p.zflow && (p.Lz_min - 0.5 * dz < p.zmin)) ? 1 : 0;
  auto add = [&](int axis, int fixed, int o_lo, int o_n, int i_lo, int i_n, double edge) {
    InflowFace& F = T.f[T.nfaces++];
    F.axis = axis;
    F.fixed = fixed;
    F.o_lo = o_lo;
    F.o_n = o_n;
    F.i_lo = i_lo;
    F.i_n = i_n;
    F.edge = edge;
    F.first = T.cells;
    T.cells += (long long)o_n * i_n;
  };
  if (p.xflow && (p.Lx_max + 0.5 * dx > p.xmax))
    add(0, Nx + 2, 2 - zneg, Nz + zneg + zpos, 2 - yneg, Ny + yneg + ypos, p.Lx_max);
  if (p.xflow && (p.Lx_min - 0.5 * dx < p.xmin))
    add(0, 1, 2 - zneg, Nz + zneg + zpos, 2 - yneg, Ny + yneg + ypos, p.Lx_min - dx);
  if (ypos > 0) add(1, Ny + 2, 2, Nz + zpos, 2, Nx, p.Ly_max);
  if (yneg > 0) add(1, 1, 2 - zneg, Nz + zneg, 2, Nx, p.Ly_min - dy);
  if (zpos > 0) add(2, Nz + 2, 2 - yneg, Ny + yneg, 2, Nx, p.Lz_max);
  if (zneg > 0) add(2, 1, 2, Ny + ypos, 2, Nx, p.Lz_min - dz);
  T.group_prefix[0] = 0;
  for (int s = 0; s < 8; ++s)
    T.group_prefix[s + 1] = T.group_prefix[s] + (s < p.species ? p.ipp[s] * (1 + p.epp[s] + p.hpp[s]) : 0);
  T.per_cell = T.group_prefix[p.species];
  return T;
}

}  // namespace picard

namespace {

template <class T>
int dalloc(picard_ctx* c, T*& p, size_t n) {
  void* q = nullptr;
  size_t bytes = std::max<size_t>(n, 1) * sizeof(T);
  // stream-ordered: creating or destroying a context does not synchronise
  // the device, so contexts of concurrent runs come and go independently
  cudaError_t e = cudaMallocAsync(&q, bytes, c->st);
  if (e != cudaSuccess)
    return fail(PICARD_ERR_CUDA, "cudaMallocAsync(" + std::to_string(bytes) + " B): " + cudaGetErrorString(e));
  c->allocs.push_back(q);
  e = cudaMemsetAsync(q, 0, bytes, c->st);
  if (e != cudaSuccess) return check_cuda(e, "cudaMemsetAsync");
  p = static_cast<T*>(q);
  return PICARD_OK;
}

// Frees one allocation of dalloc on the context's stream.
void release(picard_ctx* c, void* q) {
  auto it = std::find(c->allocs.begin(), c->allocs.end(), q);
  if (it == c->allocs.end()) return;
  c->allocs.erase(it);
  cudaFreeAsync(q, c->st);
}

}  // namespace

namespace picard {
int dev_alloc(picard_ctx* c, void** p, size_t bytes) {
  unsigned char* q = nullptr;
  PICARD_TRY(dalloc(c, q, bytes));
  *p = q;
  return PICARD_OK;
}
}  // namespace picard

namespace {

struct Sizes {
  long long cap, nodes, cells, dsize;
  int species, nb_compact, nb_jacobi, nb_inflow;
};

Sizes sizes_of(const picard_params& p) {
  Sizes s;
  s.cap = p.max_per_proc;
  s.nodes = (long long)(p.nx + 2) * (p.ny + 2) * (p.nz + 2);
  s.cells = (long long)p.nx * p.ny * p.nz;
  s.dsize = (long long)(2 * p.nx + 1) * (2 * p.ny + 1) * (2 * p.nz + 1);
  s.species = p.species;
  s.nb_compact = compact_blocks(s.cap) + 1;
  const InflowTable T = make_inflow_table(p);
  s.nb_inflow = T.cells * T.per_cell > 0 ? inflow_blocks(T.cells * T.per_cell) : 0;
  KParams K = make_kparams(p);
  s.nb_jacobi = jacobi_geom(K).nblocks;
  return s;
}

int validate(const picard_params* p, int layout, int solver) {
  if (!p) return fail(PICARD_ERR_BAD_ARG, "params is NULL");
  if (p->nx < 1 || p->ny < 1 || p->nz < 1) return fail(PICARD_ERR_BAD_ARG, "grid dimensions must be positive");
  if (p->species < 2 || p->species > 8) return fail(PICARD_ERR_BAD_ARG, "species must be in 2..8");
  if (p->max_per_proc < 1) return fail(PICARD_ERR_BAD_ARG, "max_per_proc must be positive");
  if (layout != PICARD_LAYOUT_F64 && layout != PICARD_LAYOUT_CELL32) return fail(PICARD_ERR_BAD_ARG, "unknown layout");
  if (solver != PICARD_SOLVER_F64 && solver != PICARD_SOLVER_F32_REFINE && solver != PICARD_SOLVER_SPECTRAL)
    return fail(PICARD_ERR_BAD_ARG, "unknown solver");
  if (layout == PICARD_LAYOUT_CELL32 &&
      (p->nx + 2 > (int)kCellMaskX || p->ny + 2 > (int)kCellMaskY || p->nz + 2 > (int)kCellMaskZ))
    return fail(PICARD_ERR_BAD_ARG, "CELL32 layout holds at most 2045 x 2045 x 1021 cells");
  if (!(p->dxyz[0] > 0.0 && p->dxyz[1] > 0.0 && p->dxyz[2] > 0.0))
    return fail(PICARD_ERR_BAD_ARG, "params not derived (call picard_params_derive first)");
  return PICARD_OK;
}

int sync_count(picard_ctx* c) {
  PICARD_CUDA(cudaMemcpyAsync(c->h_pinned_i, c->d_count, sizeof(int), cudaMemcpyDeviceToHost, c->st));
  PICARD_CUDA(cudaStreamSynchronize(c->st));
  c->stats.d2h_bytes += sizeof(int);
  c->num_local = c->h_pinned_i[0];
  return PICARD_OK;
}

int push_count(picard_ctx* c) {
  c->h_pinned_i[1] = int(c->num_local);
  PICARD_CUDA(cudaMemcpyAsync(c->d_count, c->h_pinned_i + 1, sizeof(int), cudaMemcpyHostToDevice, c->st));
  PICARD_CUDA(cudaStreamSynchronize(c->st));
  c->stats.h2d_bytes += sizeof(int);
  return PICARD_OK;
}

int check_dev_err(picard_ctx* c) {
  PICARD_CUDA(cudaMemcpyAsync(c->h_pinned_i + 2, c->d_err, sizeof(int), cudaMemcpyDeviceToHost, c->st));
  PICARD_CUDA(cudaStreamSynchronize(c->st));
  c->stats.d2h_bytes += sizeof(int);
  int e = c->h_pinned_i[2];
  if (e == kDevCapacity) {
    cudaMemsetAsync(c->d_err, 0, sizeof(int), c->st);
    return fail(PICARD_ERR_CAPACITY, "particle capacity max_per_proc exceeded on the device");
  }
  if (e == kDevTimeout) {
    cudaMemsetAsync(c->d_err, 0, sizeof(int), c->st);
    return fail(PICARD_ERR_TIMEOUT, "a bounded device wait gave up");
  }
  if (e == kDevRange) {
    cudaMemsetAsync(c->d_err, 0, sizeof(int), c->st);
    return fail(PICARD_ERR_STATE, "a particle move left its range on the device and was skipped");
  }
  return PICARD_OK;
}

int check_dev_err_timeout(picard_ctx* c) {
  PICARD_CUDA(cudaMemcpyAsync(c->h_pinned_i + 5, c->d_err, sizeof(int), cudaMemcpyDeviceToHost, c->st));
  PICARD_CUDA(cudaStreamSynchronize(c->st));
  c->stats.d2h_bytes += sizeof(int);
  if (c->h_pinned_i[5] == kDevTimeout) {
    cudaMemsetAsync(c->d_err, 0, sizeof(int), c->st);
    return fail(PICARD_ERR_TIMEOUT, "a tensor-core BCpotentials block timed out waiting for its MMAs");
  }
  return PICARD_OK;
}

int ensure_capacity(picard_ctx* c, long long add) {
  if (c->num_local + add > c->capacity)
    return fail(PICARD_ERR_CAPACITY, "particle count " + std::to_string(c->num_local + add) +
                                         " would exceed max_per_proc " + std::to_string(c->capacity));
  return PICARD_OK;
}

}  // namespace

namespace picard {
int sync_count_public(picard_ctx* c) {
  PICARD_TRY(check_dev_err(c));
  return sync_count(c);
}

int check_dev_err_public(picard_ctx* c) { return check_dev_err(c); }

int bc_potentials_async(picard_ctx* c) {
  if (c->bcpot_tensor == PICARD_BCPOT_FFT) return bc_potentials_fft(c);
  if (c->bcpot_tensor == PICARD_BCPOT_TENSOR) {
    if (!c->tc_cs) {
      long long cs = 0, pe = 0;
      bcpot_tc_scratch(c->K, &cs, &pe);
      unsigned short* csb = nullptr;
      PICARD_TRY(dalloc(c, csb, (size_t)cs));
      PICARD_TRY(dalloc(c, c->tc_partial, (size_t)pe));
      c->tc_cs = csb;
    }
    PICARD_CUDA(launch_bc_potentials_tc(c->K, c->C, c->D, c->U, c->tc_cs, c->tc_partial, c->d_err, c->st));
    return PICARD_OK;
  }
  PICARD_CUDA(launch_bc_potentials(c->K, c->C, c->D, c->U, c->st));
  return PICARD_OK;
}

static cudaError_t launch_outflow_split(picard_ctx* c, long long n, const OutflowSplit* sp) {
  if (c->layout == PICARD_LAYOUT_F64)
    return launch_outflow_f64(c->K, c->f64, n, c->out_words, c->blk_counts, c->blk_offsets, c->d_count, 0, c->d_err,
                              c->st, sp);
  return launch_outflow_c32(c->K, c->c32, n, c->out_words, c->blk_counts, c->blk_offsets, c->d_count, 0, c->d_err,
                            c->st, sp);
}

cudaError_t launch_outflow(picard_ctx* c, int wrap) {
  if (c->layout == PICARD_LAYOUT_F64)
    return launch_outflow_f64(c->K, c->f64, c->num_local, c->out_words, c->blk_counts, c->blk_offsets, c->d_count,
                              wrap, c->d_err, c->st);
  return launch_outflow_c32(c->K, c->c32, c->num_local, c->out_words, c->blk_counts, c->blk_offsets, c->d_count, wrap,
                            c->d_err, c->st);
}

cudaError_t launch_inflow_fused(picard_ctx* c, int iteration) {
  const long long cand = (long long)c->inflow.cells * c->inflow.per_cell;
  if (cand > 0 && !c->inflow_stage.x) {
    const long long slots = inflow_stage_slots(cand);
    double* x = nullptr;
    int8_t* sp = nullptr;
    if (dalloc(c, x, (size_t)(6 * slots)) != PICARD_OK || dalloc(c, sp, (size_t)slots) != PICARD_OK)
      return cudaErrorMemoryAllocation;
    c->inflow_stage.x = x;
    c->inflow_stage.sp = sp;
  }
  if (c->layout == PICARD_LAYOUT_F64)
    return launch_inflow_fused_f64(c->K, c->inflow, iteration, c->f64, c->d_count, c->capacity, c->inflow_counts,
                                   c->inflow_offsets, c->d_err, c->inflow_stage, c->st);
  return launch_inflow_fused_c32(c->K, c->inflow, iteration, c->c32, c->d_count, c->capacity, c->inflow_counts,
                                 c->inflow_offsets, c->d_err, c->inflow_stage, c->st);
}

int count_issue(picard_ctx* c) {
  PICARD_CUDA(cudaMemcpyAsync(c->h_pinned_i + 2, c->d_err, sizeof(int), cudaMemcpyDeviceToHost, c->st));
  PICARD_CUDA(cudaMemcpyAsync(c->h_pinned_i, c->d_count, sizeof(int), cudaMemcpyDeviceToHost, c->st));
  c->stats.d2h_bytes += 2 * sizeof(int);
  return PICARD_OK;
}

int count_collect(picard_ctx* c) {
  PICARD_CUDA(cudaStreamSynchronize(c->st));
  if (c->h_pinned_i[2] == kDevCapacity) {
    cudaMemsetAsync(c->d_err, 0, sizeof(int), c->st);
    return fail(PICARD_ERR_CAPACITY, "particle capacity max_per_proc exceeded on the device");
  }
  if (c->h_pinned_i[2] == kDevTimeout) {
    cudaMemsetAsync(c->d_err, 0, sizeof(int), c->st);
    return fail(PICARD_ERR_TIMEOUT, "a bounded device wait gave up");
  }
  if (c->h_pinned_i[2] == kDevRange) {
    cudaMemsetAsync(c->d_err, 0, sizeof(int), c->st);
    return fail(PICARD_ERR_STATE, "a particle move left its range on the device and was skipped");
  }
  c->num_local = c->h_pinned_i[0];
  return PICARD_OK;
}
}  // namespace picard

// ======================================================================= ABI

extern "C" {

const char* picard_gpu_last_error(void) { return g_last_error.c_str(); }

int picard_gpu_pool_keep(int32_t device, uint64_t bytes) {
  int count = 0;
  PICARD_CUDA(cudaGetDeviceCount(&count));
  if (device < 0 || device >= count) return fail(PICARD_ERR_BAD_ARG, "no such device");
  cudaMemPool_t pool;
  PICARD_CUDA(cudaDeviceGetDefaultMemPool(&pool, device));
  PICARD_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &bytes));
  return PICARD_OK;
}

int picard_gpu_footprint(const picard_params* p, int32_t layout, int32_t solver, uint64_t* bytes) {
  PICARD_TRY(validate(p, layout, solver));
  if (!bytes) return fail(PICARD_ERR_BAD_ARG, "bytes is NULL");
  Sizes s = sizes_of(*p);
  double per_particle = layout == PICARD_LAYOUT_F64 ? 49.0 : 29.0;
  double b = per_particle * (double)s.cap;
  b += (double)s.nodes * (8.0 * s.species /*Nacc*/ + 8.0 * s.species /*N*/ + 8 * 3 /*C,U,b*/ + 24 /*E*/ + 8 /*U1*/);
  if (layout == PICARD_LAYOUT_CELL32) b += 16.0 * s.nodes;
  if (solver == PICARD_SOLVER_F64) b += 8.0 * s.nodes;
  else if (solver == PICARD_SOLVER_SPECTRAL) b += (double)spectral_bytes(make_kparams(*p));
  else b += 16.0 * (double)f32_elems(make_kparams(*p));
  b += 8.0 * (double)s.dsize;
  b += 8.0 * (double)s.cells;                // produce counts + offsets
  b += 8.0 * (double)s.nb_compact * (3 + kOutflowWordsPerBlock);  // BCoutflow scratch
  b += 8.0 * (double)s.nb_inflow * 2;        // fused BCinflow scan
  {
    const InflowTable T = make_inflow_table(*p);  // fused BCinflow survivors' staging area
    const long long cand = (long long)T.cells * T.per_cell;
    if (cand > 0) b += 49.0 * (double)inflow_stage_slots(cand);
  }
  b += 8.0 * (kMaxSweepsPerRound + 1.0) * s.nb_jacobi;  // sweep partials
  if (layout == PICARD_LAYOUT_CELL32) {      // BCpotentials scratch of the layout's default method
    const KParams K = make_kparams(*p);
    if (bcpot_fft_supported(K)) {
      b += (double)bcpot_fft_bytes(K);
    } else {
      long long cs = 0, pe = 0;
      bcpot_tc_scratch(K, &cs, &pe);
      b += 2.0 * (double)cs + 8.0 * (double)pe;
    }
  }
  *bytes = (uint64_t)b;
  return PICARD_OK;
}

int picard_gpu_create(const picard_params* p, int32_t layout, int32_t solver, picard_ctx** out) {
  PICARD_TRY(validate(p, layout, solver));
  if (!out) return fail(PICARD_ERR_BAD_ARG, "out is NULL");
  picard_ctx* c = new picard_ctx();
  c->prm = *p;
  c->K = make_kparams(*p);
  c->layout = layout;
  c->solver = solver;
  c->capacity = p->max_per_proc;
  c->inflow = make_inflow_table(*p);
  c->G = jacobi_geom(c->K);
  c->bcpot_tensor = layout != PICARD_LAYOUT_CELL32 ? PICARD_BCPOT_DIRECT
                    : bcpot_fft_supported(c->K)   ? PICARD_BCPOT_FFT
                                                  : PICARD_BCPOT_TENSOR;
  int rc = PICARD_OK;
  auto bail = [&](int code) {
    picard_gpu_destroy(c);
    return code;
  };
  if (cudaGetDevice(&c->device) != cudaSuccess) return bail(fail(PICARD_ERR_CUDA, "no CUDA device"));
  if ((rc = check_cuda(cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking), "cudaStreamCreate"))) return bail(rc);
  Sizes s = sizes_of(*p);
  const long long cap = s.cap;
  // one particle buffer: BCoutflow removes in place
  if (layout == PICARD_LAYOUT_F64) {
    PartF64& a = c->f64;
    if ((rc = dalloc(c, a.x, cap)) || (rc = dalloc(c, a.y, cap)) || (rc = dalloc(c, a.z, cap)) ||
        (rc = dalloc(c, a.vx, cap)) || (rc = dalloc(c, a.vy, cap)) || (rc = dalloc(c, a.vz, cap)) ||
        (rc = dalloc(c, a.sp, cap)))
      return bail(rc);
  } else {
    PartC32& a = c->c32;
    if ((rc = dalloc(c, a.cell, cap)) || (rc = dalloc(c, a.fx, cap)) || (rc = dalloc(c, a.fy, cap)) ||
        (rc = dalloc(c, a.fz, cap)) || (rc = dalloc(c, a.vx, cap)) || (rc = dalloc(c, a.vy, cap)) ||
        (rc = dalloc(c, a.vz, cap)) || (rc = dalloc(c, a.sp, cap)))
      return bail(rc);
  }
  const long long nn = s.nodes;
  if ((rc = dalloc(c, c->d_count, 1)) || (rc = dalloc(c, c->d_err, 1)) || (rc = dalloc(c, c->d_info, 4)) ||
      (rc = dalloc(c, c->Nacc, nn * s.species)) || (rc = dalloc(c, c->N, nn * s.species)) ||
      (rc = dalloc(c, c->C, nn)) || (rc = dalloc(c, c->U, nn)) || (rc = dalloc(c, c->E, 3 * nn)) ||
      (rc = dalloc(c, c->D, s.dsize)) || (rc = dalloc(c, c->b, nn)) || (rc = dalloc(c, c->U1, nn)))
    return bail(rc);
  if (layout == PICARD_LAYOUT_CELL32 && (rc = dalloc(c, c->E32, nn))) return bail(rc);
  if (solver == PICARD_SOLVER_F64) {
    if ((rc = dalloc(c, c->Usnap, nn))) return bail(rc);
  } else if (solver == PICARD_SOLVER_SPECTRAL) {
    if ((rc = spectral_alloc(c))) return bail(rc);
  } else {
    const long long fe = f32_elems(c->K);
    if ((rc = dalloc(c, c->w[0], fe)) || (rc = dalloc(c, c->w[1], fe)) || (rc = dalloc(c, c->r, 2 * fe))) return bail(rc);
    if (c->G.tma) {
      int e0 = make_tensor_map(&c->tmw[0], c->w[0], c->K, 40, 10, c->G.zc + 2);
      int e1 = make_tensor_map(&c->tmw[1], c->w[1], c->K, 40, 10, c->G.zc + 2);
      int e2 = make_tensor_map(&c->tmr[0], c->r, c->K, 32, 8, c->G.zc);
      int e3 = make_tensor_map(&c->tmr[1], c->r + fe, c->K, 32, 8, c->G.zc);
      e0 |= make_tensor_map(&c->tmw2[0], c->w[0], c->K, 72, 10, c->G.zc + 2);
      e1 |= make_tensor_map(&c->tmw2[1], c->w[1], c->K, 72, 10, c->G.zc + 2);
      e2 |= make_tensor_map(&c->tmr2[0], c->r, c->K, 64, 8, c->G.zc);
      e3 |= make_tensor_map(&c->tmr2[1], c->r + fe, c->K, 64, 8, c->G.zc);
      if (c->G.zc <= 8) {
        e0 |= make_tensor_map(&c->tmw3[0], c->w[0], c->K, 72, 12, c->G.zc + 4);
        e1 |= make_tensor_map(&c->tmw3[1], c->w[1], c->K, 72, 12, c->G.zc + 4);
        e2 |= make_tensor_map(&c->tmr3[0], c->r, c->K, 72, 10, c->G.zc + 2);
        e3 |= make_tensor_map(&c->tmr3[1], c->r + fe, c->K, 72, 10, c->G.zc + 2);
      }
      if (e0 || e1 || e2 || e3)
        return bail(fail(PICARD_ERR_CUDA, "cuTensorMapEncodeTiled failed (" + std::to_string(e0 | e1 | e2 | e3) + ")"));
    }
  }
  if ((rc = dalloc(c, c->partials, (size_t)(c->m_max + 1) * c->G.nblocks)) ||
      (rc = dalloc(c, c->r2, c->m_max + 1)))
    return bail(rc);
  int scan_extra = scan_scratch_ints(s.nb_compact) + 4;
  if ((rc = dalloc(c, c->blk_counts, s.nb_compact)) ||
      (rc = dalloc(c, c->blk_offsets, 2 * (size_t)s.nb_compact + 2 + scan_extra)) ||
      (rc = dalloc(c, c->out_words, (size_t)kOutflowWordsPerBlock * s.nb_compact)))
    return bail(rc);
  if (s.nb_inflow > 0 &&
      ((rc = dalloc(c, c->inflow_counts, s.nb_inflow)) ||
       (rc = dalloc(c, c->inflow_offsets, (size_t)s.nb_inflow + 2 + scan_scratch_ints(s.nb_inflow) + 4))))
    return bail(rc);
  int cells = int(s.cells);
  if ((rc = dalloc(c, c->cell_counts, cells)) ||
      (rc = dalloc(c, c->cell_offsets, (size_t)cells + 2 + scan_scratch_ints(cells) + 4)))
    return bail(rc);
  c->red_blocks = std::max<int>(148 * 16, rhs_blocks(c->K));
  if ((rc = dalloc(c, c->red_partial, c->red_blocks)) || (rc = dalloc(c, c->red_result, 8))) return bail(rc);
  if ((rc = check_cuda(cudaMallocHost((void**)&c->h_pinned, sizeof(double) * (c->m_max + 16)), "cudaMallocHost")))
    return bail(rc);
  if ((rc = check_cuda(cudaMallocHost((void**)&c->h_pinned_i, sizeof(int) * 16), "cudaMallocHost"))) return bail(rc);
  for (int e = 0; e < 4; ++e)
    if ((rc = check_cuda(cudaEventCreate(&c->ev[e]), "cudaEventCreate"))) return bail(rc);
  for (int e = 0; e < 6; ++e)
    if ((rc = check_cuda(cudaEventCreate(&c->pev[e]), "cudaEventCreate"))) return bail(rc);
  if ((rc = tune_sweep(c, false))) return bail(rc);
  if ((rc = check_cuda(cudaStreamSynchronize(c->st), "create"))) return bail(rc);
  c->launches_at_reset = launches_so_far();
  *out = c;
  return PICARD_OK;
}

int picard_gpu_destroy(picard_ctx* c) {
  if (!c) return PICARD_OK;
  if (c->st) {
    for (void* q : c->allocs) cudaFreeAsync(q, c->st);
    cudaStreamSynchronize(c->st);
  }
  bcpot_fft_free(c);
  if (c->h_pinned) cudaFreeHost(c->h_pinned);
  if (c->h_pinned_i) cudaFreeHost(c->h_pinned_i);
  for (int e = 0; e < 4; ++e)
    if (c->ev[e]) cudaEventDestroy(c->ev[e]);
  for (int e = 0; e < 6; ++e)
    if (c->pev[e]) cudaEventDestroy(c->pev[e]);
  if (c->st) cudaStreamDestroy(c->st);
  delete c;
  return PICARD_OK;
}

int picard_gpu_synchronize(picard_ctx* c) {
  if (!c) return fail(PICARD_ERR_BAD_ARG, "ctx is NULL");
  PICARD_CUDA(cudaStreamSynchronize(c->st));
  return PICARD_OK;
}

int picard_gpu_get_stats(picard_ctx* c, picard_stats* out) {
  if (!c || !out) return fail(PICARD_ERR_BAD_ARG, "NULL argument");
  *out = c->stats;
  out->kernel_launches = launches_so_far() - c->launches_at_reset;
  out->last_sweeps = c->last_sweeps;
  return PICARD_OK;
}

int picard_gpu_reset_stats(picard_ctx* c) {
  if (!c) return fail(PICARD_ERR_BAD_ARG, "ctx is NULL");
  c->stats = picard_stats{};
  c->launches_at_reset = launches_so_far();
  return PICARD_OK;
}

int picard_gpu_get_stream(picard_ctx* c, void** stream) {
  if (!c || !stream) return fail(PICARD_ERR_BAD_ARG, "NULL argument");
  *stream = (void*)c->st;
  return PICARD_OK;
}

int picard_gpu_get_num_local(picard_ctx* c, int32_t* n) {
  if (!c || !n) return fail(PICARD_ERR_BAD_ARG, "NULL argument");
  *n = int32_t(c->num_local);
  return PICARD_OK;
}

// ------------------------------------------------------------ transfers

int picard_gpu_set_particles(picard_ctx* c, const double* rp, const int32_t* ip, int32_t n) {
  if (!c || (n > 0 && (!rp || !ip))) return fail(PICARD_ERR_BAD_ARG, "NULL argument");
  if (n < 0 || n > c->capacity) return fail(PICARD_ERR_CAPACITY, "num_local exceeds max_per_proc");
  std::vector<double> soa((size_t)6 * n);
  std::vector<int8_t> sp(n);
  for (int32_t p = 0; p < n; ++p) {
    for (int q = 0; q < 6; ++q) soa[(size_t)q * n + p] = rp[(size_t)8 * p + q];
    if (ip[p] < 1 || ip[p] > c->prm.species) return fail(PICARD_ERR_BAD_ARG, "int_particles holds an unknown species");
    sp[p] = int8_t(ip[p] - 1);
  }
  PartF64 dst;
  std::vector<void*> tmp;
  if (c->layout == PICARD_LAYOUT_F64) {
    dst = c->f64;
  } else {
    double* buf = nullptr;
    int8_t* sb = nullptr;
    PICARD_CUDA(cudaMallocAsync(&buf, sizeof(double) * 6 * std::max<int32_t>(n, 1), c->st));
    PICARD_CUDA(cudaMallocAsync(&sb, std::max<int32_t>(n, 1), c->st));
    tmp = {buf, sb};
    dst.x = buf;
    dst.y = buf + n;
    dst.z = buf + 2 * (size_t)n;
    dst.vx = buf + 3 * (size_t)n;
    dst.vy = buf + 4 * (size_t)n;
    dst.vz = buf + 5 * (size_t)n;
    dst.sp = sb;
  }
  double* cols[6] = {dst.x, dst.y, dst.z, dst.vx, dst.vy, dst.vz};
  for (int q = 0; q < 6; ++q)
    PICARD_CUDA(cudaMemcpyAsync(cols[q], soa.data() + (size_t)q * n, sizeof(double) * n, cudaMemcpyHostToDevice, c->st));
  PICARD_CUDA(cudaMemcpyAsync(dst.sp, sp.data(), n, cudaMemcpyHostToDevice, c->st));
  if (c->layout == PICARD_LAYOUT_CELL32) PICARD_CUDA(launch_f64_to_c32(c->K, dst, n, c->c32, c->st));
  for (void* q : tmp) cudaFreeAsync(q, c->st);
  PICARD_CUDA(cudaStreamSynchronize(c->st));
  c->stats.h2d_bytes += (int64_t)n * 49;
  c->num_local = n;
  return push_count(c);
}

int picard_gpu_get_particles(picard_ctx* c, double* rp, int32_t* ip, int32_t capacity, int32_t* num_local) {
  if (!c) return fail(PICARD_ERR_BAD_ARG, "ctx is NULL");
  const long long n = c->num_local;
  if (num_local) *num_local = int32_t(n);
  if (!rp && !ip) return PICARD_OK;
  if (capacity < n) return fail(PICARD_ERR_CAPACITY, "host arrays smaller than num_local");
  PartF64 src;
  std::vector<void*> tmp;
  if (c->layout == PICARD_LAYOUT_F64) {
    src = c->f64;
  } else {
    double* buf = nullptr;
    int8_t* sb = nullptr;
    PICARD_CUDA(cudaMallocAsync(&buf, sizeof(double) * 6 * std::max<long long>(n, 1), c->st));
    PICARD_CUDA(cudaMallocAsync(&sb, std::max<long long>(n, 1), c->st));
    tmp = {buf, sb};
    src.x = buf;
    src.y = buf + n;
    src.z = buf + 2 * n;
    src.vx = buf + 3 * n;
    src.vy = buf + 4 * n;
    src.vz = buf + 5 * n;
    src.sp = sb;
    PICARD_CUDA(launch_c32_to_f64(c->K, c->c32, n, src, c->st));
  }
  std::vector<double> soa((size_t)6 * n);
  std::vector<int8_t> sp(n);
  double* cols[6] = {src.x, src.y, src.z, src.vx, src.vy, src.vz};
  for (int q = 0; q < 6; ++q)
    PICARD_CUDA(cudaMemcpyAsync(soa.data() + (size_t)q * n, cols[q], sizeof(double) * n, cudaMemcpyDeviceToHost, c->st));
  PICARD_CUDA(cudaMemcpyAsync(sp.data(), src.sp, n, cudaMemcpyDeviceToHost, c->st));
  for (void* q : tmp) cudaFreeAsync(q, c->st);
  PICARD_CUDA(cudaStreamSynchronize(c->st));
  c->stats.d2h_bytes += (int64_t)n * 49;
  for (long long p = 0; p < n; ++p) {
    if (rp) {
      for (int q = 0; q < 6; ++q) rp[(size_t)8 * p + q] = soa[(size_t)q * n + p];
      rp[(size_t)8 * p + 6] = 0.0;
      rp[(size_t)8 * p + 7] = 0.0;
    }
    if (ip) ip[p] = int32_t(sp[p]) + 1;
  }
  return PICARD_OK;
}

static int field_geometry(picard_ctx* c, int which, double** dev, int* ncomp, long long* n) {
  const long long nn = c->K.nodes;
  const int S = c->prm.species;
  switch (which) {
    case PICARD_FIELD_U: *dev = c->U; *ncomp = 1; *n = nn; return PICARD_OK;
    case PICARD_FIELD_C: *dev = c->C; *ncomp = 1; *n = nn; return PICARD_OK;
    case PICARD_FIELD_E: *dev = c->E; *ncomp = 3; *n = nn; return PICARD_OK;
    case PICARD_FIELD_N: *dev = c->N; *ncomp = S; *n = nn; return PICARD_OK;
    case PICARD_FIELD_F:
      if (!c->F) return fail(PICARD_ERR_STATE, "flux F exists after picard_gpu_particles_gridify_all");
      *dev = c->F; *ncomp = 3 * S; *n = nn; return PICARD_OK;
    case PICARD_FIELD_D:
      *dev = c->D; *ncomp = 1;
      *n = (long long)(2 * c->prm.nx + 1) * (2 * c->prm.ny + 1) * (2 * c->prm.nz + 1);
      return PICARD_OK;
  }
  return fail(PICARD_ERR_BAD_ARG, "unknown field");
}

// Device planes [comp][node] <-> reference order (comp fastest).  For F the
// device plane index is s*3 + c and the reference order is F(s, c, node).
static inline size_t ref_index(int which, int S, int plane, long long g) {
  if (which == PICARD_FIELD_F) {
    int s = plane / 3, c = plane % 3;
    return (size_t)s + (size_t)S * ((size_t)c + 3 * (size_t)g);
  }
  int ncomp = which == PICARD_FIELD_E ? 3 : (which == PICARD_FIELD_N ? S : 1);
  return (size_t)plane + (size_t)ncomp * (size_t)g;
}

int picard_gpu_get_field(picard_ctx* c, int32_t which, double* out) {
  if (!c || !out) return fail(PICARD_ERR_BAD_ARG, "NULL argument");
  double* dev;
  int ncomp;
  long long n;
  PICARD_TRY(field_geometry(c, which, &dev, &ncomp, &n));
  std::vector<double> h((size_t)ncomp * n);
  PICARD_CUDA(cudaMemcpyAsync(h.data(), dev, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, c->st));
  PICARD_CUDA(cudaStreamSynchronize(c->st));
  c->stats.d2h_bytes += (int64_t)(sizeof(double) * h.size());
  for (int pl = 0; pl < ncomp; ++pl)
    for (long long g = 0; g < n; ++g) out[ref_index(which, c->prm.species, pl, g)] = h[(size_t)pl * n + g];
  return PICARD_OK;
}

int picard_gpu_set_field(picard_ctx* c, int32_t which, const double* in) {
  if (!c || !in) return fail(PICARD_ERR_BAD_ARG, "NULL argument");
  if (which == PICARD_FIELD_F && !c->F) PICARD_TRY(dalloc(c, c->F, (size_t)3 * c->prm.species * c->K.nodes));
  double* dev;
  int ncomp;
  long long n;
  PICARD_TRY(field_geometry(c, which, &dev, &ncomp, &n));
  std::vector<double> h((size_t)ncomp * n);
  for (int pl = 0; pl < ncomp; ++pl)
    for (long long g = 0; g < n; ++g) h[(size_t)pl * n + g] = in[ref_index(which, c->prm.species, pl, g)];
  PICARD_CUDA(cudaMemcpyAsync(dev, h.data(), sizeof(double) * h.size(), cudaMemcpyHostToDevice, c->st));
  c->stats.h2d_bytes += (int64_t)(sizeof(double) * h.size());
  if (which == PICARD_FIELD_D) bcpot_fft_invalidate(c);
  if (which == PICARD_FIELD_E && c->E32) {
    std::vector<float4> e32(n);
    for (long long g = 0; g < n; ++g)
      e32[g] = make_float4(float(h[g]), float(h[n + g]), float(h[2 * n + g]), 0.0f);
    PICARD_CUDA(cudaMemcpyAsync(c->E32, e32.data(), sizeof(float4) * n, cudaMemcpyHostToDevice, c->st));
    PICARD_CUDA(cudaStreamSynchronize(c->st));
  }
  PICARD_CUDA(cudaStreamSynchronize(c->st));
  return PICARD_OK;
}

// ------------------------------------------------ one entry per subroutine

// CalcDistance.f90:1-95
int picard_gpu_calc_distance(picard_ctx* c) {
  if (!c) return fail(PICARD_ERR_BAD_ARG, "ctx is NULL");
  PICARD_CUDA(launch_calc_distance(c->K, c->D, c->st));
  bcpot_fft_invalidate(c);
  return PICARD_OK;
}

// ParticlesInitialize.f90:2-125
int picard_gpu_particles_initialize(picard_ctx* c) {
  if (!c) return fail(PICARD_ERR_BAD_ARG, "ctx is NULL");
  long long per_cell = c->inflow.group_prefix[c->prm.species];
  long long total = (long long)c->prm.nx * c->prm.ny * c->prm.nz * per_cell;
  PICARD_TRY(ensure_capacity(c, total));
  if (c->layout == PICARD_LAYOUT_F64)
    PICARD_CUDA(launch_init_f64(c->K, c->f64, c->num_local, c->st));
  else
    PICARD_CUDA(launch_init_c32(c->K, c->c32, c->num_local, c->st));
  c->num_local += total;
  return push_count(c);
}

// BCinflow.f90:2-476
int picard_gpu_bc_inflow(picard_ctx* c, int32_t iteration) {
  if (!c) return fail(PICARD_ERR_BAD_ARG, "ctx is NULL");
  long long total = c->inflow.cells * c->inflow.per_cell;
  PICARD_TRY(ensure_capacity(c, total));
  if (c->layout == PICARD_LAYOUT_F64)
    PICARD_CUDA(launch_inflow_f64(c->K, c->inflow, iteration, c->f64, c->num_local, c->st));
  else
    PICARD_CUDA(launch_inflow_c32(c->K, c->inflow, iteration, c->c32, c->num_local, c->st));
  c->num_local += total;
  return push_count(c);
}

// AdvancePosition.f90:4-19
int picard_gpu_advance_position(picard_ctx* c, double dt) {
  if (!c) return fail(PICARD_ERR_BAD_ARG, "ctx is NULL");
  if (c->layout == PICARD_LAYOUT_F64)
    PICARD_CUDA(launch_advance_position_f64(c->K, c->f64, c->num_local, dt, c->st));
  else
    PICARD_CUDA(launch_advance_position_c32(c->K, c->c32, c->num_local, dt, c->st));
  return PICARD_OK;
}

// ParticlesProduce.f90:1-113
int picard_gpu_particles_produce(picard_ctx* c, int32_t iteration) {
  if (!c) return fail(PICARD_ERR_BAD_ARG, "ctx is NULL");
  const int cells = c->prm.nx * c->prm.ny * c->prm.nz;
  PICARD_CUDA(launch_produce_count(c->K, iteration, c->cell_counts, c->st));
  int* total = c->cell_offsets + cells;
  PICARD_CUDA(launch_scan_int(c->cell_counts, c->cell_offsets, cells, total, c->cell_offsets + cells + 2, c->st));
  PICARD_CUDA(cudaMemcpyAsync(c->h_pinned_i + 3, total, sizeof(int), cudaMemcpyDeviceToHost, c->st));
  PICARD_CUDA(cudaStreamSynchronize(c->st));
  c->stats.d2h_bytes += sizeof(int);
  long long add = c->h_pinned_i[3];
  if (add == 0) return PICARD_OK;
  PICARD_TRY(ensure_capacity(c, add));
  if (c->layout == PICARD_LAYOUT_F64)
    PICARD_CUDA(launch_produce_emit_f64(c->K, iteration, c->cell_offsets, c->f64, c->d_count,
                                        c->capacity, c->d_err, c->st));
  else
    PICARD_CUDA(launch_produce_emit_c32(c->K, iteration, c->cell_offsets, c->c32, c->d_count,
                                        c->capacity, c->d_err, c->st));
  PICARD_TRY(check_dev_err(c));
  return sync_count(c);
}

// BCoutflow.f90:5-87, in place and in the reference's order (outflow.cuh)
//
// In two stages around a read of the survivor count n': when the window
// [n', n) is wide (2^16 positions or more) and at least 64 times its
// survivors -- right after BCinflow has appended every candidate -- its chains
// are resolved by pointer jumping (outflow.cuh), with scratch of two ints per
// window position allocated on first use.
int picard_gpu_bc_outflow(picard_ctx* c) {
  if (!c) return fail(PICARD_ERR_BAD_ARG, "ctx is NULL");
  const long long n = c->num_local;
  OutflowSplit sp{1, 0, c->d_info, {nullptr, nullptr}};
  PICARD_CUDA(launch_outflow_split(c, n, &sp));
  PICARD_CUDA(cudaMemcpyAsync(c->h_pinned_i + 6, c->d_info, sizeof(int), cudaMemcpyDeviceToHost, c->st));
  PICARD_TRY(sync_count(c));
  c->stats.d2h_bytes += sizeof(int);
  const long long np = c->num_local, window = n - np, m = c->h_pinned_i[6];
  sp.stage = 2;
  sp.np = np;
  if (window >= (1LL << 16) && window >= 64 * m) {
    if (c->jump_cap < window) {
      const long long cap = std::min<long long>(c->capacity, std::max<long long>(window, 2 * c->jump_cap));
      for (int q = 0; q < 2; ++q) {
        if (c->jump[q]) {
          release(c, c->jump[q]);
          c->jump[q] = nullptr;
        }
        PICARD_TRY(dalloc(c, c->jump[q], (size_t)cap));
      }
      c->jump_cap = cap;
    }
    sp.nxt[0] = c->jump[0];
    sp.nxt[1] = c->jump[1];
  }
  PICARD_CUDA(launch_outflow_split(c, n, &sp));
  return check_dev_err(c);
}

// ParticlesTransfer.f90:2-614 (one rank: periodic wrap, ibid. 494-519)
int picard_gpu_particles_transfer(picard_ctx* c) {
  if (!c) return fail(PICARD_ERR_BAD_ARG, "ctx is NULL");
  if (c->layout == PICARD_LAYOUT_F64)
    PICARD_CUDA(launch_transfer_f64(c->K, c->f64, c->num_local, c->st));
  else
    PICARD_CUDA(launch_transfer_c32(c->K, c->c32, c->num_local, c->st));
  return PICARD_OK;
}

static int deposit(picard_ctx* c, bool with_flux) {
  const long long nn = c->K.nodes;
  const int S = c->prm.species;
  PICARD_CUDA(cudaMemsetAsync(c->Nacc, 0, sizeof(unsigned long long) * nn * S, c->st));
  unsigned long long* Facc = nullptr;
  if (with_flux) {
    if (!c->Facc) PICARD_TRY(dalloc(c, c->Facc, (size_t)3 * S * nn));
    if (!c->F) PICARD_TRY(dalloc(c, c->F, (size_t)3 * S * nn));
    Facc = c->Facc;
    PICARD_CUDA(cudaMemsetAsync(Facc, 0, sizeof(unsigned long long) * nn * S * 3, c->st));
  }
  if (c->layout == PICARD_LAYOUT_F64)
    PICARD_CUDA(launch_deposit_f64(c->K, c->f64, c->num_local, c->Nacc, Facc, c->st));
  else
    PICARD_CUDA(launch_deposit_c32(c->K, c->c32, c->num_local, c->Nacc, Facc, c->st));
  PICARD_CUDA(launch_finish_deposit(c->K, c->Nacc, c->N, c->C, c->st));
  if (with_flux) PICARD_CUDA(launch_finish_flux(c->K, Facc, c->F, c->st));
  return PICARD_OK;
}

// ParticlesGridify.f90:1-296
int picard_gpu_particles_gridify(picard_ctx* c) {
  if (!c) return fail(PICARD_ERR_BAD_ARG, "ctx is NULL");
  return deposit(c, false);
}

// ParticlesGridifyAll.f90:1-455
int picard_gpu_particles_gridify_all(picard_ctx* c) {
  if (!c) return fail(PICARD_ERR_BAD_ARG, "ctx is NULL");
  return deposit(c, true);
}

int picard_gpu_set_option(picard_ctx* c, int32_t option, int32_t value) {
  if (!c) return fail(PICARD_ERR_BAD_ARG, "ctx is NULL");
  if (option == PICARD_OPT_BCPOT_TENSOR) {
    if (value < PICARD_BCPOT_DIRECT || value > PICARD_BCPOT_FFT)
      return fail(PICARD_ERR_BAD_ARG, "BCPOT_TENSOR must be 0 (direct), 1 (tensor cores) or 2 (FFT)");
    if (value == PICARD_BCPOT_FFT && !bcpot_fft_supported(c->K))
      return fail(PICARD_ERR_BAD_ARG, "FFT BCpotentials: a face is longer than its shared-memory FFT");
    c->bcpot_tensor = value;
    return PICARD_OK;
  }
  if (option == PICARD_OPT_SWEEP_CTAS) {
    if (value < -1) return fail(PICARD_ERR_BAD_ARG, "SWEEP_CTAS must be -1, 0 or a CTA count");
    if (value == 0) {
      c->G.ctas = -1;  // forget the cached shape of this context
      return tune_sweep(c, true);
    }
    c->G.ctas = value < 0 ? 0 : value;
    return PICARD_OK;
  }
  if (option == PICARD_OPT_SWEEP_PDL) {
    c->G.pdl = value != 0;
    return PICARD_OK;
  }
  if (option == PICARD_OPT_SWEEP_RESIDENT) {
    if (value < 0 || value > kResidentShapes) return fail(PICARD_ERR_BAD_ARG, "SWEEP_RESIDENT must be 0..5");
    return set_resident(c, value);
  }
  if (option == PICARD_OPT_SWEEP_PAIRS) {
    c->G.pairs = value != 0;
    if (!c->G.pairs) c->G.fused2 = 0;
    return PICARD_OK;
  }
  if (option == PICARD_OPT_SWEEP_FUSED) {
    if (value && (!c->G.tma || c->G.zc > 8)) return fail(PICARD_ERR_STATE, "two-sweep launches need the TMA sweep with zc <= 8");
    c->G.fused2 = value != 0;
    if (c->G.fused2) c->G.pairs = 1;
    return PICARD_OK;
  }
  if (option == PICARD_OPT_SWEEP_STAGES) {
    if (value != 1 && value != 2) return fail(PICARD_ERR_BAD_ARG, "SWEEP_STAGES must be 1 or 2");
    c->G.stages = value;
    return PICARD_OK;
  }
  if (option == PICARD_OPT_SWEEP_R_GLOBAL) {
    c->G.rglobal = value != 0;
    if (c->G.rglobal) c->G.pairs = 1, c->G.fused2 = 0;
    return PICARD_OK;
  }
  if (option == PICARD_OPT_SORT_EVERY) {
    if (value < 0) return fail(PICARD_ERR_BAD_ARG, "SORT_EVERY must be >= 0");
    c->sort_every = value;
    return PICARD_OK;
  }
  if (option == PICARD_OPT_WAIT_TEST) {
    if (value != 0 && value != 1) return fail(PICARD_ERR_BAD_ARG, "WAIT_TEST must be 0 or 1");
    c->wait_test = value;
    return PICARD_OK;
  }
  return fail(PICARD_ERR_BAD_ARG, "unknown option");
}

int picard_gpu_get_option(picard_ctx* c, int32_t option, int32_t* value) {
  if (!c || !value) return fail(PICARD_ERR_BAD_ARG, "NULL argument");
  switch (option) {
    case PICARD_OPT_BCPOT_TENSOR: *value = c->bcpot_tensor; return PICARD_OK;
    case PICARD_OPT_SWEEP_CTAS: *value = c->G.ctas; return PICARD_OK;
    case PICARD_OPT_SWEEP_PDL: *value = c->G.pdl; return PICARD_OK;
    case PICARD_OPT_SWEEP_STAGES: *value = c->G.stages; return PICARD_OK;
    case PICARD_OPT_SWEEP_PAIRS: *value = c->G.pairs; return PICARD_OK;
    case PICARD_OPT_SWEEP_FUSED: *value = c->G.fused2; return PICARD_OK;
    case PICARD_OPT_SWEEP_RESIDENT: *value = resident_option_value(c); return PICARD_OK;
    case PICARD_OPT_WAIT_TEST: *value = c->wait_test; return PICARD_OK;
    case PICARD_OPT_SWEEP_R_GLOBAL: *value = c->G.rglobal; return PICARD_OK;
    case PICARD_OPT_SORT_EVERY: *value = c->sort_every; return PICARD_OK;
  }
  return fail(PICARD_ERR_BAD_ARG, "unknown option");
}

// BCpotentials.f90:1-145
int picard_gpu_bc_potentials(picard_ctx* c) {
  if (!c) return fail(PICARD_ERR_BAD_ARG, "ctx is NULL");
  PICARD_TRY(bc_potentials_async(c));
  return c->bcpot_tensor == PICARD_BCPOT_TENSOR ? check_dev_err_timeout(c) : PICARD_OK;
}

// CalcEfield.f90:3-232
int picard_gpu_calc_efield(picard_ctx* c) {
  if (!c) return fail(PICARD_ERR_BAD_ARG, "ctx is NULL");
  PICARD_CUDA(launch_efield(c->K, c->U, c->E, c->E32, c->st));
  return PICARD_OK;
}

// BCfields.f90:3-94: on one rank the open-face ghost layers of E are zero
// already (picard_gpu_calc_efield writes them); this re-zeroes them so the
// routine also holds after picard_gpu_set_field.
int picard_gpu_bc_fields(picard_ctx* c) {
  if (!c) return fail(PICARD_ERR_BAD_ARG, "ctx is NULL");
  PICARD_CUDA(launch_bc_fields(c->K, c->E, c->E32, c->st));
  return PICARD_OK;
}

static int advance_velocity(picard_ctx* c, double dt, double deltat, int mode) {
  if (!c) return fail(PICARD_ERR_BAD_ARG, "ctx is NULL");
  if (!(dt != 0.0)) return fail(PICARD_ERR_BAD_ARG, "dt must be nonzero");
  if (c->layout == PICARD_LAYOUT_F64)
    PICARD_CUDA(launch_advance_velocity_f64(c->K, c->f64, c->num_local, c->E, dt, deltat, mode, c->st));
  else
    PICARD_CUDA(launch_advance_velocity_c32(c->K, c->c32, c->num_local, c->E32, dt, deltat, mode, c->st));
  return PICARD_OK;
}

// AdvanceVelocity.f90:6-125
int picard_gpu_advance_velocity(picard_ctx* c, double dt) { return advance_velocity(c, dt, 0.0, 0); }
// AdvanceVelocity.f90:128-236
int picard_gpu_advance_velocity_exp(picard_ctx* c, double deltat, double dt) {
  return advance_velocity(c, dt, deltat, 1);
}
// AdvanceVelocity.f90:239-347
int picard_gpu_advance_velocity_imp(picard_ctx* c, double deltat, double dt) {
  return advance_velocity(c, dt, deltat, 2);
}

// picard.f90:651-665
int picard_gpu_energy(picard_ctx* c, double out[3], int32_t* num) {
  if (!c || !out) return fail(PICARD_ERR_BAD_ARG, "NULL argument");
  ReduceBuf rb{c->red_partial, c->red_result, c->red_blocks};
  if (c->layout == PICARD_LAYOUT_F64)
    PICARD_CUDA(launch_energy_particles_f64(c->K, c->f64, c->num_local, rb, c->st));
  else
    PICARD_CUDA(launch_energy_particles_c32(c->K, c->c32, c->num_local, rb, c->st));
  ReduceBuf rf{c->red_partial, c->red_result + 1, c->red_blocks};
  PICARD_CUDA(launch_energy_field(c->K, c->E, rf.partial, rf.result, c->st));
  PICARD_CUDA(cudaMemcpyAsync(c->h_pinned, c->red_result, 2 * sizeof(double), cudaMemcpyDeviceToHost, c->st));
  PICARD_CUDA(cudaStreamSynchronize(c->st));
  c->stats.d2h_bytes += 2 * sizeof(double);
  out[0] = c->h_pinned[0];
  out[1] = c->h_pinned[1];
  // B is uniform (updateBfield is not implemented in the reference)
  double b2 = 0.0;
  for (int c3 = 0; c3 < 3; ++c3) b2 += c->prm.B0[c3] * c->prm.B0[c3];
  double nodes = (double)c->prm.nx * c->prm.ny * c->prm.nz;
  out[2] = nodes * b2 * 0.5 / kMu0 * c->K.dV;
  if (num) *num = int32_t(c->num_local);
  return PICARD_OK;
}

}  // extern "C"
