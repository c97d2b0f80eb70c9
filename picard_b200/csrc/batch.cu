// batch.cu -- many independent runs advanced together (the batched
// parameter sweep): picard_batch_run_fused.
//
// Each run is its own picard_ctx (own memory, own stream).  Per iteration of
// picard.f90:554-674 the batched loop issues every run's particle phases on the
// runs' streams before waiting on any of them (the particle-count round trips
// of all runs travel together), then solves every run's Poisson problem in
// ticks: each run plans its rounds of sweeps from its own anchor (the
// F32_REFINE loop of solve_f32.cuh, unchanged), and one tick is ONE launch
// advancing every run that is in the middle of a round by one sweep -- the
// run table (tensor maps, stencil, coefficients, output, tile range) rides in
// the kernel parameters -- instead of one launch per run.  Anchors, reductions
// and the stop tests stay per run, asynchronous to the ticks; runs that
// converge drop out.  One launch per tick covers every run: each CTA takes
// the tile body of its run's class -- the x-pair TMA sweep, or the 32-wide one
// for runs whose x extent would leave half of a 64-wide tile empty -- with the
// same per-node arithmetic and per-tile partials as the single-run kernels,
// so every run's result is bit-identical to the same run advanced alone with
// picard_gpu_run_fused.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <functional>
#include <memory>
#include <mutex>
#include <thread>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "context.cuh"
#include "grid.cuh"
#include "kernels.cuh"
#include "picard_gpu.h"
#include "solve_f32.cuh"
#include "stencil.cuh"
#include "pair_tile.cuh"
#include "tile32.cuh"

using namespace picard;

namespace picard {
namespace {

constexpr int kBatchRuns = 40;  // runs per launch (kernel parameter space)
constexpr int kTicksAhead = 6;  // batched sweep launches queued ahead of the device
// Working set (w in, w out, the anchor residual: 12 B a node) of the runs that
// sweep together.  Kept within the L2 (126 MB) so that consecutive ticks find
// their tiles there instead of streaming every run from HBM on every sweep;
// the other runs wait, and join as runs of the set converge.
constexpr double kTickSetBytes = 80e6;
long long g_batch_ctas = 0;  // CTAs launched by batched sweeps (PICARD_BATCH_LOG)

// Host threads that issue the runs' per-run work in parallel (launches on the
// runs' own streams, waits on them), so that one host thread's launch rate and
// round trips do not bound a batch of many small runs.  run(n, fn) calls fn(r)
// for every r < n, run r on worker r % threads, and returns when all are done
// with the status of the lowest-numbered failing run (its message re-raised on
// the calling thread).  Each run's work stays in its own stream order, so the
// results do not depend on the thread count.
class RunPool {
 public:
  RunPool(int threads, int device) : T_(threads), device_(device) {
    for (int w = 1; w < T_; ++w) th_.emplace_back([this, w]() { worker(w); });
  }
  ~RunPool() {
    {
      std::lock_guard<std::mutex> lk(mu_);
      stop_ = true;
    }
    cv_.notify_all();
    for (std::thread& t : th_) t.join();
  }
  int run(int n, const std::function<int(int)>& fn) {
    rc_.assign(n, PICARD_OK);
    msg_.assign(n, std::string());
    {
      std::lock_guard<std::mutex> lk(mu_);
      fn_ = &fn;
      n_ = n;
      pending_ = T_ - 1;
      ++gen_;
    }
    cv_.notify_all();
    slice(0);  // the calling thread is worker 0
    {
      std::unique_lock<std::mutex> lk(mu_);
      done_cv_.wait(lk, [&]() { return pending_ == 0; });
    }
    for (int r = 0; r < n; ++r)
      if (rc_[r] != PICARD_OK) return fail(rc_[r], msg_[r]);
    return PICARD_OK;
  }

 private:
  void slice(int w) {
    for (int r = w; r < n_; r += T_) {
      const int q = (*fn_)(r);
      if (q != PICARD_OK) {
        rc_[r] = q;
        msg_[r] = picard_gpu_last_error();
      }
    }
  }
  void worker(int w) {
    cudaSetDevice(device_);
    long long seen = 0;
    for (;;) {
      {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait(lk, [&]() { return stop_ || gen_ != seen; });
        if (stop_) return;
        seen = gen_;
      }
      slice(w);
      {
        std::lock_guard<std::mutex> lk(mu_);
        if (--pending_ == 0) done_cv_.notify_one();
      }
    }
  }
  const int T_, device_;
  std::vector<std::thread> th_;
  std::mutex mu_;
  std::condition_variable cv_, done_cv_;
  const std::function<int(int)>* fn_ = nullptr;
  int n_ = 0, pending_ = 0;
  long long gen_ = 0;
  bool stop_ = false;
  std::vector<int> rc_;
  std::vector<std::string> msg_;
};

// Pools kept between batched calls (the continuous-batching server calls the
// batched step once per iteration): a call takes a pool of its device and
// thread count from the cache, or makes one, and puts it back when done.
std::mutex g_pool_mu;
std::vector<std::pair<std::pair<int, int>, std::unique_ptr<RunPool>>> g_pools;

std::unique_ptr<RunPool> take_pool(int device, int threads) {
  {
    std::lock_guard<std::mutex> lk(g_pool_mu);
    for (auto it = g_pools.begin(); it != g_pools.end(); ++it)
      if (it->first == std::make_pair(device, threads)) {
        std::unique_ptr<RunPool> p = std::move(it->second);
        g_pools.erase(it);
        return p;
      }
  }
  return std::unique_ptr<RunPool>(new RunPool(threads, device));
}

void give_pool(int device, int threads, std::unique_ptr<RunPool> p) {
  std::lock_guard<std::mutex> lk(g_pool_mu);
  g_pools.emplace_back(std::make_pair(device, threads), std::move(p));
}

struct alignas(64) BatchRun {
  CUtensorMap tw;  // w of the sweep's input iterate (boxes 72 x 10 x zc+2; 32-wide tiles 40 x 10 x zc+2)
  CUtensorMap tr;  // the run's live anchor residual (boxes 64 x 8 x zc; 32-wide tiles 32 x 8 x zc)
  Stencil S;
  JacobiCoefF J;
  float* wout;
  double* partial;
  int gx2, gx, gy, tiles, tile_base, w_zero;
  int zc, w32;  // the run's tile depth and width (sweep_batch_any_kernel)
};

struct BatchArgs {
  BatchRun run[kBatchRuns];
  int nruns;
  int total_tiles;
  int* err;
};
static_assert(sizeof(BatchArgs) < 32000, "kernel parameter space");

// The run whose tile range holds CTA t: the last r with tile_base <= t (the
// bases are cumulative, so non-decreasing).  A binary search: the lookup sits
// before the tile's TMA issue, on every tile's critical path.
__device__ __forceinline__ int batch_run_of(const BatchArgs& A, int t) {
  int lo = 0, hi = A.nruns - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (A.run[mid].tile_base <= t)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

// The x-pair sweep (pair_tile.cuh, as in grid.cu sweep_tma2_kernel) over a
// table of runs: CTA t takes tile t - tile_base of the run whose tile range
// holds t.
template <int ZC>
__global__ void __launch_bounds__(256) sweep_batch_kernel(const __grid_constant__ BatchArgs A) {
  constexpr int kBoxX = 72, kTile = 64, kTy = 8, kTx = 32;
  constexpr int kW = (ZC + 2) * (kTy + 2) * kBoxX, kR = ZC * kTy * kTile;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  float* sw = reinterpret_cast<float*>(smem_raw);
  float* sr = sw + kW;
  __shared__ __align__(8) unsigned long long mbar;
  __shared__ double rows[2][kTy];
  const int tx = threadIdx.x, ty = threadIdx.y, tid = tx + kTx * ty;
  const int t = blockIdx.x;
  const int r = batch_run_of(A, t);
  const BatchRun& R = A.run[r];
  const int lt = t - R.tile_base;
  const uint32_t mb = (uint32_t)__cvta_generic_to_shared(&mbar);
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mb) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  const int bx2 = lt % R.gx2, by = (lt / R.gx2) % R.gy, bz = lt / (R.gx2 * R.gy);
  const int x0 = bx2 * kTile, y0 = by * kTy, z0 = bz * ZC;
  if (tid == 0) {
    uint32_t bytes = (uint32_t)(kR * sizeof(float));
    if (!R.w_zero) bytes += (uint32_t)(kW * sizeof(float));
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mb), "r"(bytes) : "memory");
    if (!R.w_zero)
      asm volatile(
          "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
          ::"r"((uint32_t)__cvta_generic_to_shared(sw)), "l"((unsigned long long)&R.tw), "r"(x0), "r"(y0), "r"(z0),
          "r"(mb)
          : "memory");
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
        ::"r"((uint32_t)__cvta_generic_to_shared(sr)), "l"((unsigned long long)&R.tr), "r"(x0 + 4), "r"(y0 + 1),
        "r"(z0 + 1), "r"(mb)
        : "memory");
  }
  bool done = false;
  for (long long it = 0; it < (1LL << 24); ++it) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(mb), "r"(0u)
        : "memory");
    if (ok) {
      done = true;
      break;
    }
  }
  if (!__syncthreads_and(done ? 1 : 0)) {
    if (tid == 0) atomicCAS(A.err, 0, int(kDevTimeout));
    // let this CTA's copies land (bounded) before it exits
    for (long long it = 0; it < (1LL << 24); ++it) {
      uint32_t ok;
      asm volatile(
          "{\n\t.reg .pred p;\n\t"
          "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
          "selp.u32 %0, 1, 0, p;\n\t}"
          : "=r"(ok)
          : "r"(mb), "r"(0u)
          : "memory");
      if (ok) break;
    }
    return;
  }
  pair_tile_sweep<ZC>(sw, sr, R.S, R.J, R.wout, R.partial, R.w_zero, bx2, by, bz, R.gx, R.gy, rows);
}

// The 32-wide tile body (tile32.cuh, as in grid.cu sweep_tma_kernel) over a
// table of runs, for runs whose x extent would leave half of a 64-wide tile
// empty.
template <int ZC>
__global__ void __launch_bounds__(256) sweep_batch32_kernel(const __grid_constant__ BatchArgs A) {
  constexpr int kW = (ZC + 2) * (kT32Ty + 2) * kT32BoxX, kR = ZC * kT32Ty * kT32Tx;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  float* sw = reinterpret_cast<float*>(smem_raw);
  float* sr = sw + kW;
  __shared__ __align__(8) unsigned long long mbar;
  const int tid = threadIdx.x + kT32Tx * threadIdx.y;
  const int t = blockIdx.x;
  const int r = batch_run_of(A, t);
  const BatchRun& R = A.run[r];
  const int lt = t - R.tile_base;
  const uint32_t mb = (uint32_t)__cvta_generic_to_shared(&mbar);
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mb) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  const int bx = lt % R.gx, by = (lt / R.gx) % R.gy, bz = lt / (R.gx * R.gy);
  const int x0 = bx * kT32Tx, y0 = by * kT32Ty, z0 = bz * ZC;
  if (tid == 0) {
    uint32_t bytes = (uint32_t)(kR * sizeof(float));
    if (!R.w_zero) bytes += (uint32_t)(kW * sizeof(float));
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mb), "r"(bytes) : "memory");
    if (!R.w_zero)
      asm volatile(
          "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
          ::"r"((uint32_t)__cvta_generic_to_shared(sw)), "l"((unsigned long long)&R.tw), "r"(x0), "r"(y0), "r"(z0),
          "r"(mb)
          : "memory");
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
        ::"r"((uint32_t)__cvta_generic_to_shared(sr)), "l"((unsigned long long)&R.tr), "r"(x0 + 4), "r"(y0 + 1),
        "r"(z0 + 1), "r"(mb)
        : "memory");
  }
  bool done = false;
  for (long long it = 0; it < (1LL << 24); ++it) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(mb), "r"(0u)
        : "memory");
    if (ok) {
      done = true;
      break;
    }
  }
  if (!__syncthreads_and(done ? 1 : 0)) {
    if (tid == 0) atomicCAS(A.err, 0, int(kDevTimeout));
    for (long long it = 0; it < (1LL << 24); ++it) {
      uint32_t ok;
      asm volatile(
          "{\n\t.reg .pred p;\n\t"
          "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
          "selp.u32 %0, 1, 0, p;\n\t}"
          : "=r"(ok)
          : "r"(mb), "r"(0u)
          : "memory");
      if (ok) break;
    }
    return;
  }
  tile32_sweep<ZC>(sw, sr, R.S, R.J, R.wout, R.partial + (bx + (long long)R.gx * (by + (long long)R.gy * bz)),
                   R.w_zero, bx, by, bz);
}

// Bounded wait for a CTA's TMA boxes; false (after recording kDevTimeout and
// letting the copies land, also bounded) when they did not arrive.
__device__ inline bool batch_wait_boxes(uint32_t mb, int tid, int* err) {
  bool done = false;
  for (long long it = 0; it < (1LL << 24); ++it) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(mb), "r"(0u)
        : "memory");
    if (ok) {
      done = true;
      break;
    }
  }
  if (__syncthreads_and(done ? 1 : 0)) return true;
  if (tid == 0) atomicCAS(err, 0, int(kDevTimeout));
  for (long long it = 0; it < (1LL << 24); ++it) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(mb), "r"(0u)
        : "memory");
    if (ok) break;
  }
  return false;
}

// Issue one tile's w and r boxes (w only when the entering iterate is not zero).
__device__ inline void batch_issue_boxes(const BatchRun& R, uint32_t mb, float* sw, float* sr, uint32_t wbytes,
                                         uint32_t rbytes, int x0, int y0, int z0) {
  uint32_t bytes = rbytes;
  if (!R.w_zero) bytes += wbytes;
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mb), "r"(bytes) : "memory");
  if (!R.w_zero)
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
        ::"r"((uint32_t)__cvta_generic_to_shared(sw)), "l"((unsigned long long)&R.tw), "r"(x0), "r"(y0), "r"(z0),
        "r"(mb)
        : "memory");
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
      ::"r"((uint32_t)__cvta_generic_to_shared(sr)), "l"((unsigned long long)&R.tr), "r"(x0 + 4), "r"(y0 + 1),
      "r"(z0 + 1), "r"(mb)
      : "memory");
}

// Tile lt of run R with the x-pair body (64 x 8 x ZC).
template <int ZC>
__device__ inline void batch_pair_tile(const BatchRun& R, int lt, float* smem, uint32_t mb, int tid, int* err,
                                       double (*rows)[8]) {
  constexpr int kW = (ZC + 2) * 10 * 72, kR = ZC * 8 * 64;
  float* sw = smem;
  float* sr = smem + kW;
  const int bx2 = lt % R.gx2, by = (lt / R.gx2) % R.gy, bz = lt / (R.gx2 * R.gy);
  if (tid == 0) batch_issue_boxes(R, mb, sw, sr, kW * 4u, kR * 4u, bx2 * 64, by * 8, bz * ZC);
  if (!batch_wait_boxes(mb, tid, err)) return;
  pair_tile_sweep<ZC>(sw, sr, R.S, R.J, R.wout, R.partial, R.w_zero, bx2, by, bz, R.gx, R.gy, rows);
}

// Tile lt of run R with the 32-wide body (32 x 8 x ZC).
template <int ZC>
__device__ inline void batch_w32_tile(const BatchRun& R, int lt, float* smem, uint32_t mb, int tid, int* err) {
  constexpr int kW = (ZC + 2) * (kT32Ty + 2) * kT32BoxX, kR = ZC * kT32Ty * kT32Tx;
  float* sw = smem;
  float* sr = smem + kW;
  const int bx = lt % R.gx, by = (lt / R.gx) % R.gy, bz = lt / (R.gx * R.gy);
  if (tid == 0) batch_issue_boxes(R, mb, sw, sr, kW * 4u, kR * 4u, bx * kT32Tx, by * kT32Ty, bz * ZC);
  if (!batch_wait_boxes(mb, tid, err)) return;
  tile32_sweep<ZC>(sw, sr, R.S, R.J, R.wout, R.partial + (bx + (long long)R.gx * (by + (long long)R.gy * bz)),
                   R.w_zero, bx, by, bz);
}

// One tick over runs of every class -- tile depth 4 or 8, x-pair or 32-wide
// tiles -- in ONE launch: CTA t finds its run and takes the body of that run's
// class, so a tick pays one dependent-launch floor instead of one per class.
// Each run's tiles, arithmetic and partials are those of its class's own
// kernel: the same bits.  Dynamic shared memory is the largest class's in the
// launch.
__global__ void __launch_bounds__(256, 8) sweep_batch_any_kernel(const __grid_constant__ BatchArgs A) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  float* smem = reinterpret_cast<float*>(smem_raw);
  __shared__ __align__(8) unsigned long long mbar;
  __shared__ double rows[2][8];
  const int tid = threadIdx.x + 32 * threadIdx.y;
  const int t = blockIdx.x;
  const int r = batch_run_of(A, t);
  const BatchRun& R = A.run[r];
  const int lt = t - R.tile_base;
  const uint32_t mb = (uint32_t)__cvta_generic_to_shared(&mbar);
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mb) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  if (R.w32) {
    if (R.zc == 8)
      batch_w32_tile<8>(R, lt, smem, mb, tid, A.err);
    else
      batch_w32_tile<4>(R, lt, smem, mb, tid, A.err);
  } else {
    if (R.zc == 8)
      batch_pair_tile<8>(R, lt, smem, mb, tid, A.err, rows);
    else
      batch_pair_tile<4>(R, lt, smem, mb, tid, A.err, rows);
  }
}

// Shared memory of one tile of a class.
inline size_t batch_class_smem(int zc, bool w32) {
  return w32 ? sizeof(float) * ((size_t)(zc + 2) * 10 * 40 + (size_t)zc * 8 * 32)
             : sizeof(float) * ((size_t)(zc + 2) * 10 * 72 + (size_t)zc * 8 * 64);
}

cudaError_t launch_batch_any(const BatchArgs& A, size_t smem, int pdl, cudaStream_t st) {
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(sweep_batch_any_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)batch_class_smem(8, false));
    if (e != cudaSuccess) return e;
    attr = true;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(A.total_tiles);
  cfg.blockDim = dim3(32, 8);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = pdl;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  note_launch();
  return cudaLaunchKernelEx(&cfg, sweep_batch_any_kernel, A);
}

template <int ZC>
cudaError_t launch_batch32_zc(const BatchArgs& A, int pdl, cudaStream_t st) {
  constexpr size_t smem = sizeof(float) * ((size_t)(ZC + 2) * 10 * 40 + (size_t)ZC * 8 * 32);
  static bool attr = false;
  if (!attr) {
    cudaError_t e =
        cudaFuncSetAttribute(sweep_batch32_kernel<ZC>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(A.total_tiles);
  cfg.blockDim = dim3(32, 8);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = pdl;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  note_launch();
  return cudaLaunchKernelEx(&cfg, sweep_batch32_kernel<ZC>, A);
}

template <int ZC>
cudaError_t launch_batch_zc(const BatchArgs& A, int pdl, cudaStream_t st) {
  constexpr size_t smem = sizeof(float) * ((size_t)(ZC + 2) * 10 * 72 + (size_t)ZC * 8 * 64);
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(sweep_batch_kernel<ZC>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(A.total_tiles);
  cfg.blockDim = dim3(32, 8);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = pdl;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  note_launch();
  return cudaLaunchKernelEx(&cfg, sweep_batch_kernel<ZC>, A);
}

struct RunSolve {
  picard_ctx* c = nullptr;
  EpotSetup e;
  F32Solve S;
  SpecSolve Q;           // SOLVER_SPECTRAL: the closed-form solve
  bool spectral = false;
  bool batched = false;  // the batched loop drives this run's solve
  bool active = false;   // in the set of runs that sweep together
  bool w32 = false;      // 32-wide tiles (tile32.cuh) instead of 64-wide x pairs
  bool done = true;
  int phase = 0;         // 0 round to plan, 1 sweeping, 2 anchor and stop test in flight
  int p = 0;             // sweeps of the current round done
  long long sweeps = 0;
  bool converged = true;
};

// One tick: the next sweep of every run in the middle of a round, in
// launches of at most kBatchRuns runs of one tile depth.  Runs whose round is
// complete after the tick are appended to `ended`.  pdl: the tick may overlap
// the previous one on the batch stream (griddepcontrol.wait orders it after
// its predecessor there); the first tick of a solve phase follows event waits
// on the runs' streams, which PDL would not cover, so it is a plain launch.
int launch_tick(std::vector<RunSolve*>& runs, int* err, cudaStream_t st, bool pdl, std::vector<RunSolve*>& ended,
                long long* launches, int unified) {
  bool first = !pdl;
  // unified 1: one launch per tile depth (the x-pair and 32-wide runs of that
  // depth together); 2: one launch for every class
  for (int zgroup = 0; unified && zgroup < (unified == 2 ? 1 : 2); ++zgroup) {
    BatchArgs A;
    std::memset(&A, 0, sizeof(A));
    A.err = err;
    size_t smem = 0;
    auto flush = [&]() -> int {
      if (A.nruns == 0) return PICARD_OK;
      PICARD_CUDA(launch_batch_any(A, smem, first ? 0 : 1, st));
      first = false;
      ++*launches;
      g_batch_ctas += A.total_tiles;
      std::memset(&A, 0, sizeof(A));
      A.err = err;
      smem = 0;
      return PICARD_OK;
    };
    for (RunSolve* rs : runs) {
      if (rs->done || !rs->batched || rs->phase != 1) continue;
      if (unified == 1 && rs->c->G.zc != (zgroup ? 8 : 4)) continue;
      picard_ctx* c = rs->c;
      const bool w32 = rs->w32;
      const int t = rs->p + 1;                  // sweep t of the round
      const int in = rs->S.wcur, out = 1 - in;  // never write the buffer being read
      BatchRun& R = A.run[A.nruns];
      R.tw = w32 ? c->tmw[in] : c->tmw2[in];
      R.tr = w32 ? c->tmr[rs->S.rcur] : c->tmr2[rs->S.rcur];
      R.S = make_stencil(c->K);
      R.J = jacobi_coef_f(c->K);
      R.wout = c->w[out];
      rs->S.wcur = out;
      R.partial = c->partials + (size_t)(t - 1) * c->G.nblocks;
      R.gx2 = (c->K.nx + 63) / 64;
      R.gx = (int)c->G.grid.x;
      R.gy = (int)c->G.grid.y;
      R.tiles = (w32 ? R.gx : R.gx2) * (int)c->G.grid.y * (int)c->G.grid.z;
      R.tile_base = A.total_tiles;
      R.w_zero = t == 1 ? 1 : 0;
      R.zc = c->G.zc;
      R.w32 = w32 ? 1 : 0;
      smem = std::max(smem, batch_class_smem(c->G.zc, w32));
      A.total_tiles += R.tiles;
      rs->p = t;
      if (t == rs->S.m_eff) ended.push_back(rs);
      if (++A.nruns == kBatchRuns) PICARD_TRY(flush());
    }
    PICARD_TRY(flush());
  }
  if (unified) return PICARD_OK;
  for (int cls = 0; cls < 4; ++cls) {
    const int zc = cls & 1 ? 8 : 4;
    const bool w32 = cls >= 2;
    BatchArgs A;
    std::memset(&A, 0, sizeof(A));
    A.err = err;
    auto flush = [&]() -> int {
      if (A.nruns == 0) return PICARD_OK;
      const int use_pdl = first ? 0 : 1;
      first = false;
      cudaError_t e = w32 ? (zc == 8 ? launch_batch32_zc<8>(A, use_pdl, st) : launch_batch32_zc<4>(A, use_pdl, st))
                          : (zc == 8 ? launch_batch_zc<8>(A, use_pdl, st) : launch_batch_zc<4>(A, use_pdl, st));
      PICARD_CUDA(e);
      ++*launches;
      g_batch_ctas += A.total_tiles;
      std::memset(&A, 0, sizeof(A));
      A.err = err;
      return PICARD_OK;
    };
    for (RunSolve* rs : runs) {
      if (rs->done || !rs->batched || rs->phase != 1 || rs->c->G.zc != zc || rs->w32 != w32) continue;
      picard_ctx* c = rs->c;
      const int t = rs->p + 1;                  // sweep t of the round
      const int in = rs->S.wcur, out = 1 - in;  // never write the buffer being read
      BatchRun& R = A.run[A.nruns];
      R.tw = w32 ? c->tmw[in] : c->tmw2[in];
      R.tr = w32 ? c->tmr[rs->S.rcur] : c->tmr2[rs->S.rcur];
      R.S = make_stencil(c->K);
      R.J = jacobi_coef_f(c->K);
      R.wout = c->w[out];
      rs->S.wcur = out;
      R.partial = c->partials + (size_t)(t - 1) * c->G.nblocks;
      R.gx2 = (c->K.nx + 63) / 64;
      R.gx = (int)c->G.grid.x;
      R.gy = (int)c->G.grid.y;
      R.tiles = (w32 ? R.gx : R.gx2) * (int)c->G.grid.y * (int)c->G.grid.z;
      R.tile_base = A.total_tiles;
      R.w_zero = t == 1 ? 1 : 0;
      A.total_tiles += R.tiles;
      rs->p = t;
      if (t == rs->S.m_eff) ended.push_back(rs);
      if (++A.nruns == kBatchRuns) PICARD_TRY(flush());
    }
    PICARD_TRY(flush());
  }
  return PICARD_OK;
}

}  // namespace
}  // namespace picard

namespace {

// nsteps iterations of every run; run r takes iterations it0[r]+1 .. it0[r]+nsteps.
int batch_run_impl(picard_ctx** ctxs, int32_t n, const int32_t* it0, int32_t nsteps, int64_t* sweeps_total) {
  if (!ctxs || n < 1) return fail(PICARD_ERR_BAD_ARG, "no contexts");
  for (int r = 0; r < n; ++r) {
    if (!ctxs[r]) return fail(PICARD_ERR_BAD_ARG, "a context is NULL");
    for (int q = 0; q < r; ++q)
      if (ctxs[q] == ctxs[r]) return fail(PICARD_ERR_BAD_ARG, "a context appears twice in the batch");
  }
  int dev = 0;
  PICARD_CUDA(cudaGetDevice(&dev));
  for (int r = 0; r < n; ++r)
    if (ctxs[r]->device != dev) return fail(PICARD_ERR_BAD_ARG, "batched contexts must live on the current device");
  cudaStream_t bst = nullptr;
  cudaEvent_t bev = nullptr;
  std::vector<cudaEvent_t> rev(n, nullptr), dev_ev(n, nullptr);
  cudaEvent_t tick_ev[kTicksAhead] = {};
  auto cleanup = [&]() {
    if (bst) cudaStreamSynchronize(bst);
    for (int r = 0; r < n; ++r) {
      if (rev[r]) cudaEventDestroy(rev[r]);
      if (dev_ev[r]) cudaEventDestroy(dev_ev[r]);
    }
    if (bev) cudaEventDestroy(bev);
    for (cudaEvent_t& e : tick_ev)
      if (e) cudaEventDestroy(e);
    if (bst) cudaStreamDestroy(bst);
  };
  int rc = PICARD_OK;
  int* berr = nullptr;  // timeout flag of the batched sweeps (run 0's error word)
  rc = check_cuda(cudaStreamCreateWithFlags(&bst, cudaStreamNonBlocking), "cudaStreamCreate");
  if (rc == PICARD_OK) rc = check_cuda(cudaEventCreateWithFlags(&bev, cudaEventDisableTiming), "cudaEventCreate");
  for (cudaEvent_t& e : tick_ev)
    if (rc == PICARD_OK) rc = check_cuda(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate");
  for (int r = 0; r < n && rc == PICARD_OK; ++r) {
    rc = check_cuda(cudaEventCreateWithFlags(&rev[r], cudaEventDisableTiming), "cudaEventCreate");
    if (rc == PICARD_OK) rc = check_cuda(cudaEventCreateWithFlags(&dev_ev[r], cudaEventDisableTiming), "cudaEventCreate");
  }
  if (rc != PICARD_OK) {
    cleanup();
    return rc;
  }
  berr = ctxs[0]->d_err;
  std::atomic<bool> nc{false};
  // PICARD_BATCH_THREADS: host threads issuing the per-run work (default
  // min(runs, 8); 1: the calling thread alone)
  const char* thv = std::getenv("PICARD_BATCH_THREADS");
  const int threads = std::max(1, std::min(n, thv && *thv ? std::atoi(thv) : 8));
  std::unique_ptr<RunPool> pool_owner = take_pool(dev, threads);
  RunPool& pool = *pool_owner;
  struct PoolReturn {
    int dev, threads;
    std::unique_ptr<RunPool>& p;
    ~PoolReturn() { give_pool(dev, threads, std::move(p)); }
  } pool_return{dev, threads, pool_owner};
  std::vector<RunSolve> solves(n);
  std::vector<RunSolve*> rp(n);
  for (int r = 0; r < n; ++r) rp[r] = &solves[r];

  // PICARD_BATCH_W32 (default 1): 32-wide tiles for runs whose x extent
  // leaves half of a 64-wide tile empty; 0 x-pair tiles for every run.
  const char* w32v = std::getenv("PICARD_BATCH_W32");
  const bool tile_w32 = !(w32v && *w32v == '0');
  // PICARD_BATCH_UNIFIED: 2 (the default) one launch per tick for every tile
  // class (sweep_batch_any_kernel); 1 one launch per tick and tile depth; 0 one
  // launch per tick and tile class (sweep_batch_kernel, sweep_batch32_kernel).
  // Measured on the 64-run set (64 runs of 16..96^3, 20 steps): Jacobi 10.84 s
  // (2, 32-wide tiles on), 11.04 s (1), 11.33 s (0, x-pair tiles only), 11.82 s
  // (0 with 32-wide tiles: their extra launch class per tick costs more than
  // the lanes they save).
  const char* univ = std::getenv("PICARD_BATCH_UNIFIED");
  const int tick_unified = univ && *univ ? std::atoi(univ) : 2;
  // PICARD_BATCH_SET_MB: working-set budget of the runs that sweep together
  const char* setv = std::getenv("PICARD_BATCH_SET_MB");
  const double tick_set_bytes = setv && *setv ? std::atof(setv) * 1e6 : kTickSetBytes;
  // PICARD_BATCH_LOG=1: host time per phase (waits for the device included)
  const char* logv = std::getenv("PICARD_BATCH_LOG");
  const bool log = logv && *logv && *logv != '0';
  double ph[6] = {0, 0, 0, 0, 0, 0};
  long long rounds = 0, launches = 0, ticks = 0;
  g_batch_ctas = 0;
  auto now = []() { return std::chrono::steady_clock::now(); };
  auto tick = now();
  auto lap = [&](int k) {
    auto t = now();
    ph[k] += std::chrono::duration<double, std::milli>(t - tick).count();
    tick = t;
  };
  auto body = [&]() -> int {
    for (int32_t step = 1; step <= nsteps; ++step) {
      tick = now();
      // ---- AdvancePosition, ParticlesProduce (device count) for every run
      PICARD_TRY(pool.run(n, [&](int r) -> int {
        picard_ctx* c = ctxs[r];
        const KParams& K = c->K;
        const int cells = c->prm.nx * c->prm.ny * c->prm.nz;
        // CELL32 runs after their first step: the previous step's push advanced them
        if (step == 1 || c->layout != PICARD_LAYOUT_CELL32) PICARD_TRY(picard_gpu_advance_position(c, c->prm.dt));
        const int32_t it = it0[r] + step;
        PICARD_CUDA(launch_produce_count(K, it, c->cell_counts, c->st));
        PICARD_CUDA(launch_scan_int(c->cell_counts, c->cell_offsets, cells, c->cell_offsets + cells,
                                    c->cell_offsets + cells + 2, c->st));
        if (c->layout == PICARD_LAYOUT_F64)
          PICARD_CUDA(launch_produce_emit_f64(K, it, c->cell_offsets, c->f64, c->d_count,
                                              c->capacity, c->d_err, c->st));
        else
          PICARD_CUDA(launch_produce_emit_c32(K, it, c->cell_offsets, c->c32, c->d_count,
                                              c->capacity, c->d_err, c->st));
        PICARD_TRY(count_issue(c));
        return count_collect(c);
      }));
      lap(0);
      // ---- BCoutflow + ParticlesTransfer (in place), BCinflow (fused)
      PICARD_TRY(pool.run(n, [&](int r) -> int {
        picard_ctx* c = ctxs[r];
        const int32_t it = it0[r] + step;
        PICARD_CUDA(launch_outflow(c, 1));
        PICARD_CUDA(launch_inflow_fused(c, it));
        PICARD_TRY(count_issue(c));
        return count_collect(c);
      }));
      lap(1);
      // ---- ParticlesGridify, BCpotentials (FFT runs: one launch per stage
      // for all of them), b and ||b||
      PICARD_TRY(pool.run(n, [&](int r) -> int { return picard_gpu_particles_gridify(ctxs[r]); }));
      PICARD_TRY(bc_potentials_batch(ctxs, n, bst, rev.data(), bev));
      PICARD_TRY(pool.run(n, [&](int r) -> int {
        PICARD_TRY(epot_rhs_issue(ctxs[r]));
        PICARD_CUDA(cudaStreamSynchronize(ctxs[r]->st));
        return PICARD_OK;
      }));
      lap(2);
      // ---- CalcEpotential: closed-form solves and solves of their own
      // issued per run in parallel; FP32 runs in lockstep ticks below
      PICARD_TRY(pool.run(n, [&](int r) -> int {
        picard_ctx* c = ctxs[r];
        RunSolve& rs = solves[r];
        rs = RunSolve();
        rs.c = c;
        rs.e = epot_setup(c, c->prm.maxerr, c->prm.maxit);
        rs.done = rs.e.trivial;
        rs.sweeps = 0;
        rs.converged = true;
        if (rs.done) return PICARD_OK;
        if (c->solver == PICARD_SOLVER_SPECTRAL) {
          // closed form: queued now, its Parseval evaluations collected for
          // every such run together below
          rs.spectral = true;
          PICARD_TRY(spec_begin(rs.Q, c, rs.e.tol, rs.e.smax, rs.e.maxit));
        } else if (c->solver == PICARD_SOLVER_F32_REFINE && c->G.tma && c->G.zc <= 8) {
          rs.batched = true;
          // 32-wide tiles when 64-wide ones would leave a 32-column half empty
          rs.w32 = tile_w32 && ((c->K.nx + 31) / 32) % 2 == 1;
          PICARD_TRY(f32_begin(rs.S, c, rs.e.tol, rs.e.smax, rs.e.maxit, rs.e.sigma));
        } else {
          // not batchable (FP64 solver or periodic axes): its own solve
          int32_t sw = 0;
          int q = picard_gpu_calc_epotential(c, c->prm.maxerr, c->prm.maxit, &sw);
          if (q == PICARD_ERR_NOT_CONVERGED) nc = true;
          else if (q != PICARD_OK) return q;
          if (sweeps_total) sweeps_total[r] += sw;
          rs.done = true;
          rs.batched = false;
          rs.e.trivial = false;
        }
        return PICARD_OK;
      }));
      // Rounds are asynchronous across runs: every tick advances each run in
      // the middle of a round by one sweep; a run whose round ends gets its
      // anchor, reduction and stop test on its own stream while the ticks go
      // on for the others, and starts its next round once the host has its
      // decision (its anchor then is complete, so later ticks need no wait).
      for (int r = 0; r < n; ++r)
        if (solves[r].batched && !solves[r].done) {
          PICARD_CUDA(cudaEventRecord(rev[r], ctxs[r]->st));  // anchor 0
          PICARD_CUDA(cudaStreamWaitEvent(bst, rev[r], 0));
        }
      bool first_tick = true;
      std::vector<RunSolve*> ended;
      long long issued = 0, retired = 0;  // ticks queued / known complete
      // runs join the sweeping set largest first (they need the most sweeps),
      // within the working-set budget
      std::vector<int> order;
      for (int r = 0; r < n; ++r)
        if (solves[r].batched && !solves[r].done) order.push_back(r);
      std::stable_sort(order.begin(), order.end(),
                       [&](int a, int b) { return ctxs[a]->K.nodes > ctxs[b]->K.nodes; });
      size_t next_join = 0;
      double set_bytes = 0.0;
      for (;;) {
        for (int r = 0; r < n; ++r) {
          RunSolve& rs = solves[r];
          if (rs.active && rs.done) {
            rs.active = false;
            set_bytes -= 12.0 * double(ctxs[r]->K.nodes);
          }
        }
        while (next_join < order.size()) {
          const double b = 12.0 * double(ctxs[order[next_join]]->K.nodes);
          if (set_bytes > 0.0 && set_bytes + b > tick_set_bytes) break;
          solves[order[next_join]].active = true;
          set_bytes += b;
          ++next_join;
        }
        int sweeping = 0, waiting = 0;
        for (int r = 0; r < n; ++r) {
          RunSolve& rs = solves[r];
          if (rs.done || !rs.batched || !rs.active) continue;
          if (rs.phase == 0) {
            f32_plan(rs.S);
            rs.phase = 1;
            rs.p = 0;
            ++rounds;
          }
          sweeping += rs.phase == 1;
          waiting += rs.phase == 2;
        }
        if (sweeping == 0 && waiting == 0 && next_join == order.size()) break;
        if (sweeping > 0) {
          // keep at most kTicksAhead ticks queued, so that a run whose stop
          // test the host has just read joins the ticks right away instead of
          // behind a long queue
          if (issued - retired == kTicksAhead) {
            PICARD_CUDA(cudaEventSynchronize(tick_ev[retired % kTicksAhead]));
            ++retired;
          }
          ended.clear();
          PICARD_TRY(launch_tick(rp, berr, bst, !first_tick, ended, &launches, tick_unified));
          ++ticks;
          first_tick = false;
          PICARD_CUDA(cudaEventRecord(tick_ev[issued % kTicksAhead], bst));
          ++issued;
          for (RunSolve* rs : ended) {
            const int r = int(rs - solves.data());
            PICARD_CUDA(cudaEventRecord(rev[r], bst));
            PICARD_CUDA(cudaStreamWaitEvent(ctxs[r]->st, rev[r], 0));
            PICARD_CUDA(cudaEventRecord(ctxs[r]->ev[0], ctxs[r]->st));  // no per-run sweep timing in a batch
            PICARD_TRY(f32_issue_tail(rs->S));
            PICARD_CUDA(cudaEventRecord(dev_ev[r], ctxs[r]->st));
            rs->phase = 2;
          }
        }
        // collect the stop tests that have landed (block when nothing else can move)
        for (int r = 0; r < n; ++r) {
          RunSolve& rs = solves[r];
          if (rs.done || !rs.batched || !rs.active || rs.phase != 2) continue;
          cudaError_t q = sweeping > 0 ? cudaEventQuery(dev_ev[r]) : cudaEventSynchronize(dev_ev[r]);
          if (q == cudaErrorNotReady) continue;
          PICARD_CUDA(q);
          PICARD_TRY(f32_finish(rs.S, false));
          if (rs.S.done) {
            rs.done = true;
            rs.sweeps = rs.S.sweeps;
            rs.converged = rs.S.converged;
          } else {
            rs.phase = 0;
          }
          if (sweeping == 0) break;  // one at a time while blocking: replan at once
        }
      }
      // closed-form solves: each worker takes its runs' Parseval evaluations
      // in turn, one host round trip per evaluation for all of them
      PICARD_TRY(pool.run(threads, [&](int w) -> int {
        for (bool pending = true; pending;) {
          pending = false;
          for (int r = w; r < n; r += threads) {
            RunSolve& rs = solves[r];
            if (!rs.spectral || rs.done) continue;
            PICARD_CUDA(cudaStreamSynchronize(ctxs[r]->st));
            if (rs.Q.done) {
              spec_account(rs.Q);
              rs.done = true;
              rs.sweeps = rs.Q.d;
              rs.converged = rs.Q.converged;
              continue;
            }
            PICARD_TRY(spec_collect(rs.Q));
            pending = true;
          }
        }
        return PICARD_OK;
      }));
      PICARD_TRY(pool.run(n, [&](int r) -> int {
        RunSolve& rs = solves[r];
        if (!rs.batched && !rs.spectral && !rs.e.trivial) return PICARD_OK;  // solved on its own above
        int32_t sw = 0;
        int q = epot_finish(ctxs[r], rs.e, rs.sweeps, rs.converged, &sw);
        if (q == PICARD_ERR_NOT_CONVERGED) nc = true;
        else if (q != PICARD_OK) return q;
        if (sweeps_total) sweeps_total[r] += sw;
        return PICARD_OK;
      }));
      lap(3);
      // ---- CalcEfield + BCfields, AdvanceVelocity (CELL32, when another step
      // follows: fused with that step's AdvancePosition, as the single-run loop)
      PICARD_TRY(pool.run(n, [&](int r) -> int {
        picard_ctx* c = ctxs[r];
        PICARD_TRY(picard_gpu_calc_efield(c));
        if (step < nsteps && c->layout == PICARD_LAYOUT_CELL32)
          PICARD_CUDA(launch_push_advance_c32(c->K, c->c32, c->num_local, c->E32, c->prm.dt, c->st));
        else
          PICARD_TRY(picard_gpu_advance_velocity(c, c->prm.dt));
        c->stats.steps += 1;
        c->stats.particle_steps += c->num_local;
        return PICARD_OK;
      }));
      lap(4);
    }
    for (int r = 0; r < n; ++r) {
      PICARD_TRY(count_issue(ctxs[r]));  // a wait that gave up in the last step
      PICARD_TRY(count_collect(ctxs[r]));
    }
    return PICARD_OK;
  };
  rc = body();
  if (log)
    std::fprintf(stderr,
                 "picard batch %d runs: particles %.1f ms, compaction+inflow %.1f ms, deposit+bcpot+rhs %.1f ms, "
                 "jacobi %.1f ms (%lld rounds, %lld ticks, %lld launches, %lld CTAs), push %.1f ms\n",
                 n, ph[0], ph[1], ph[2], ph[3], rounds, ticks, launches, g_batch_ctas, ph[4]);
  if (rc == PICARD_OK) rc = check_cuda(cudaStreamSynchronize(bst), "batch stream");
  cleanup();
  if (rc != PICARD_OK) return rc;
  if (nc) return fail(PICARD_ERR_NOT_CONVERGED, "at least one Jacobi solve hit 2*maxit+1 sweeps");
  return PICARD_OK;
}

}  // namespace

extern "C" int picard_batch_run_fused(picard_ctx** ctxs, int32_t n, int32_t iter_start, int32_t iter_end,
                                      int64_t* sweeps_total) {
  if (n < 1 || n > (1 << 20)) return fail(PICARD_ERR_BAD_ARG, "bad run count");
  if (iter_end < iter_start) return fail(PICARD_ERR_BAD_ARG, "iter_end < iter_start");
  std::vector<int32_t> it0((size_t)n, iter_start);
  return batch_run_impl(ctxs, n, it0.data(), iter_end - iter_start, sweeps_total);
}

extern "C" int picard_batch_step(picard_ctx** ctxs, int32_t n, const int32_t* iterations, int64_t* sweeps_total) {
  if (!iterations || n < 1 || n > (1 << 20)) return fail(PICARD_ERR_BAD_ARG, "bad arguments");
  std::vector<int32_t> it0((size_t)n);
  for (int r = 0; r < n; ++r) it0[(size_t)r] = iterations[r] - 1;
  return batch_run_impl(ctxs, n, it0.data(), 1, sweeps_total);
}
