// sort.cu -- stable counting sort of the particles by cell.
//
// On one rank ParticlesTransfer (ParticlesTransfer.f90:488-519) only wraps
// coordinates across periodic faces; its slot in the loop is where the
// particles are put back in cell order.  The cell of a particle is the node
// whose cell [x_c - dx/2, x_c + dx/2) holds it, (i_c, j_c, k_c) with
// i_c = floor((x - Lx_min)/dx + 1) (0-based node index, clamped to
// [-1, N+2]), and its key is
//   ((k_c + 1) (Ny + 4) + j_c + 1) (Nx + 4) + i_c + 1,
// x fastest: the order in which ParticlesInitialize (ParticlesInitialize.f90:
// 54-119) creates them.  The tiled deposit and the E-field gather rely on it:
// a chunk of consecutive particles then covers a small box of nodes.  The
// loop breaks it slowly -- particles cross cells, BCoutflow fills holes with
// particles from the end of the array, new particles are appended -- and a
// sort every few hundred steps restores it.
//
// The sort is stable: particles of one cell keep their order, so the result
// is a function of the particle arrays alone and every later step is
// deterministic.  It is a permutation: every particle keeps every bit, N is a
// sum of fixed-point integers (order-independent) and every other phase
// treats particles one by one, so a sorted run holds the same particle set
// and the same fields as an unsorted one, bit for bit.
//
// Particles move ~10^-3 cells per step, so the array stays a concatenation of
// long runs of one key.  The sort works on those runs:
//   1. heads: a particle whose key differs from its predecessor's starts a
//      run; per 2,048-particle tile, the number of heads (one pass over the
//      keys);
//   2. an exclusive scan gives each tile's first run; each head writes its
//      run's key and start (a second pass).  If no run's key is below the
//      previous run's, the array is already sorted and nothing moves;
//   3. the R runs are sorted by key with a stable LSD radix sort (8 bits per
//      pass; R is a few per cell on a developed plasma);
//   4. an exclusive scan of the run lengths in sorted order gives every run's
//      destination, and one pass copies each particle to the other particle
//      buffer at its run's destination plus its place in the run.
// Traffic on a developed plasma: two key passes (16 B per CELL32 particle
// each, the offsets decide the cell), the radix sort of the runs, and one
// copy (29 B read, 29 B written).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <string>

#include "common.cuh"
#include "context.cuh"
#include "kernels.cuh"

namespace picard {
namespace {

constexpr int kSortThreads = 256;
constexpr int kSortItems = 8;
constexpr int kSortTile = kSortThreads * kSortItems;  // particles (or runs) per block
constexpr int kSortWords = kSortTile / 32;            // ballot words per tile

struct SortKeyGeom {
  int nx, ny, nz;
  int nx4, ny4;
};

__device__ __forceinline__ uint32_t cell_sort_key(const SortKeyGeom& G, int i, int j, int k) {
  i = min(max(i, -1), G.nx + 2);
  j = min(max(j, -1), G.ny + 2);
  k = min(max(k, -1), G.nz + 2);
  return (uint32_t(k + 1) * uint32_t(G.ny4) + uint32_t(j + 1)) * uint32_t(G.nx4) + uint32_t(i + 1);
}

// CELL32: the CIC base node plus one where the in-cell offset is >= 1/2.
struct SortC32 {
  PartC32 a;
  SortKeyGeom G;
  __device__ uint32_t key(long long p) const {
    int i, j, k;
    unpack_cell(__ldg(a.cell + p), i, j, k);
    return cell_sort_key(G, i + int(__ldg(a.fx + p) >> 31), j + int(__ldg(a.fy + p) >> 31),
                         k + int(__ldg(a.fz + p) >> 31));
  }
  __device__ void copy(const SortC32& d, long long to, long long from) const {
    d.a.cell[to] = a.cell[from];
    d.a.fx[to] = a.fx[from];
    d.a.fy[to] = a.fy[from];
    d.a.fz[to] = a.fz[from];
    d.a.vx[to] = a.vx[from];
    d.a.vy[to] = a.vy[from];
    d.a.vz[to] = a.vz[from];
    d.a.sp[to] = a.sp[from];
  }
};

// F64: floor((x - Lx_min)/dx + 1) per axis.
struct SortF64 {
  PartF64 a;
  SortKeyGeom G;
  double Lx_min, Ly_min, Lz_min, dx, dy, dz;
  __device__ uint32_t key(long long p) const {
    const int i = __double2int_rd((__ldg(a.x + p) - Lx_min) / dx + 1.0);
    const int j = __double2int_rd((__ldg(a.y + p) - Ly_min) / dy + 1.0);
    const int k = __double2int_rd((__ldg(a.z + p) - Lz_min) / dz + 1.0);
    return cell_sort_key(G, i, j, k);
  }
  __device__ void copy(const SortF64& d, long long to, long long from) const {
    d.a.x[to] = a.x[from];
    d.a.y[to] = a.y[from];
    d.a.z[to] = a.z[from];
    d.a.vx[to] = a.vx[from];
    d.a.vy[to] = a.vy[from];
    d.a.vz[to] = a.vz[from];
    d.a.sp[to] = a.sp[from];
  }
};

// Keys of one tile into skey, its head ballots into words (word q * 8 + warp
// holds item q of that warp: bit l is particle base + 256 q + 32 warp + l,
// so words run in particle order), their exclusive prefix into wpre, and the
// tile's head count.
template <class L>
__device__ int tile_heads(const L& lay, long long n, long long base, uint32_t* skey, unsigned* words, int* wpre) {
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
#pragma unroll
  for (int q = 0; q < kSortItems; ++q) {
    const long long p = base + (long long)q * kSortThreads + t;
    skey[q * kSortThreads + t] = p < n ? lay.key(p) : 0u;
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < kSortItems; ++q) {
    const int idx = q * kSortThreads + t;
    const long long p = base + idx;
    bool head = false;
    if (p < n) {
      if (p == 0)
        head = true;
      else
        head = (idx == 0 ? lay.key(p - 1) : skey[idx - 1]) != skey[idx];
    }
    const unsigned m = __ballot_sync(0xffffffffu, head);
    if (lane == 0) words[q * (kSortThreads / 32) + warp] = m;
  }
  __syncthreads();
  __shared__ int total;
  if (warp == 0) {
    const int c0 = __popc(words[2 * lane]), v = c0 + __popc(words[2 * lane + 1]);
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    wpre[2 * lane] = x - v;
    wpre[2 * lane + 1] = x - v + c0;
    if (lane == 31) total = x;
  }
  __syncthreads();
  return total;
}

// Heads up to and including item idx of the tile.
__device__ __forceinline__ int heads_through(const unsigned* words, const int* wpre, int idx) {
  const int w = (idx >> 8) * (kSortThreads / 32) + ((idx & 255) >> 5);
  const int l = idx & 31;
  return wpre[w] + __popc(words[w] & (0xffffffffu >> (31 - l)));
}

template <class L>
__global__ void __launch_bounds__(kSortThreads) sort_heads_kernel(L lay, long long n, int* tile_counts) {
  __shared__ uint32_t skey[kSortTile];
  __shared__ unsigned words[kSortWords];
  __shared__ int wpre[kSortWords];
  const int c = tile_heads(lay, n, (long long)blockIdx.x * kSortTile, skey, words, wpre);
  if (threadIdx.x == 0) tile_counts[blockIdx.x] = c;
}

// Each head writes its run's key and first particle; the last block also
// closes the list with run_start[R] = n.  *descents counts heads whose key is
// below the previous particle's (zero: the array is already sorted).
template <class L>
__global__ void __launch_bounds__(kSortThreads)
    sort_runs_kernel(L lay, long long n, const int* tile_offsets, const int* runs, uint32_t* run_key, int* run_start,
                     int* descents) {
  __shared__ uint32_t skey[kSortTile];
  __shared__ unsigned words[kSortWords];
  __shared__ int wpre[kSortWords];
  const long long base = (long long)blockIdx.x * kSortTile;
  tile_heads(lay, n, base, skey, words, wpre);
  const int first = tile_offsets[blockIdx.x];
  int desc = 0;
#pragma unroll
  for (int q = 0; q < kSortItems; ++q) {
    const int idx = q * kSortThreads + threadIdx.x;
    const long long p = base + idx;
    if (p >= n || !((words[(idx >> 8) * (kSortThreads / 32) + ((idx & 255) >> 5)] >> (idx & 31)) & 1u)) continue;
    const int r = first + heads_through(words, wpre, idx) - 1;
    run_key[r] = skey[idx];
    run_start[r] = int(p);
    if (p > 0 && (idx == 0 ? lay.key(p - 1) : skey[idx - 1]) > skey[idx]) ++desc;
  }
  desc = __reduce_add_sync(0xffffffffu, desc);
  if ((threadIdx.x & 31) == 0 && desc) atomicAdd(descents, desc);
  if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) run_start[*runs] = int(n);
}

// ------------------------------------------------- LSD radix sort of the runs
//
// Per pass: a digit histogram per 2,048-key tile (hist[d * tiles + tile]),
// an exclusive scan of it (the stable global offsets), and a scatter in which
// warp w ranks its 256 keys (8 rounds of 32, in order) with match_any against
// per-warp digit counters, so equal digits keep their order within the warp,
// across warps (prefix over warps) and across tiles (the scan).

__global__ void __launch_bounds__(kSortThreads)
    radix_hist_kernel(const uint32_t* keys, int count, int shift, int tiles, int* hist) {
  __shared__ int h[256];
  h[threadIdx.x] = 0;
  __syncthreads();
  const long long base = (long long)blockIdx.x * kSortTile;
  // keys of nearby runs share their upper digits: one shared atomic per
  // distinct digit of a warp instead of one per key
#pragma unroll
  for (int q = 0; q < kSortItems; ++q) {
    const long long i = base + (long long)q * kSortThreads + threadIdx.x;
    const unsigned d = i < count ? ((keys[i] >> shift) & 255u) : 256u;
    const unsigned peers = __match_any_sync(0xffffffffu, d);
    if (d < 256u && (threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(&h[d], __popc(peers));
  }
  __syncthreads();
  hist[(long long)threadIdx.x * tiles + blockIdx.x] = h[threadIdx.x];
}

// vin == nullptr: the values are the key indices (the first pass).
__global__ void __launch_bounds__(kSortThreads)
    radix_scatter_kernel(const uint32_t* kin, const int* vin, uint32_t* kout, int* vout, int count, int shift,
                         int tiles, const int* offsets, int* err) {
  __shared__ int cnt[kSortThreads / 32][256];
  __shared__ int gbase[256];
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
#pragma unroll
  for (int w = 0; w < kSortThreads / 32; ++w) cnt[w][t] = 0;
  __syncthreads();
  const long long base = (long long)blockIdx.x * kSortTile + (long long)warp * (32 * kSortItems);
  uint32_t k[kSortItems];
  int v[kSortItems], rank[kSortItems];
  const unsigned lt = (1u << lane) - 1u;
#pragma unroll
  for (int q = 0; q < kSortItems; ++q) {
    const long long i = base + q * 32 + lane;
    const bool ok = i < count;
    k[q] = ok ? kin[i] : 0u;
    v[q] = ok ? (vin ? vin[i] : int(i)) : 0;
    const unsigned d = ok ? ((k[q] >> shift) & 255u) : 256u;
    const unsigned peers = __match_any_sync(0xffffffffu, d);
    int before = 0;
    if (ok) before = cnt[warp][d];
    __syncwarp();
    if (ok) {
      rank[q] = before + __popc(peers & lt);
      if ((peers & lt) == 0u) cnt[warp][d] = before + __popc(peers);
    }
    __syncwarp();
  }
  __syncthreads();
  {
    int s = 0;
#pragma unroll
    for (int w = 0; w < kSortThreads / 32; ++w) {
      const int c = cnt[w][t];
      cnt[w][t] = s;
      s += c;
    }
    gbase[t] = offsets[(long long)t * tiles + blockIdx.x];
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < kSortItems; ++q) {
    const long long i = base + q * 32 + lane;
    if (i >= count) continue;
    const unsigned d = (k[q] >> shift) & 255u;
    const int pos = gbase[d] + cnt[warp][d] + rank[q];
    if (pos < 0 || pos >= count) {  // never taken: the ranks are a permutation
      atomicCAS(err, 0, int(kDevRange));
      continue;
    }
    kout[pos] = k[q];
    vout[pos] = v[q];
  }
}

// len[q] = length of run ids[q] (sorted order).
__global__ void run_len_kernel(const int* ids, const int* run_start, int count, int* len, int* err) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= count) return;
  const int r = ids[q];
  if (r < 0 || r >= count) {
    atomicCAS(err, 0, int(kDevRange));
    len[q] = 0;
  } else {
    len[q] = run_start[r + 1] - run_start[r];
  }
}

__global__ void run_dst_kernel(const int* ids, const int* off, int count, int* run_dst, int* err) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= count) return;
  const int r = ids[q];
  if (r < 0 || r >= count)
    atomicCAS(err, 0, int(kDevRange));
  else
    run_dst[r] = off[q];
}

// Every particle to its run's destination plus its place in the run.
template <class L>
__global__ void __launch_bounds__(kSortThreads)
    sort_move_kernel(L src, L dst, long long n, const int* tile_offsets, const int* run_start, const int* run_dst,
                     int* err) {
  __shared__ uint32_t skey[kSortTile];
  __shared__ unsigned words[kSortWords];
  __shared__ int wpre[kSortWords];
  const long long base = (long long)blockIdx.x * kSortTile;
  tile_heads(src, n, base, skey, words, wpre);
  const int first = tile_offsets[blockIdx.x];
#pragma unroll
  for (int q = 0; q < kSortItems; ++q) {
    const int idx = q * kSortThreads + threadIdx.x;
    const long long p = base + idx;
    if (p >= n) continue;
    const int r = first + heads_through(words, wpre, idx) - 1;
    const long long to = (long long)run_dst[r] + (p - run_start[r]);
    if (to < 0 || to >= n) {  // never taken: the destinations are a permutation
      atomicCAS(err, 0, int(kDevRange));
      continue;
    }
    src.copy(dst, to, p);
  }
}

int blocks_of(long long n) { return int((n + kSortTile - 1) / kSortTile); }

// Scratch of a sort of up to cap particles (allocated on first use, sized for
// the worst case of one run per particle).
int ensure_sort_buffers(picard_ctx* c) {
  SortBuf& b = c->sortbuf;
  if (b.cap == c->capacity && b.run_start) return PICARD_OK;
  const long long cap = c->capacity;
  const int tiles = blocks_of(cap);
  const long long hist = 256LL * tiles;
  if (hist > 0x7fffffffLL) return fail(PICARD_ERR_BAD_ARG, "particle capacity too large for the sort");
  const long long scan_n = std::max<long long>(hist, cap);
  auto ia = [&](int*& p, long long n) { return dev_alloc(c, (void**)&p, sizeof(int) * (size_t)n); };
  auto ua = [&](uint32_t*& p, long long n) { return dev_alloc(c, (void**)&p, sizeof(uint32_t) * (size_t)n); };
  int rc;
  if ((rc = ua(b.key[0], cap)) || (rc = ua(b.key[1], cap)) || (rc = ia(b.val[0], cap)) || (rc = ia(b.val[1], cap)) ||
      (rc = ia(b.run_start, cap + 1)) || (rc = ia(b.tile_counts, tiles)) || (rc = ia(b.tile_offsets, tiles + 1)) ||
      (rc = ia(b.hist, hist)) || (rc = ia(b.hist_off, hist)) || (rc = ia(b.info, 8)) ||
      (rc = ia(b.scan_scratch, scan_scratch_ints(int(scan_n)) + 4)))
    return rc;
  if (c->layout == PICARD_LAYOUT_F64) {
    PartF64& a = c->f64b;
    auto da = [&](double*& p) { return dev_alloc(c, (void**)&p, sizeof(double) * (size_t)cap); };
    if ((rc = da(a.x)) || (rc = da(a.y)) || (rc = da(a.z)) || (rc = da(a.vx)) || (rc = da(a.vy)) || (rc = da(a.vz)) ||
        (rc = dev_alloc(c, (void**)&a.sp, (size_t)cap)))
      return rc;
  } else {
    PartC32& a = c->c32b;
    auto fa = [&](float*& p) { return dev_alloc(c, (void**)&p, sizeof(float) * (size_t)cap); };
    if ((rc = ua(a.cell, cap)) || (rc = ua(a.fx, cap)) || (rc = ua(a.fy, cap)) || (rc = ua(a.fz, cap)) ||
        (rc = fa(a.vx)) || (rc = fa(a.vy)) || (rc = fa(a.vz)) || (rc = dev_alloc(c, (void**)&a.sp, (size_t)cap)))
      return rc;
  }
  b.cap = cap;
  return PICARD_OK;
}

template <class L>
int sort_with(picard_ctx* c, const L& src, const L& dst, bool* moved) {
  SortBuf& b = c->sortbuf;
  const long long n = c->num_local;
  const int tiles = blocks_of(n);
  cudaStream_t st = c->st;
  int* runs = b.info;         // R
  int* descents = b.info + 1;
  PICARD_CUDA(cudaMemsetAsync(b.info, 0, 8 * sizeof(int), st));
  note_launch();
  sort_heads_kernel<<<tiles, kSortThreads, 0, st>>>(src, n, b.tile_counts);
  PICARD_CUDA(cudaGetLastError());
  PICARD_CUDA(launch_scan_int(b.tile_counts, b.tile_offsets, tiles, runs, b.scan_scratch, st));
  note_launch();
  sort_runs_kernel<<<tiles, kSortThreads, 0, st>>>(src, n, b.tile_offsets, runs, b.key[0], b.run_start, descents);
  PICARD_CUDA(cudaGetLastError());
  PICARD_CUDA(cudaMemcpyAsync(c->h_pinned_i + 4, b.info, 2 * sizeof(int), cudaMemcpyDeviceToHost, st));
  PICARD_CUDA(cudaStreamSynchronize(st));
  c->stats.d2h_bytes += 2 * sizeof(int);
  const int R = c->h_pinned_i[4];
  *moved = c->h_pinned_i[5] != 0;
  if (std::getenv("PICARD_SORT_LOG"))
    std::fprintf(stderr, "picard sort: %lld particles, %d runs, %d descents\n", n, R, c->h_pinned_i[5]);
  if (!*moved) return PICARD_OK;  // keys already non-decreasing: the stable sort is the identity

  // 3. radix sort of the R run keys (values: run ids)
  const uint32_t kmax = uint32_t((long long)c->sort_geom_keys - 1);
  int bits = 0;
  while (bits < 32 && (kmax >> bits) != 0u) ++bits;
  const int passes = std::max(1, (bits + 7) / 8);
  const int rt = blocks_of(R);
  int cur = 0;
  for (int ps = 0; ps < passes; ++ps) {
    note_launch();
    radix_hist_kernel<<<rt, kSortThreads, 0, st>>>(b.key[cur], R, 8 * ps, rt, b.hist);
    PICARD_CUDA(cudaGetLastError());
    PICARD_CUDA(launch_scan_int(b.hist, b.hist_off, 256 * rt, b.info + 2, b.scan_scratch, st));
    note_launch();
    radix_scatter_kernel<<<rt, kSortThreads, 0, st>>>(b.key[cur], ps == 0 ? nullptr : b.val[cur], b.key[cur ^ 1],
                                                      b.val[cur ^ 1], R, 8 * ps, rt, b.hist_off, c->d_err);
    PICARD_CUDA(cudaGetLastError());
    cur ^= 1;
  }
  const int* ids = b.val[cur];
  // 4. destinations of the runs, then the particles
  int* len = reinterpret_cast<int*>(b.key[cur ^ 1]);
  int* off = b.val[cur ^ 1];
  int* run_dst = reinterpret_cast<int*>(b.key[cur]);
  const int lb = (R + 255) / 256;
  note_launch();
  run_len_kernel<<<lb, 256, 0, st>>>(ids, b.run_start, R, len, c->d_err);
  PICARD_CUDA(cudaGetLastError());
  PICARD_CUDA(launch_scan_int(len, off, R, b.info + 3, b.scan_scratch, st));
  note_launch();
  run_dst_kernel<<<lb, 256, 0, st>>>(ids, off, R, run_dst, c->d_err);
  PICARD_CUDA(cudaGetLastError());
  note_launch();
  sort_move_kernel<<<tiles, kSortThreads, 0, st>>>(src, dst, n, b.tile_offsets, b.run_start, run_dst, c->d_err);
  PICARD_CUDA(cudaGetLastError());
  return check_dev_err_public(c);
}

}  // namespace

int sort_particles(picard_ctx* c) {
  if (c->num_local < 2) return PICARD_OK;
  const picard_params& p = c->prm;
  const long long keys = (long long)(p.nx + 4) * (p.ny + 4) * (p.nz + 4);
  if (keys > 0xffffffffLL) return fail(PICARD_ERR_BAD_ARG, "grid too large for 32-bit cell keys");
  c->sort_geom_keys = keys;
  PICARD_TRY(ensure_sort_buffers(c));
  const SortKeyGeom G{p.nx, p.ny, p.nz, p.nx + 4, p.ny + 4};
  bool moved = false;
  if (c->layout == PICARD_LAYOUT_F64) {
    const KParams& K = c->K;
    const SortF64 src{c->f64, G, K.Lx_min, K.Ly_min, K.Lz_min, K.dx, K.dy, K.dz};
    const SortF64 dst{c->f64b, G, K.Lx_min, K.Ly_min, K.Lz_min, K.dx, K.dy, K.dz};
    PICARD_TRY(sort_with(c, src, dst, &moved));
    if (moved) std::swap(c->f64, c->f64b);
  } else {
    PICARD_TRY(sort_with(c, SortC32{c->c32, G}, SortC32{c->c32b, G}, &moved));
    if (moved) std::swap(c->c32, c->c32b);
  }
  c->stats_sorts += 1;
  if (moved) c->stats_sorts_moved += 1;
  return PICARD_OK;
}

}  // namespace picard

extern "C" int picard_gpu_sort_particles(picard_ctx* c) {
  if (!c) return picard::fail(PICARD_ERR_BAD_ARG, "ctx is NULL");
  return picard::sort_particles(c);
}
