// outflow.cuh -- BCoutflow in place, in the reference's particle order.
//
// BCoutflow.f90:24-83 walks the particles from the last to the first and
// replaces each removed particle by the current last one (then shortens the
// array).  When position q is removed, the current last position is
// q + S(q), with S(q) the number of survivors above q.  If that position was
// itself removed earlier, it holds the particle it received then.  So the
// particle that finally fills a hole p below n' (the number of survivors) is
// found by following q -> q + S(q) from p until q is a survivor.
//
// Every position is read at most once by that process, so the chains of
// different holes are disjoint and together at most n long.  Every source is
// a survivor at or above n' and every destination a hole below it, so all
// holes fill in parallel, in place, and the array ends exactly as the
// reference's loop leaves it.
//
// Pass 1 (mark): one keep word per 32 particles (the keep bits, and the
// survivors of the block before the word), one survivor count per block, and
// the ParticlesTransfer periodic wrap of the survivors in place.  An exclusive
// scan of the block counts gives n' and the block offsets.  Pass 2 (fill):
// every hole below n' follows its chain and copies the particle it reaches.
//
// A layout L provides
//   Key load_key(long long p)  -- what the test reads first (issued for all of
//        a thread's items before any is tested, so the loads overlap);
//   bool keep_wrap(long long p, Key key, int wrap)  -- the BCoutflow test of
//        particle p; when wrap != 0 also wraps a survivor across periodic faces;
//   void move(long long dst, long long src).
#pragma once

#include "common.cuh"
#include "kernels.cuh"

namespace picard {
namespace {

constexpr int kOutflowThreads = 256;
constexpr int kOutflowItems = 8;
constexpr int kOutflowTile = kOutflowThreads * kOutflowItems;  // particles per block
constexpr int kOutflowWords = kOutflowTile / 32;               // keep words per block
static_assert(kOutflowWords == kOutflowWordsPerBlock, "keep words per block");

// Item q of thread t is particle base + 256 q + t, so word 8 q + warp of the
// block holds the ballot of item q of that warp: bit l is particle 32 w + l.
template <class L>
__global__ void __launch_bounds__(kOutflowThreads)
    outflow_mark_kernel(L lay, long long n, uint2* words, int* block_counts, int wrap) {
  __shared__ unsigned bits[kOutflowWords];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const long long base = (long long)blockIdx.x * kOutflowTile;
  typename L::Key key[kOutflowItems];
#pragma unroll
  for (int q = 0; q < kOutflowItems; ++q) {
    const long long p = base + (long long)q * kOutflowThreads + threadIdx.x;
    if (p < n) key[q] = lay.load_key(p);
  }
#pragma unroll
  for (int q = 0; q < kOutflowItems; ++q) {
    const long long p = base + (long long)q * kOutflowThreads + threadIdx.x;
    const bool keep = p < n && lay.keep_wrap(p, key[q], wrap);
    const unsigned m = __ballot_sync(0xffffffffu, keep);
    if (lane == 0) bits[q * (kOutflowThreads / 32) + warp] = m;
  }
  __syncthreads();
  if (warp == 0) {
    const unsigned b0 = bits[2 * lane], b1 = bits[2 * lane + 1];
    const int c0 = __popc(b0), v = c0 + __popc(b1);
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    const int before = x - v;
    uint2* w = words + (long long)blockIdx.x * kOutflowWords;
    w[2 * lane] = make_uint2(b0, unsigned(before));
    w[2 * lane + 1] = make_uint2(b1, unsigned(before + c0));
    if (lane == 31) block_counts[blockIdx.x] = x;
  }
}

// Survivors among particles 0 .. q (q < n); w = the keep word of q.
__device__ __forceinline__ long long kept_through(const int* block_offsets, long long q, uint2 w) {
  const unsigned upto = w.x & (0xffffffffu >> (31 - int(q & 31)));
  return (long long)block_offsets[q / kOutflowTile] + (long long)w.y + __popc(upto);
}

// Between q and the next survivor above it S is constant, so the chain steps
// q, q + S, q + 2S, ... until it first passes that survivor.  The step count k
// is the smallest k >= 1 with a survivor in (q, q + kS], found by galloping
// and bisection on kept_through (O(1) per probe).  With survivors dense the
// first probe succeeds and the jump is the single hop q + S(q); a
// pathological pattern -- say only the last particle survives -- takes a few
// dozen probes instead of a walk over every position.
template <class L>
__global__ void __launch_bounds__(kOutflowThreads)
    outflow_fill_kernel(L lay, long long n, const uint2* words, const int* block_offsets, const int* survivors,
                        int* err) {
  const long long np = *survivors;
  const long long base = (long long)blockIdx.x * kOutflowTile;
  if (base >= np) return;
  // a tile whose particles all survive has no hole
  if (blockIdx.x + 1 < gridDim.x && block_offsets[blockIdx.x + 1] - block_offsets[blockIdx.x] == kOutflowTile) return;
  for (int q = 0; q < kOutflowItems; ++q) {
    const long long p = base + (long long)q * kOutflowThreads + threadIdx.x;
    if (p >= np) break;
    uint2 w = words[p >> 5];
    if ((w.x >> (p & 31)) & 1u) continue;  // a survivor below n' stays where it is
    long long s = p;
    bool found = false;
    // the chain rises strictly and stays below n, so n jumps always suffice
    for (long long hop = 0; hop < n; ++hop) {
      const long long kept = kept_through(block_offsets, s, w);
      const long long above = np - kept;
      if (above < 1) break;                    // not reachable from a hole below n'
      const long long kmax = (n - 1 - s) / above;  // s + k * above stays below n
      if (kmax < 1) break;
      long long k = 1;
      uint2 wt = words[(s + above) >> 5];
      if (kept_through(block_offsets, s + above, wt) == kept) {
        // no survivor within one hop: kept_through(s + lo S) == kept, find hi
        long long lo = 1, hi = 2;
        bool bracketed = false;
        for (int g = 0; g < 64; ++g) {
          const long long h = hi < kmax ? hi : kmax;
          const long long t = s + h * above;
          if (kept_through(block_offsets, t, words[t >> 5]) > kept) {
            hi = h;
            bracketed = true;
            break;
          }
          if (h >= kmax) break;
          lo = h;
          hi = 2 * hi;
        }
        if (!bracketed) break;
        while (hi - lo > 1) {
          const long long mid = lo + (hi - lo) / 2;
          const long long t = s + mid * above;
          if (kept_through(block_offsets, t, words[t >> 5]) > kept)
            hi = mid;
          else
            lo = mid;
        }
        k = hi;
        wt = words[(s + k * above) >> 5];
      }
      s += k * above;
      w = wt;
      if ((w.x >> (s & 31)) & 1u) {
        found = true;
        break;
      }
    }
    if (found)
      lay.move(p, s);
    else
      atomicCAS(err, 0, int(kDevRange));
  }
}

// ------------------------------------------------ the fill by pointer jumping
//
// When the window [n', n) is wide and its survivors sparse -- BCoutflow right
// after BCinflow has appended every inflow candidate, most of which are
// removed -- a chain steps through the window ~(n - n') / m times (m
// survivors in the window), each step a dependent pair of loads, and the
// longest chain sets the time.  The same chains are then resolved in
// ceil(log2(n - n')) parallel rounds instead: every window position x holds
// the next position of its chain, x + S(x) (itself for a survivor), and each
// round replaces it by the next position's entry, so after the rounds every
// position holds the survivor its chain ends at.  The holes below n' then
// take the survivor at the end of the chain from q + S(q), exactly as in
// outflow_fill_kernel.

// m (the survivors in the window, = the holes below n') into info[0].
__global__ void outflow_window_kernel(const uint2* words, const int* block_offsets, const int* survivors, int* info) {
  const long long np = *survivors;
  info[0] = np > 0 ? int(np - kept_through(block_offsets, np - 1, words[(np - 1) >> 5])) : 0;
}

__global__ void outflow_jump_init_kernel(long long n, const uint2* words, const int* block_offsets,
                                         const int* survivors, int* nxt) {
  const long long np = *survivors;
  for (long long x = np + (long long)blockIdx.x * blockDim.x + threadIdx.x; x < n;
       x += (long long)gridDim.x * blockDim.x) {
    const uint2 w = words[x >> 5];
    if ((w.x >> (x & 31)) & 1u)
      nxt[x - np] = int(x);
    else
      nxt[x - np] = int(x + (np - kept_through(block_offsets, x, w)));  // in [x, n)
  }
}

__global__ void outflow_jump_kernel(const int* __restrict__ in, int* __restrict__ out, long long n,
                                    const int* survivors) {
  const long long np = *survivors;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n - np;
       i += (long long)gridDim.x * blockDim.x)
    out[i] = in[in[i] - np];
}

template <class L>
__global__ void __launch_bounds__(kOutflowThreads)
    outflow_fill_jump_kernel(L lay, long long n, const uint2* words, const int* block_offsets, const int* survivors,
                             const int* term, int* err) {
  const long long np = *survivors;
  const long long base = (long long)blockIdx.x * kOutflowTile;
  if (base >= np) return;
  for (int q = 0; q < kOutflowItems; ++q) {
    const long long p = base + (long long)q * kOutflowThreads + threadIdx.x;
    if (p >= np) break;
    const uint2 w = words[p >> 5];
    if ((w.x >> (p & 31)) & 1u) continue;
    const long long s = p + (np - kept_through(block_offsets, p, w));
    const long long t = (s >= np && s < n) ? (long long)term[s - np] : -1;
    if (t >= np && t < n && ((words[t >> 5].x >> (t & 31)) & 1u))
      lay.move(p, t);
    else
      atomicCAS(err, 0, int(kDevRange));
  }
}

// n particles of `lay`; *count receives the number of survivors.  words holds
// compact_blocks(n) * 64 entries, block_counts compact_blocks(n), and
// block_offsets 2 compact_blocks(n) + 2 + scan_scratch_ints(...) ints.
// split: the stages of OutflowSplit (kernels.cuh), or null for all at once.
template <class L>
cudaError_t launch_outflow_inplace(const L& lay, long long n, uint2* words, int* block_counts, int* block_offsets,
                                   int* count, int wrap, int* err, cudaStream_t st,
                                   const OutflowSplit* split = nullptr) {
  if (n <= 0) {
    if (split && split->stage == 2) return cudaSuccess;
    cudaError_t e = cudaMemsetAsync(count, 0, sizeof(int), st);
    if (e == cudaSuccess && split) e = cudaMemsetAsync(split->info, 0, sizeof(int), st);
    return e;
  }
  const int nb = int((n + kOutflowTile - 1) / kOutflowTile);
  if (!split || split->stage == 1) {
    note_launch();
    outflow_mark_kernel<<<nb, kOutflowThreads, 0, st>>>(lay, n, words, block_counts, wrap);
    cudaError_t e = launch_scan_int(block_counts, block_offsets, nb, count, block_offsets + nb + 1, st);
    if (e != cudaSuccess) return e;
    if (split) {
      note_launch();
      outflow_window_kernel<<<1, 1, 0, st>>>(words, block_offsets, count, split->info);
      return cudaGetLastError();
    }
  }
  if (split && split->nxt[0] && n > split->np) {
    const long long W = n - split->np;
    const long long want = (W + 255) / 256;
    const int g = int(want < 148LL * 16 ? want : 148LL * 16);
    note_launch();
    outflow_jump_init_kernel<<<g, 256, 0, st>>>(n, words, block_offsets, count, split->nxt[0]);
    int* a = split->nxt[0];
    int* b = split->nxt[1];
    for (long long hops = 1; hops < W; hops <<= 1) {
      note_launch();
      outflow_jump_kernel<<<g, 256, 0, st>>>(a, b, n, count);
      int* t = a;
      a = b;
      b = t;
    }
    note_launch();
    outflow_fill_jump_kernel<<<nb, kOutflowThreads, 0, st>>>(lay, n, words, block_offsets, count, a, err);
    return cudaGetLastError();
  }
  note_launch();
  outflow_fill_kernel<<<nb, kOutflowThreads, 0, st>>>(lay, n, words, block_offsets, count, err);
  return cudaGetLastError();
}

}  // namespace
}  // namespace picard
