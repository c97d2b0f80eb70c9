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
//   bool keep_wrap(long long p, int wrap)  -- the BCoutflow test of particle
//        p; when wrap != 0 also wraps a survivor across periodic faces;
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
#pragma unroll
  for (int q = 0; q < kOutflowItems; ++q) {
    const long long p = base + (long long)q * kOutflowThreads + threadIdx.x;
    const bool keep = p < n && lay.keep_wrap(p, wrap);
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

// The first survivor above s, or -1: the rest of s's keep word, then the
// following words, skipping whole blocks that have no survivor.
__device__ __forceinline__ long long next_survivor(const uint2* words, const int* block_counts, long long s, int nb) {
  const long long nwords = (long long)nb * kOutflowWords;
  long long wi = s >> 5;
  const int sh = int(s & 31);
  unsigned bits = sh == 31 ? 0u : (words[wi].x & (0xffffffffu << (sh + 1)));
  while (bits == 0u) {
    if (++wi >= nwords) return -1;
    if ((wi & (kOutflowWords - 1)) == 0) {
      long long b = wi / kOutflowWords;
      while (b < nb && block_counts[b] == 0) ++b;
      if (b >= nb) return -1;
      wi = b * kOutflowWords;
    }
    bits = words[wi].x;
  }
  return (wi << 5) + (__ffs(bits) - 1);
}

// Between q and the next survivor g above it, S is constant, so the chain
// steps q, q + S, q + 2S, ... until it first reaches g or beyond: the kernel
// jumps there directly (with survivors dense, that is the single hop
// q + S(q)).  A pathological pattern -- say only the last particle survives --
// then takes one jump instead of a walk over every position.
template <class L>
__global__ void __launch_bounds__(kOutflowThreads)
    outflow_fill_kernel(L lay, long long n, const uint2* words, const int* block_counts, int nb,
                        const int* block_offsets, const int* survivors, int* err) {
  const long long np = *survivors;
  const long long base = (long long)blockIdx.x * kOutflowTile;
  if (base >= np) return;
  for (int q = 0; q < kOutflowItems; ++q) {
    const long long p = base + (long long)q * kOutflowThreads + threadIdx.x;
    if (p >= np) break;
    uint2 w = words[p >> 5];
    if ((w.x >> (p & 31)) & 1u) continue;  // a survivor below n' stays where it is
    long long s = p;
    bool found = false;
    // the chain rises strictly and stays below n, so n jumps always suffice
    for (long long hop = 0; hop < n; ++hop) {
      const long long above = np - kept_through(block_offsets, s, w);
      if (above < 1) break;  // not reachable from a hole below n'
      const long long g = next_survivor(words, block_counts, s, nb);
      if (g < 0) break;
      const long long t = s + (g - s + above - 1) / above * above;
      if (t >= n) break;
      s = t;
      w = words[s >> 5];
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

// n particles of `lay`; *count receives the number of survivors.  words holds
// compact_blocks(n) * 64 entries, block_counts compact_blocks(n), and
// block_offsets 2 compact_blocks(n) + 2 + scan_scratch_ints(...) ints.
template <class L>
cudaError_t launch_outflow_inplace(const L& lay, long long n, uint2* words, int* block_counts, int* block_offsets,
                                   int* count, int wrap, int* err, cudaStream_t st) {
  if (n <= 0) return cudaMemsetAsync(count, 0, sizeof(int), st);
  const int nb = int((n + kOutflowTile - 1) / kOutflowTile);
  note_launch();
  outflow_mark_kernel<<<nb, kOutflowThreads, 0, st>>>(lay, n, words, block_counts, wrap);
  cudaError_t e = launch_scan_int(block_counts, block_offsets, nb, count, block_offsets + nb + 1, st);
  if (e != cudaSuccess) return e;
  note_launch();
  outflow_fill_kernel<<<nb, kOutflowThreads, 0, st>>>(lay, n, words, block_counts, nb, block_offsets, count, err);
  return cudaGetLastError();
}

}  // namespace
}  // namespace picard
