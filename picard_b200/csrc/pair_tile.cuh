// pair_tile.cuh -- one 64 x 8 x ZC tile of an FP32 Jacobi sweep of the
// increment with x pairs, shared by the single-run x-pair kernel and the
// batched multi-run kernel so that both compute every node and every partial
// identically.
//
// Each thread updates the two x-adjacent nodes 2 tx and 2 tx + 1 of its row
// with packed FP32 pair arithmetic (add/sub/mul/fma .rn.f32x2: each lane is
// rounded like the scalar __fadd_rn/__fsub_rn/__fmul_rn/__fmaf_rn of
// jacobi_res_f32, subnormals included) and 8-byte shared-memory loads and
// global stores.  The tile's w box (72 x 10 x (ZC+2), origin the aligned
// column 64 bx) and r box (64 x 8 x ZC, origin the tile's first interior
// column) are in shared memory.  Each 64-wide tile is two of the 32 x 8 x ZC
// tiles the residual partials are defined on (lanes 0-15 and 16-31): their
// per-column FP32 sums over z are formed node by node, and the 32-lane shuffle
// tree of block_sum_store is reproduced exactly -- its steps 16, 8, 4, 2 are
// shuffles by 8, 4, 2, 1 of both pair components, its step 1 the in-lane sum
// of the pair.
#pragma once

#include "stencil.cuh"

namespace picard {

__device__ __forceinline__ unsigned long long pk2(float lo, float hi) {
  unsigned long long r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
  return r;
}
__device__ __forceinline__ float2 up2(unsigned long long v) {
  float2 r;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(r.x), "=f"(r.y) : "l"(v));
  return r;
}
__device__ __forceinline__ unsigned long long add2(unsigned long long a, unsigned long long b) {
  unsigned long long d;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ unsigned long long sub2(unsigned long long a, unsigned long long b) {
  unsigned long long d;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ unsigned long long mul2(unsigned long long a, unsigned long long b) {
  unsigned long long d;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ unsigned long long fma2(unsigned long long a, unsigned long long b, unsigned long long c) {
  unsigned long long d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
  return d;
}

constexpr int kPairBoxX = 72, kPairTile = 64, kPairTy = 8;

// rows: [2][8] shared doubles (row sums of the two 32-wide tiles).  Ends with
// the CTA's threads past a barrier; the caller separates tiles by another.
// FULL: the tile lies wholly inside the interior (pair_tile_full), so no lane
// is masked and every plane is swept -- the same arithmetic without the
// bounds selects.
// W_ZERO: the iterate entering the sweep is zero (the first sweep after an
// anchor), so the w box is not read.  A compile-time flag: with a run-time one
// every plane's loads sat behind a branch and the sweep ran ~15 % slower.
// R_GLOBAL: r is read from global memory (rg, the padded array; 8-byte pair
// loads) instead of the shared-memory r box sr, so a tile needs only the w box
// in shared memory.
template <int ZC, bool FULL, bool W_ZERO, bool R_GLOBAL = false>
__device__ __forceinline__ void pair_tile_sweep_body(const float* sw, const float* sr, const Stencil& S,
                                                     const JacobiCoefF& J, float* wout, double* partial,
                                                     int bx2, int by, int bz, int gx, int gy,
                                                     double (*rows)[kPairTy], const float* rg = nullptr) {
  const int tx = threadIdx.x, ty = threadIdx.y, tid = tx + 32 * ty;
  const long long plane = (long long)S.fpitch * S.nyp;
  const unsigned long long m2 = pk2(-2.0f, -2.0f), ix2 = pk2(J.idx2, J.idx2), iy2 = pk2(J.idy2, J.idy2),
                           iz2 = pk2(J.idz2, J.idz2), naf = pk2(-J.af, -J.af);
  const int i0 = bx2 * kPairTile + 2 * tx + 1, j = by * kPairTy + ty + 1, z0 = bz * ZC;
  const bool act0 = FULL || (i0 <= S.nx && j <= S.ny), act1 = FULL || (i0 + 1 <= S.nx && j <= S.ny);
  const int kend = FULL ? ZC : min(ZC, S.nz - z0);
  // w rows of this thread's pair: plane kk (0 .. ZC+1), row 0 .. 9, columns 2 tx + 4, + 5
  auto wrow = [&](int kk, int row) {
    return *reinterpret_cast<const unsigned long long*>(sw + (kk * (kPairTy + 2) + row) * kPairBoxX + 2 * tx + 4);
  };
  auto wcol = [&](int kk, int row, int col) { return sw[(kk * (kPairTy + 2) + row) * kPairBoxX + col]; };
  unsigned long long wm = W_ZERO ? 0ull : wrow(0, ty + 1);
  unsigned long long wc = W_ZERO ? 0ull : wrow(1, ty + 1);
  unsigned long long r2 = 0ull;  // (+0.0f, +0.0f)
  float* out = wout + fidx(S, i0, j, z0 + 1);
  const float* rin = R_GLOBAL ? rg + fidx(S, i0, j, z0 + 1) : nullptr;
#pragma unroll
  for (int kk = 1; kk <= ZC; ++kk) {
    if (FULL || kk <= kend) {
      unsigned long long wp = 0ull, ym = 0ull, yp = 0ull;
      float xl = 0.0f, xr = 0.0f;
      const float2 c = up2(wc);
      if (!W_ZERO) {
        wp = wrow(kk + 1, ty + 1);
        ym = wrow(kk, ty);
        yp = wrow(kk, ty + 2);
        xl = wcol(kk, ty + 1, 2 * tx + 3);  // x - 1 of the pair's first node
        xr = wcol(kk, ty + 1, 2 * tx + 6);  // x + 1 of the pair's second node
      }
      const unsigned long long xm = pk2(xl, c.x), xp = pk2(c.y, xr);
      unsigned long long rr;
      if (R_GLOBAL) {
        // the pair (i0, i0 + 1) starts at an even float (fidx adds 3 to an odd
        // i0, rows are 8-float aligned); lanes past the interior load nothing
        if (FULL || act1)
          rr = __ldg(reinterpret_cast<const unsigned long long*>(rin));
        else
          rr = pk2(act0 ? __ldg(rin) : 0.0f, 0.0f);
        rin += plane;
      } else {
        rr = *reinterpret_cast<const unsigned long long*>(sr + ((kk - 1) * kPairTy + ty) * kPairTile + 2 * tx);
      }
      // jacobi_res_f32 on both lanes
      const unsigned long long sx = add2(xp, xm), sy = add2(yp, ym), sz = add2(wp, wm);
      unsigned long long lap = mul2(fma2(m2, wc, sx), ix2);
      lap = fma2(fma2(m2, wc, sy), iy2, lap);
      lap = fma2(fma2(m2, wc, sz), iz2, lap);
      const unsigned long long res = sub2(rr, lap);
      const float2 rf = up2(res);
      const unsigned long long resm = FULL ? res : pk2(act0 ? rf.x : 0.0f, act1 ? rf.y : 0.0f);
      r2 = fma2(resm, resm, r2);
      const float2 wn = up2(fma2(naf, res, wc));
      if (FULL || act1) {
        *reinterpret_cast<float2*>(out) = wn;
      } else if (act0) {
        out[0] = wn.x;
      }
      out += plane;
      wm = wc;
      wc = wp;
    }
  }
  // partials of the two 32-wide tiles, block_sum_store's tree reproduced
  const float2 rr2 = up2(r2);
  double v0 = (double)rr2.x, v1 = (double)rr2.y;
#pragma unroll
  for (int o = 8; o > 0; o >>= 1) {
    v0 += __shfl_down_sync(0xffffffffu, v0, o);
    v1 += __shfl_down_sync(0xffffffffu, v1, o);
  }
  if ((tx & 15) == 0) rows[tx >> 4][ty] = v0 + v1;
  __syncthreads();
  if (tid < 2) {
    const int bx = 2 * bx2 + tid;
    if (bx < gx) {
      double sum = 0.0;
      for (int q = 0; q < kPairTy; ++q) sum += rows[tid][q];
      partial[bx + (long long)gx * (by + (long long)gy * bz)] = sum;
    }
  }
}

// The tile (bx2, by, bz) lies wholly inside the nx x ny x nz interior.
__device__ __forceinline__ bool pair_tile_full(const Stencil& S, int bx2, int by, int z0, int zc) {
  return (bx2 + 1) * kPairTile <= S.nx && (by + 1) * kPairTy <= S.ny && z0 + zc <= S.nz;
}

template <int ZC, bool W_ZERO, bool R_GLOBAL = false>
__device__ __forceinline__ void pair_tile_sweep_wz(const float* sw, const float* sr, const Stencil& S,
                                                   const JacobiCoefF& J, float* wout, double* partial, int bx2,
                                                   int by, int bz, int gx, int gy, double (*rows)[kPairTy],
                                                   const float* rg = nullptr) {
  if (pair_tile_full(S, bx2, by, bz * ZC, ZC))
    pair_tile_sweep_body<ZC, true, W_ZERO, R_GLOBAL>(sw, sr, S, J, wout, partial, bx2, by, bz, gx, gy, rows, rg);
  else
    pair_tile_sweep_body<ZC, false, W_ZERO, R_GLOBAL>(sw, sr, S, J, wout, partial, bx2, by, bz, gx, gy, rows, rg);
}

// The same with the zero-iterate flag known only at run time (per run in the
// batched kernel): one branch per tile.
template <int ZC>
__device__ __forceinline__ void pair_tile_sweep(const float* sw, const float* sr, const Stencil& S,
                                                const JacobiCoefF& J, float* wout, double* partial, int w_zero,
                                                int bx2, int by, int bz, int gx, int gy, double (*rows)[kPairTy]) {
  if (w_zero)
    pair_tile_sweep_wz<ZC, true>(sw, sr, S, J, wout, partial, bx2, by, bz, gx, gy, rows);
  else
    pair_tile_sweep_wz<ZC, false>(sw, sr, S, J, wout, partial, bx2, by, bz, gx, gy, rows);
}

}  // namespace picard
