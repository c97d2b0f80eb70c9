// tile32.cuh -- one 32 x 8 x ZC tile of an FP32 Jacobi sweep of the
// increment, one node per thread, shared by the single-run TMA sweep kernel
// and the batched multi-run kernel so that both compute every node and every
// partial identically.  The tile's w box (40 x 10 x (ZC+2), origin the
// aligned column 32 bx) and r box (32 x 8 x ZC, origin the tile's first
// interior column) are in shared memory.
#pragma once

#include "stencil.cuh"

namespace picard {

constexpr int kT32Tx = 32, kT32Ty = 8, kT32BoxX = 40;

// Sum of v over the block (32-lane shuffle tree in double, then the warps'
// sums in warp order by thread 0) into *out.  Ends with the block's threads
// past a barrier.
__device__ inline void block_sum_store(double v, double* out) {
  __shared__ double sh[32];
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  int t = threadIdx.x + blockDim.x * threadIdx.y;
  if ((t & 31) == 0) sh[t >> 5] = v;
  __syncthreads();
  if (t == 0) {
    double s = 0.0;
    int nw = (blockDim.x * blockDim.y) >> 5;
    for (int w = 0; w < nw; ++w) s += sh[w];
    *out = s;
  }
}

// Sweep of the tile (bx, by, bz); its partial (sum over the tile of the
// squared residuals, per-column FP32 sums in z order) goes to *partial.
template <int ZC>
__device__ __forceinline__ void tile32_sweep(const float* sw, const float* sr, const Stencil& S, const JacobiCoefF& J,
                                             float* wout, double* partial, int w_zero, int bx, int by, int bz) {
  const int tx = threadIdx.x, ty = threadIdx.y;
  const long long plane = (long long)S.fpitch * S.nyp;
  const int x0 = bx * kT32Tx, y0 = by * kT32Ty, z0 = bz * ZC;
  const int i = x0 + tx + 1, j = y0 + ty + 1;
  float r2 = 0.0f;
  if (i <= S.nx && j <= S.ny) {
    const int kend = min(ZC, S.nz - z0);
    long long c = fidx(S, i, j, z0 + 1);
    const int col = tx + 4;  // smem column of node i
    if (w_zero) {
      for (int kk = 1; kk <= kend; ++kk, c += plane) {
        float res = sr[((kk - 1) * kT32Ty + ty) * kT32Tx + tx];
        r2 = acc_r2_f32(r2, res);
        wout[c] = jacobi_next_f32(J, 0.0f, res);
      }
    } else {
      auto W = [&](int kk, int row, int cc) { return sw[(kk * (kT32Ty + 2) + row) * kT32BoxX + cc]; };
      float wm = W(0, ty + 1, col);
      float wc = W(1, ty + 1, col);
      for (int kk = 1; kk <= kend; ++kk, c += plane) {
        float wp = W(kk + 1, ty + 1, col);
        float res = jacobi_res_f32(J, wc, W(kk, ty + 1, col - 1), W(kk, ty + 1, col + 1), W(kk, ty, col),
                                   W(kk, ty + 2, col), wm, wp, sr[((kk - 1) * kT32Ty + ty) * kT32Tx + tx]);
        r2 = acc_r2_f32(r2, res);
        wout[c] = jacobi_next_f32(J, wc, res);
        wm = wc;
        wc = wp;
      }
    }
  }
  block_sum_store((double)r2, partial);
}

}  // namespace picard
