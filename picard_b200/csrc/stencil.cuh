// stencil.cuh -- node addressing of the FP32 Jacobi arrays and the FP32
// Jacobi update shared by every sweep kernel.
#pragma once

#include "common.cuh"
#include "grid.cuh"

namespace picard {

struct Stencil {
  int nx, ny, nz, nxp, nyp;
  int px, py, pz;  // periodic axes
  long long nodes;
  int fpitch;      // row pitch (floats) of the FP32 solver arrays
};

Stencil make_stencil(const KParams& P);
JacobiCoefF jacobi_coef_f(const KParams& P);

// FP32 solver arrays (increment w, scaled residual r) are padded: node
// (i, j, k) sits at column i + 3 of a row of fpitch floats, fpitch a multiple
// of 8.  Interior rows then start on 16-byte boundaries (column 4) and every
// TMA box origin (column 32 b) is 16-byte aligned.
__host__ __device__ inline long long fidx(const Stencil& S, int i, int j, int k) {
  return (long long)(i + 3) + (long long)S.fpitch * ((long long)j + (long long)S.nyp * k);
}

// One node of an FP32 sweep of the increment (CalcEpotential.f90:50-56 on
// the increment): res = r - L w with
//   L w = (w(x+1) + w(x-1) - 2 w) / dx^2 + (y) + (z),
// then w' = w - af res and the squared residual accumulates as r2 + res^2.
// Every rounding is explicit, so each sweep kernel -- whatever its tiling,
// staging or launch shape -- gives every node and every per-tile partial the
// same bits.
__device__ __forceinline__ float jacobi_res_f32(const JacobiCoefF& J, float wc, float xm, float xp, float ym,
                                                float yp, float zm, float zp, float r) {
  const float sx = __fadd_rn(xp, xm);
  const float sy = __fadd_rn(yp, ym);
  const float sz = __fadd_rn(zp, zm);
  float lap = __fmul_rn(__fmaf_rn(-2.0f, wc, sx), J.idx2);
  lap = __fmaf_rn(__fmaf_rn(-2.0f, wc, sy), J.idy2, lap);
  lap = __fmaf_rn(__fmaf_rn(-2.0f, wc, sz), J.idz2, lap);
  return __fsub_rn(r, lap);
}
__device__ __forceinline__ float jacobi_next_f32(const JacobiCoefF& J, float wc, float res) {
  return __fmaf_rn(-J.af, res, wc);
}
__device__ __forceinline__ float acc_r2_f32(float r2, float res) { return __fmaf_rn(res, res, r2); }

}  // namespace picard
