// grid.cuh -- launch wrappers of grid.cu (node-array kernels).
#pragma once

#include "common.cuh"

namespace picard {

// CalcEpotential.f90:44-47 coefficients and the squared cell sizes.
struct JacobiCoef {
  double ax, ay, az, af;
  double dx2, dy2, dz2;
};
struct JacobiCoefF {
  float af, idx2, idy2, idz2;
};
// Launch shape of the sweep kernels: (32, 8) threads over (x, y), each
// thread marching zc nodes along z.
struct JacobiGeom {
  dim3 grid, block;
  int zc;
  int nblocks;
};

JacobiGeom jacobi_geom(const KParams& P);
JacobiCoef jacobi_coef(const KParams& P);

cudaError_t launch_finish_deposit(const KParams& P, const unsigned long long* Nacc, double* N, double* C,
                                  cudaStream_t st);
cudaError_t launch_finish_flux(const KParams& P, const unsigned long long* Facc, double* F, cudaStream_t st);
cudaError_t launch_bc_potentials(const KParams& P, const double* C, const double* D, double* U, cudaStream_t st);
int rhs_blocks(const KParams& P);
cudaError_t launch_rhs(const KParams& P, const double* C, double* b, double* partial, double* bnorm2,
                       cudaStream_t st);
cudaError_t launch_sweep_f64(const KParams& P, const JacobiGeom& G, const double* Uin, double* Uout, const double* b,
                             double* partial, cudaStream_t st);
cudaError_t launch_sweep_f32(const KParams& P, const JacobiGeom& G, const float* win, float* wout, const float* r,
                             double* partial, int w_zero, cudaStream_t st);
cudaError_t launch_anchor(const KParams& P, const JacobiGeom& G, const double* Vin, double* Vout, const float* w,
                          const double* b, float* r, double sigma, double* partial, int w_zero, cudaStream_t st);
cudaError_t launch_finalize(const KParams& P, const double* V, const float* w, double sigma, double* U, int w_zero,
                            cudaStream_t st);
cudaError_t launch_refresh_periodic(const KParams& P, double* U, cudaStream_t st);
cudaError_t launch_reduce_sweeps(const double* partial, int nb, int m, double* r2, cudaStream_t st);
cudaError_t launch_efield(const KParams& P, const double* U, double* E, float4* E32, cudaStream_t st);
cudaError_t launch_bc_fields(const KParams& P, double* E, float4* E32, cudaStream_t st);
cudaError_t launch_energy_field(const KParams& P, const double* E, double* partial, double* out, cudaStream_t st);

}  // namespace picard
