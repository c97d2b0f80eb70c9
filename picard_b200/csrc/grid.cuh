// grid.cuh -- launch wrappers of grid.cu (node-array kernels).
#pragma once

#include <cuda.h>

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
  int tma;  // all axes open: the TMA-staged sweep kernel is used (zc in {4, 8, 16})
  // TMA sweep launch shape (results do not depend on it): CTAs of the
  // persistent grid (0: one per tile) and programmatic dependent launch
  int ctas = 0;
  int pdl = 1;
  int stages = 1;  // shared-memory stages per CTA (2: the next tile is prefetched)
  int pairs = 0;   // 1: the x-pair kernel (64-wide tiles)
  int fused2 = 0;  // 1 (with pairs): two sweeps per launch where a batch allows
  int rglobal = 0; // 1 (with pairs, one CTA per tile, one stage, or fused2): r read from global memory
  // register-resident sweeps (jacobi_resident.cu): one cooperative launch per
  // batch of sweeps over CTAs of 32 x res_by x res_nz nodes
  int res = 0;
  int res_by = 0, res_nz = 0, res_cgx = 0, res_cgy = 0, res_cgz = 0, res_ctas = 0;
};
// Plans the resident sweep with CTA shape `shape_index` (0 = smallest);
// returns 1 and fills G.res* when all its CTAs can be co-resident on the
// current device, else 0 (G.res = 0).
int resident_plan(const KParams& P, JacobiGeom& G, int shape_index);
constexpr int kResidentShapes = 5;
// Floats of the face-exchange buffer the planned resident sweep needs.
long long resident_face_floats(const JacobiGeom& G);
// m sweeps (the first from w = 0 when w_zero, else from win) in one
// cooperative launch: partial[t * nblocks + tile] for t < m, w of the last
// sweep to wout.  bar: one counter, zeroed here.
cudaError_t launch_sweeps_resident(const KParams& P, const JacobiGeom& G, const float* r, const float* win,
                                   float* wout, float* faces, unsigned int* bar, double* partial, int m, int w_zero,
                                   int* err, cudaStream_t st, int wait_test = 0);
// The x-pair TMA sweep (64-wide tiles; w boxes 72 x 10 x zc+2, r boxes 64 x
// 8 x zc): launch, occupancy and tile count.  Writes the same partials (in
// the 32-wide tile layout) as launch_sweep_tma.  With G.rglobal, one CTA per
// tile and one stage, r is read from global memory (r, the padded array tr
// describes) and only the w box is staged.
cudaError_t launch_sweep_tma2(const KParams& P, const JacobiGeom& G, const CUtensorMap* tw, const CUtensorMap* tr,
                              const float* r, float* wout, double* partial, int w_zero, int* err, cudaStream_t st);
int sweep_tma2_occupancy(const JacobiGeom& G, int stages);
// Sweeps s and s+1 in one launch (x pairs, temporal blocking; zc 4 or 8):
// reads w_{s-1} through tw (boxes 72 x 12 x zc+4) and r through tr (boxes 72 x
// 10 x zc+2) -- or, with G.rglobal, r from global memory at r -- writes
// w_{s+1} and the partials of sweep s (partialA) and s+1 (partialB);
// bit-identical to two launch_sweep_tma2 calls.
cudaError_t launch_sweep2_tma(const KParams& P, const JacobiGeom& G, const CUtensorMap* tw, const CUtensorMap* tr,
                              const float* r, float* wout, double* partialA, double* partialB, int w_zero, int* err,
                              cudaStream_t st);
int sweep_tma2_tiles(const KParams& P, const JacobiGeom& G);
// CTAs of one SM the TMA sweep kernel of this geometry can hold.
int sweep_tma_occupancy(const JacobiGeom& G, int stages);

// Row pitch (floats) of the padded FP32 solver arrays: node (i, j, k) at
// column i + 3, rows a multiple of 8 floats (32 bytes).
int f32_pitch(const KParams& P);
long long f32_elems(const KParams& P);
// TMA descriptor of one padded FP32 array with box_x x box_y x box_z boxes
// (w: 40 x 10 x zc+2 from the aligned column below the tile's halo; r: 32 x 8
// x zc from the tile's first interior column).  Returns a CUresult.
int make_tensor_map(CUtensorMap* m, float* base, const KParams& P, int box_x, int box_y, int box_z);
cudaError_t launch_sweep_tma(const KParams& P, const JacobiGeom& G, const CUtensorMap* tw, const CUtensorMap* tr,
                             float* wout, double* partial, int w_zero, int* err, cudaStream_t st);

JacobiGeom jacobi_geom(const KParams& P);
JacobiCoef jacobi_coef(const KParams& P);

cudaError_t launch_finish_deposit(const KParams& P, const unsigned long long* Nacc, double* N, double* C,
                                  cudaStream_t st);
cudaError_t launch_finish_flux(const KParams& P, const unsigned long long* Facc, double* F, cudaStream_t st);
cudaError_t launch_bc_potentials(const KParams& P, const double* C, const double* D, double* U, cudaStream_t st);
// Tensor-core BCpotentials (bcpot_tc.cu): scratch sizes (bf16 split charge,
// FP64 per-CTA partial tiles) and the launch.
void bcpot_tc_scratch(const KParams& P, long long* cs_elems, long long* partial_elems);
size_t bcpot_tc_smem_bytes(const KParams& P);
cudaError_t launch_bc_potentials_tc(const KParams& P, const double* C, const double* D, double* U, void* cs_buf,
                                    double* partial, int* err, cudaStream_t st);
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
