// kernels.cuh -- launch wrappers shared between the translation units of
// libpicard_gpu.  Each wrapper enqueues work on `st` and returns the launch
// status; none of them synchronises.
#pragma once

#include "common.cuh"

namespace picard {

// One inflow face of BCinflow.f90 on one rank: loop `outer` x `inner`, the
// fixed index of the face axis, and the lower-edge coordinate of that axis.
struct InflowFace {
  int axis;         // 0 = x face, 1 = y face, 2 = z face
  int fixed;        // 1-based index of the guard layer (1 or N+2)
  int o_lo, o_n;    // outer loop start (1-based) and length
  int i_lo, i_n;    // inner loop start (1-based) and length
  double edge;      // x0 / y0 / z0 of the guard layer
  long long first;  // index of the face's first guard cell in the enumeration
};
struct InflowTable {
  int nfaces;
  InflowFace f[6];
  long long cells;   // guard cells over all faces
  int per_cell;      // particles created per guard cell
  int group_prefix[9];  // slots before species s inside one cell's block
};

struct ReduceBuf {
  double* partial;      // one per block
  double* result;       // device scalar(s)
  int max_blocks;
};

// ---------------------------------------------------------- exact FP64 unit
cudaError_t launch_calc_distance(const KParams& P, double* D, cudaStream_t st);
cudaError_t launch_init_f64(const KParams& P, PartF64 out, long long start, cudaStream_t st);
cudaError_t launch_init_c32(const KParams& P, PartC32 out, long long start, cudaStream_t st);
cudaError_t launch_inflow_f64(const KParams& P, const InflowTable& T, int iteration, PartF64 out, long long start,
                              cudaStream_t st);
cudaError_t launch_inflow_c32(const KParams& P, const InflowTable& T, int iteration, PartC32 out, long long start,
                              cudaStream_t st);
// Fused inflow (fast path): candidates are generated, advanced by dt and kept
// only if BCoutflow would keep them; survivors are appended at *count in
// candidate order.  block_counts holds inflow_blocks(candidates) ints,
// block_offsets that many + 2 + scan_scratch_ints(that many).  With a
// staging area (inflow_stage_slots(candidates) slots: six doubles in planes
// of that stride and a species byte) every candidate is generated once;
// without one (x == nullptr) twice, counted and then emitted.
struct InflowStage {
  double* x = nullptr;
  int8_t* sp = nullptr;
};
long long inflow_stage_slots(long long candidates);
cudaError_t launch_inflow_fused_c32(const KParams& P, const InflowTable& T, int iteration, PartC32 out, int* count,
                                    long long capacity, int* block_counts, int* block_offsets, int* err,
                                    const InflowStage& stage, cudaStream_t st);
cudaError_t launch_inflow_fused_f64(const KParams& P, const InflowTable& T, int iteration, PartF64 out, int* count,
                                    long long capacity, int* block_counts, int* block_offsets, int* err,
                                    const InflowStage& stage, cudaStream_t st);
int inflow_blocks(long long candidates);
// ParticlesProduce: per-cell counts, then emission at offsets[].
cudaError_t launch_produce_count(const KParams& P, int iteration, int* counts, cudaStream_t st);
// Appends at *count (device); offsets[cells] holds the total, added to *count.
cudaError_t launch_produce_emit_f64(const KParams& P, int iteration, const int* offsets, PartF64 out, int* count,
                                    long long capacity, int* err, cudaStream_t st);
cudaError_t launch_produce_emit_c32(const KParams& P, int iteration, const int* offsets, PartC32 out, int* count,
                                    long long capacity, int* err, cudaStream_t st);
cudaError_t launch_advance_position_f64(const KParams& P, PartF64 a, long long n, double dt, cudaStream_t st);
cudaError_t launch_transfer_f64(const KParams& P, PartF64 a, long long n, cudaStream_t st);
// Keep words per 2048-particle BCoutflow block (one per 32 particles).
constexpr int kOutflowWordsPerBlock = 64;
// BCoutflow split around a host read of the survivor count (for callers that
// synchronise anyway): stage 1 marks, scans and writes m, the survivors at or
// above the new count n', to info[0]; stage 2 fills the holes below n', by
// pointer jumping over the window [n', n) when nxt[0] and nxt[1] (n - n' ints
// each) are given, else by following each hole's chain (outflow.cuh).
struct OutflowSplit {
  int stage;
  long long np;  // stage 2: n' (*count after stage 1)
  int* info;     // stage 1: one int
  int* nxt[2];   // stage 2: pointer-jumping scratch, or null
};
// BCoutflow in place, leaving the particles in the reference's order
// (outflow.cuh); *count receives the survivors.  wrap != 0 also applies the
// ParticlesTransfer periodic wrap to them.  words: 64 compact_blocks(n)
// entries; block_counts / block_offsets as for launch_scan_int over
// compact_blocks(n) counts.
cudaError_t launch_outflow_f64(const KParams& P, PartF64 a, long long n, uint2* words, int* block_counts,
                               int* block_offsets, int* count, int wrap, int* err, cudaStream_t st,
                               const OutflowSplit* split = nullptr);
cudaError_t launch_advance_velocity_f64(const KParams& P, PartF64 a, long long n, const double* E, double dt,
                                        double deltat, int mode, cudaStream_t st);
cudaError_t launch_deposit_f64(const KParams& P, PartF64 a, long long n, unsigned long long* Nacc,
                               unsigned long long* Facc, cudaStream_t st);
cudaError_t launch_energy_particles_f64(const KParams& P, PartF64 a, long long n, ReduceBuf rb, cudaStream_t st);
cudaError_t launch_cell_indices_f64(const KParams& P, PartF64 a, long long n, int* ijk, cudaStream_t st);

// ------------------------------------------------------------ CELL32 unit
cudaError_t launch_advance_position_c32(const KParams& P, PartC32 a, long long n, double dt, cudaStream_t st);
// AdvanceVelocity (dt) then the next step's AdvancePosition (dt) in one pass; bit-identical to the two launches.
cudaError_t launch_push_advance_c32(const KParams& P, PartC32 a, long long n, const float4* E, double dt,
                                    cudaStream_t st);
cudaError_t launch_transfer_c32(const KParams& P, PartC32 a, long long n, cudaStream_t st);
cudaError_t launch_outflow_c32(const KParams& P, PartC32 a, long long n, uint2* words, int* block_counts,
                               int* block_offsets, int* count, int wrap, int* err, cudaStream_t st,
                               const OutflowSplit* split = nullptr);
cudaError_t launch_advance_velocity_c32(const KParams& P, PartC32 a, long long n, const float4* E, double dt,
                                        double deltat, int mode, cudaStream_t st);
cudaError_t launch_deposit_c32(const KParams& P, PartC32 a, long long n, unsigned long long* Nacc,
                               unsigned long long* Facc, cudaStream_t st);
cudaError_t launch_energy_particles_c32(const KParams& P, PartC32 a, long long n, ReduceBuf rb, cudaStream_t st);
cudaError_t launch_c32_to_f64(const KParams& P, PartC32 a, long long n, PartF64 out, cudaStream_t st);
cudaError_t launch_f64_to_c32(const KParams& P, PartF64 a, long long n, PartC32 out, cudaStream_t st);
// ------------------------------------------------------------ scans
// Exclusive scan of n int32 counts into offsets; *total receives the sum.
cudaError_t launch_scan_int(const int* in, int* out, int n, int* total, int* scratch, cudaStream_t st);
int scan_scratch_ints(int n);
int compact_blocks(long long n);

}  // namespace picard
