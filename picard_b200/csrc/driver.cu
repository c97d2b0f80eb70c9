// driver.cu -- host mirror of `program picard` (picard.f90): the parameter
// defaults (145-302), the derived quantities (333-467) and the main loop
// (554-674), calling the per-subroutine entry points in the reference's order.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <string>

#include "context.cuh"
#include "picard_gpu.h"
#include "picard_io.h"

using namespace picard;

extern "C" {

// picard.f90:145-302 on one rank (iprocs = jprocs = kprocs = 1).
int picard_params_default(picard_params* p) {
  if (!p) return fail(PICARD_ERR_BAD_ARG, "params is NULL");
  std::memset(p, 0, sizeof(*p));
  p->nx = p->ny = p->nz = 30;
  p->species = 3;
  p->max_per_proc = 1 << 24;
  p->xflow = p->yflow = p->zflow = 1;
  p->maxit = 1 << 20;
  p->produce_dt_scaled = 0;
  p->xmin = p->ymin = p->zmin = -600.0;
  p->xmax = p->ymax = p->zmax = 600.0;
  p->dt = 4.0e-6;
  p->maxerr = std::pow(2.0, -16);
  for (int s = 0; s < 8; ++s) {
    p->gyration[s] = 1;
    p->fluid[s] = 0;
  }
  p->mass[0] = kMe;
  p->mass[1] = kMp * 1.0;
  p->mass[2] = kMp * 18.0;
  p->mass[3] = kMp * 4.0;
  p->mass[4] = kMp * 44.0;
  p->mass[5] = p->mass[6] = p->mass[7] = kMp * 1.0;
  for (int s = 2; s < 8; ++s) p->charge[s] = kEc;
  p->density[1] = 1.07e6;
  p->ppc[1] = 64;
  p->kelvin[0] = 8.02e4;
  p->kelvin[1] = 4.27e4;
  p->kelvin[2] = 4.27e4;
  for (int s = 0; s < 8; ++s) {
    p->v0[s][0] = -430.0e3;
    p->v0[s][1] = 0.0;
    p->v0[s][2] = 0.0;
  }
  p->B0[0] = 0.0;
  p->B0[1] = 400.0 * 1.78e-9;
  p->B0[2] = 0.0;
  p->vn[2] = 629.0;
  p->Qn[2] = std::pow(400.0, -3) * 1.99e26;
  p->Ek[2] = 1.0 * 1.52e1 * kEc;
  p->nu_i[2] = 1.26e-7;
  p->nu_d[2] = 1.26e-7;
  return PICARD_OK;
}

// picard.f90:333-467 on one rank.
int picard_params_derive(picard_params* p) {
  if (!p) return fail(PICARD_ERR_BAD_ARG, "params is NULL");
  if (p->nx < 1 || p->ny < 1 || p->nz < 1) return fail(PICARD_ERR_BAD_ARG, "grid dimensions must be positive");
  const double Lx = p->xmax - p->xmin, Ly = p->ymax - p->ymin, Lz = p->zmax - p->zmin;
  if (!(Lx > 0.0 && Ly > 0.0 && Lz > 0.0)) return fail(PICARD_ERR_BAD_ARG, "empty domain");
  const double Lx_local = Lx / 1.0, Ly_local = Ly / 1.0, Lz_local = Lz / 1.0;
  p->Lx_min = p->xmin + Lx_local * 0.0;
  p->Lx_max = p->Lx_min + Lx_local;
  p->Ly_min = p->ymin + Ly_local * 0.0;
  p->Ly_max = p->Ly_min + Ly_local;
  p->Lz_min = p->zmin + Lz_local * 0.0;
  p->Lz_max = p->Lz_min + Lz_local;
  p->dxyz[0] = Lx_local / (double)p->nx;
  p->dxyz[1] = Ly_local / (double)p->ny;
  p->dxyz[2] = Lz_local / (double)p->nz;
  p->dV = p->dxyz[0] * p->dxyz[1] * p->dxyz[2];
  // electrons quasi-neutralise (363-381)
  p->vn[0] = p->Qn[0] = p->Ek[0] = p->nu_i[0] = p->nu_d[0] = 0.0;
  p->charge[0] = -kEc;
  p->charge[1] = kEc;
  for (int s = 1; s < 8; ++s) p->density[s] = p->density[s] * (double)p->ppc[s] / (double)(p->ppc[s] > 1 ? p->ppc[s] : 1);
  double acc = 0.0;
  for (int s = 1; s < 8; ++s) acc += -p->density[s] * p->charge[s];
  p->density[0] = acc * (1.0 / p->charge[0]);
  for (int s = 0; s < 8; ++s)
    if (p->density[s] <= 0.0 || p->species < s + 1) {
      p->ppc[s] = 0;
      p->density[s] = 0.0;
    }
  acc = 0.0;
  for (int s = 1; s < 8; ++s) acc += -p->density[s] * p->charge[s] / p->charge[0];
  p->density[0] = acc;
  // particles per cell (384-392)
  for (int s = 0; s < 8; ++s) {
    int e = (int)(0.5 - p->charge[s] / p->charge[0]);
    int h = (int)(0.5 - p->charge[s] / p->charge[1]);
    p->epp[s] = e > 0 ? e : 0;
    p->hpp[s] = h > 0 ? h : 0;
  }
  p->hpp[0] = 0;
  for (int s = 2; s < 8; ++s) p->ipp[s] = p->ppc[s];
  int sh = 0;
  for (int s = 2; s < 8; ++s) sh += p->ipp[s] * p->hpp[s];
  p->ipp[1] = p->ppc[1] - sh;
  p->ipp[0] = 0;
  int se = 0;
  for (int s = 1; s < 8; ++s) se += p->ipp[s] * p->epp[s];
  p->ppc[0] = se;
  // macro-particle weights (394-401)
  for (int s = 0; s < 8; ++s) p->n2p[s] = 0.0;
  for (int s = 0; s < 8; ++s) p->n2p[s] = p->ppc[s] > 0 ? p->dV * p->density[s] * (1.0 / (double)p->ppc[s]) : p->n2p[0];
  for (int s = 0; s < 8; ++s) p->eta[s] = p->charge[s] / p->mass[s];
  // mass-weighted bulk velocity (408-413)
  for (int c = 0; c < 3; ++c) {
    double num = 0.0, den = 0.0;
    for (int s = 0; s < 8; ++s) {
      double w = (double)p->ipp[s] * (p->n2p[s] * p->mass[s] + (double)p->epp[s] * p->n2p[0] * p->mass[0] +
                                      (double)p->hpp[s] * p->n2p[1] * p->mass[1]);
      num += w * p->v0[s][c];
      den += w;
    }
    p->ve[c] = num / den;
  }
  for (int s = 0; s < 8; ++s)
    p->v0[s][3] = std::sqrt(p->v0[s][0] * p->v0[s][0] + p->v0[s][1] * p->v0[s][1] + p->v0[s][2] * p->v0[s][2]);
  p->ve[3] = std::sqrt(p->ve[0] * p->ve[0] + p->ve[1] * p->ve[1] + p->ve[2] * p->ve[2]);
  p->B0[3] = std::sqrt(p->B0[0] * p->B0[0] + p->B0[1] * p->B0[1] + p->B0[2] * p->B0[2]);
  // motional field E0 = -ve x B0 (424-427)
  p->E0[0] = p->ve[2] * p->B0[1] - p->ve[1] * p->B0[2];
  p->E0[1] = p->ve[0] * p->B0[2] - p->ve[2] * p->B0[0];
  p->E0[2] = p->ve[1] * p->B0[0] - p->ve[0] * p->B0[1];
  p->E0[3] = std::sqrt(p->E0[0] * p->E0[0] + p->E0[1] * p->E0[1] + p->E0[2] * p->E0[2]);
  // Boris factors (452-466)
  for (int s = 0; s < 8; ++s)
    for (int c = 0; c < 4; ++c) p->tB[s][c] = p->gyration[s] ? 0.5 * p->dt * p->B0[c] * p->eta[s] : 0.0;
  for (int s = 0; s < 8; ++s) {
    double d = 1.0 + p->tB[s][3] * p->tB[s][3];
    for (int c = 0; c < 4; ++c) p->sB[s][c] = 2.0 * p->tB[s][c] / d;
  }
  // energy normalisation (476-480)
  const double vol = Lx * Ly * Lz;
  const double uE0 = 0.5 * (p->E0[3] * p->E0[3] * kEps0) * vol;
  const double uB0 = 0.5 * (p->B0[3] * p->B0[3] / kMu0) * vol;
  double up = 0.0;
  for (int s = 0; s < 8; ++s)
    up += p->density[s] * (p->mass[s] * p->v0[s][3] * p->v0[s][3] + 3.0 * kKb * p->kelvin[s]);
  p->u0 = uE0 + uB0 + 0.5 * up * vol;
  return PICARD_OK;
}

static int log_energy(picard_ctx* c, int32_t it, double time, picard_log_fn fn, void* user) {
  double e[3];
  int32_t n;
  PICARD_TRY(picard_gpu_energy(c, e, &n));
  const double u0 = c->prm.u0;
  if (fn) fn(it, time, n, e[0] / u0, e[1] / u0, e[2] / u0, user);
  return PICARD_OK;
}

// The end of a step on a write step (picard.f90:602-621): the velocity push
// split around the dumps.
static int write_step(picard_ctx* c, double time, picard_io* io) {
  const picard_params& p = c->prm;
  const bool wp = io->write_particles && std::fmod(time, io->particles_interval) < p.dt;
  const bool wf = io->write_fields && std::fmod(time, io->fields_interval) < p.dt;
  PICARD_TRY(picard_gpu_advance_velocity_imp(c, 0.5 * p.dt, p.dt));
  if (wp) PICARD_TRY(picard_gpu_dump_particles(c, io->root, &io->particles_iteration));
  if (wf) {
    PICARD_TRY(picard_gpu_particles_gridify_all(c));
    PICARD_TRY(picard_gpu_dump_fields(c, io->root, &io->fields_iteration));
  }
  return picard_gpu_advance_velocity_exp(c, 0.5 * p.dt, p.dt);
}

// picard.f90:554-674; io == NULL: writeFields = writeParticles = .false.
static int run_loop(picard_ctx* c, int32_t iter_start, int32_t iter_end, int32_t log_interval, picard_log_fn log_fn,
                    void* user, picard_io* io, int64_t* sweeps_total) {
  const picard_params& p = c->prm;
  double time = (double)iter_start * p.dt;
  bool nc = false;
  for (int32_t it = iter_start + 1; it <= iter_end; ++it) {
    time = time + p.dt;
    // ParticlesModifyExp(): empty in the reference (ParticlesModify.f90:2-7)
    PICARD_TRY(picard_gpu_bc_inflow(c, it));
    PICARD_TRY(picard_gpu_advance_position(c, p.dt));
    PICARD_TRY(picard_gpu_particles_produce(c, it));
    PICARD_TRY(picard_gpu_bc_outflow(c));
    PICARD_TRY(picard_gpu_particles_transfer(c));
    PICARD_TRY(picard_gpu_particles_gridify(c));
    PICARD_TRY(picard_gpu_bc_potentials(c));
    int32_t sw = 0;
    int rc = picard_gpu_calc_epotential(c, p.maxerr, p.maxit, &sw);
    if (rc == PICARD_ERR_NOT_CONVERGED)
      nc = true;  // the reference prints a warning and carries on
    else if (rc != PICARD_OK)
      return rc;
    if (sweeps_total) *sweeps_total += sw;
    PICARD_TRY(picard_gpu_calc_efield(c));
    PICARD_TRY(picard_gpu_bc_fields(c));
    // ParticlesModifyImp(): empty (ParticlesModify.f90:9-14)
    const bool writing = io && (io->write_fields || io->write_particles) &&
                         ((io->write_fields && std::fmod(time, io->fields_interval) < p.dt) ||
                          (io->write_particles && std::fmod(time, io->particles_interval) < p.dt));
    if (writing)
      PICARD_TRY(write_step(c, time, io));
    else
      PICARD_TRY(picard_gpu_advance_velocity(c, p.dt));
    c->stats.steps += 1;
    c->stats.particle_steps += c->num_local;
    if (log_interval > 0 && it % log_interval == 0) PICARD_TRY(log_energy(c, it, time, log_fn, user));
  }
  PICARD_CUDA(cudaStreamSynchronize(c->st));
  if (nc) return fail(PICARD_ERR_NOT_CONVERGED, "at least one Jacobi solve hit 2*maxit+1 sweeps");
  return PICARD_OK;
}

int picard_gpu_run(picard_ctx* c, int32_t iter_start, int32_t iter_end, int32_t log_interval, picard_log_fn log_fn,
                   void* user, int64_t* sweeps_total) {
  if (!c) return fail(PICARD_ERR_BAD_ARG, "ctx is NULL");
  return run_loop(c, iter_start, iter_end, log_interval, log_fn, user, nullptr, sweeps_total);
}

int picard_gpu_run_io(picard_ctx* c, int32_t iter_start, int32_t iter_end, int32_t log_interval, picard_log_fn log_fn,
                      void* user, picard_io* io, int64_t* sweeps_total) {
  if (!c || !io) return fail(PICARD_ERR_BAD_ARG, "NULL argument");
  if ((io->write_fields && !(io->fields_interval > 0.0)) ||
      (io->write_particles && !(io->particles_interval > 0.0)))
    return fail(PICARD_ERR_BAD_ARG, "write interval must be positive");
  return run_loop(c, iter_start, iter_end, log_interval, log_fn, user, io, sweeps_total);
}

// The same iterations with the inflow candidates generated, advanced and
// filtered in one kernel (only survivors are stored), production appended
// before a single compaction that also applies the periodic wrap.
int picard_gpu_run_fused(picard_ctx* c, int32_t iter_start, int32_t iter_end, int64_t* sweeps_total) {
  if (!c) return fail(PICARD_ERR_BAD_ARG, "ctx is NULL");
  const picard_params& p = c->prm;
  const KParams& K = c->K;
  const int cells = p.nx * p.ny * p.nz;
  bool nc = false;
  bool advanced = false;  // the previous step's push already advanced the positions
  for (int32_t it = iter_start + 1; it <= iter_end; ++it) {
    PICARD_CUDA(cudaEventRecord(c->pev[0], c->st));
    // AdvancePosition on the particles present before BCinflow
    if (!advanced) PICARD_TRY(picard_gpu_advance_position(c, p.dt));
    // ParticlesProduce, appended behind them (device-side count)
    PICARD_CUDA(launch_produce_count(K, it, c->cell_counts, c->st));
    PICARD_CUDA(launch_scan_int(c->cell_counts, c->cell_offsets, cells, c->cell_offsets + cells,
                                c->cell_offsets + cells + 2, c->st));
    if (c->layout == PICARD_LAYOUT_F64)
      PICARD_CUDA(launch_produce_emit_f64(K, it, c->cell_offsets, c->f64, c->d_count, c->capacity,
                                          c->d_err, c->st));
    else
      PICARD_CUDA(launch_produce_emit_c32(K, it, c->cell_offsets, c->c32, c->d_count, c->capacity,
                                          c->d_err, c->st));
    PICARD_TRY(sync_count_public(c));
    // BCoutflow + ParticlesTransfer in place, in the reference's order
    PICARD_CUDA(launch_outflow(c, 1));
    // BCinflow + AdvancePosition + BCoutflow + ParticlesTransfer of the new particles
    PICARD_CUDA(launch_inflow_fused(c, it));
    PICARD_TRY(sync_count_public(c));
    // ParticlesTransfer's slot: every sort_every iterations, the particles
    // put back in cell order (a permutation; nothing downstream depends on it)
    if (c->sort_every > 0 && it % c->sort_every == 0) PICARD_TRY(sort_particles(c));
    PICARD_CUDA(cudaEventRecord(c->pev[1], c->st));
    PICARD_TRY(picard_gpu_particles_gridify(c));
    PICARD_CUDA(cudaEventRecord(c->pev[2], c->st));
    PICARD_TRY(bc_potentials_async(c));  // a timeout surfaces through the solve's error check
    PICARD_CUDA(cudaEventRecord(c->pev[3], c->st));
    int32_t sw = 0;
    int rc = picard_gpu_calc_epotential(c, p.maxerr, p.maxit, &sw);
    if (rc == PICARD_ERR_NOT_CONVERGED)
      nc = true;
    else if (rc != PICARD_OK)
      return rc;
    if (sweeps_total) *sweeps_total += sw;
    PICARD_CUDA(cudaEventRecord(c->pev[4], c->st));
    PICARD_TRY(picard_gpu_calc_efield(c));
    // AdvanceVelocity; in the CELL32 layout, when another step follows, fused
    // with that step's AdvancePosition (one pass over the particles)
    advanced = c->layout == PICARD_LAYOUT_CELL32 && it < iter_end;
    if (advanced)
      PICARD_CUDA(launch_push_advance_c32(K, c->c32, c->num_local, c->E32, p.dt, c->st));
    else
      PICARD_TRY(picard_gpu_advance_velocity(c, p.dt));
    PICARD_CUDA(cudaEventRecord(c->pev[5], c->st));
    PICARD_CUDA(cudaEventSynchronize(c->pev[5]));
    for (int ph = 0; ph < 5; ++ph) {
      float ms = 0.0f;
      if (cudaEventElapsedTime(&ms, c->pev[ph], c->pev[ph + 1]) == cudaSuccess) c->stats.phase_ms[ph] += ms;
    }
    c->stats.steps += 1;
    c->stats.particle_steps += c->num_local;
  }
  PICARD_CUDA(cudaStreamSynchronize(c->st));
  PICARD_TRY(check_dev_err_public(c));  // a wait that gave up in the last step
  if (nc) return fail(PICARD_ERR_NOT_CONVERGED, "at least one Jacobi solve hit 2*maxit+1 sweeps");
  return PICARD_OK;
}

}  // extern "C"
