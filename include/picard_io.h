/*
 * picard_io.h -- C ABI of Picard's output path: the write-step branch of the
 * main loop (picard.f90:602-627), the text dumps of Write.f90 and the plasma
 * parameter summary and warnings of WriteWarnings.f90.
 *
 * None of this is in the timed loop of a benchmark (the reference's writes are
 * off there); it is what a Fortran host that sets writeFields / writeParticles
 * needs to keep its files and the Python readers of example_fieldplot.py /
 * example_particleplot.py working.  Files are written by the host from device
 * state copied back at the write step.
 */
#ifndef PICARD_IO_H
#define PICARD_IO_H

#include <stdint.h>

#include "picard_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Fortran Ew.d edit descriptor, scale factor 0 (the E10.4 of Write.f90 and the
 * E12.6 of WriteWarnings.f90): mantissa 0.d..d with d digits, correctly rounded
 * from the binary value; the leading zero is dropped when the sign takes its
 * place; exponents of three digits lose the letter E (0.1234+100); values that
 * do not fit are w asterisks.  NaN and Infinity are right-justified words.
 * out receives w characters and a terminating NUL (w <= 64, d < w). */
PICARD_API int picard_format_e(double value, int32_t w, int32_t d, char* out);

/* DumpParticles (Write.f90:1-31): <root>/particles/particles_IIIII_RRRRR, one
 * line per live particle with x, y, z, vx, vy, vz and the species number as
 * seven E10.4 fields, in the device's storage order (the reference writes its
 * own storage order; the set of lines is what matches).  III.. is
 * *write_iteration (I5.5), RRRRR the rank (00000 for the one device domain).
 * Increments *write_iteration like the reference. */
PICARD_API int picard_gpu_dump_particles(picard_ctx* ctx, const char* root, int32_t* write_iteration);

/* DumpFields (Write.f90:34-523): <root>/fields/{UE,Ex,Ey,Ez}_IIIII_RRRRR and
 * N#, X#, Y#, Z# (density and flux x, y, z of species # = 1..species), one E10.4
 * value per line, x fastest over the (Nx+2)(Ny+2)(Nz+2) nodes ghosts included.
 * N and F are those of the last ParticlesGridifyAll (picard_gpu_particles_gridify_all).
 * Increments *write_iteration. */
PICARD_API int picard_gpu_dump_fields(picard_ctx* ctx, const char* root, int32_t* write_iteration);

/* Plasma quantities of WriteWarnings.f90:40-115 for a derived parameter block:
 * index 0 simulation electrons (species 1), 1 the largest over species 2..8,
 * 2 physical electrons. */
typedef struct picard_plasma {
  double wp[3], wc[3], va, vc[3], Ld[3], rL[3], rPU[3], Li[3], sd, rM[3];
  double cfl;                 /* dx/dt                                   */
  double freq;                /* 1/dt                                    */
  double dt_c, dt_opt_part, dt_opt_wave, dt_opt, dt_rec;
  double vth[8];
  uint32_t warnings;          /* bit k set: warning k of picard_warning   */
} picard_plasma;

/* The warnings of WriteWarnings.f90:261-496, in the reference's order. */
typedef enum picard_warning {
  PICARD_WARN_WP_E = 0,      /* wp_e > 1/dt          */
  PICARD_WARN_WP_I = 1,      /* wp_i > 1/dt          */
  PICARD_WARN_WC_E = 2,      /* wc_e > 1/dt          */
  PICARD_WARN_WC_I = 3,      /* wc_i > 1/dt          */
  PICARD_WARN_VA = 4,        /* va > dx/dt           */
  PICARD_WARN_V_E = 5,       /* v_e > dx/dt          */
  PICARD_WARN_V_I = 6,       /* v_i > dx/dt          */
  PICARD_WARN_LD_E = 7,      /* Ld_e < dx            */
  PICARD_WARN_LD_I = 8,      /* Ld_i < dx            */
  PICARD_WARN_RL_E = 9,      /* rL_e < dx            */
  PICARD_WARN_RL_I = 10,     /* rL_i < dx            */
  PICARD_WARN_RPU_E = 11,    /* rPU_e < dx           */
  PICARD_WARN_RPU_I = 12,    /* rPU_i < dx           */
  PICARD_WARN_LI_E = 13,     /* Li_e < dx            */
  PICARD_WARN_LI_I = 14,     /* Li_i < dx            */
  PICARD_WARN_IRREGULAR = 15,/* dx, dy, dz differ    */
  PICARD_WARN_IONIZING = 16, /* sum(Qn * ppc) > 0    */
  PICARD_WARN_COUNT = 17
} picard_warning;

/* WriteWarnings.f90:40-496 without the output: the quantities and the warning
 * mask.  p must be derived (picard_params_derive). */
PICARD_API int picard_params_plasma(const picard_params* p, picard_plasma* out);
/* Short text of warning k ("wp_e > 1/dt", ...), NULL if k is out of range. */
PICARD_API const char* picard_warning_text(int32_t k);

/* WriteWarnings.f90:129-255 and 258-496: <root>/parameters.dat (name = value
 * lines, E12.6 / I4 / T-F, the layout loadPar of the reference's plot scripts
 * reads) and <root>/warnings.dat (one block per warning).  Writes *warnings
 * (may be NULL) with the mask. */
PICARD_API int picard_write_parameters(const picard_params* p, const char* root, uint32_t* warnings);

/* Output switches of picard.f90:146-147, 166-167 and the write counters of
 * 445-446. */
typedef struct picard_io {
  int32_t write_fields, write_particles;
  double fields_interval, particles_interval;  /* seconds (reference: 100 dt, 1000 dt) */
  int32_t fields_iteration, particles_iteration; /* in/out: next file numbers          */
  char root[512];                              /* the reference's "save" directory    */
} picard_io;

/* picard.f90:554-674 with the write-step branch (602-627): on a step where
 * dmod(time, fields_interval) < dt or dmod(time, particles_interval) < dt,
 * AdvanceVelocityImp(dt/2), DumpParticles if due, ParticlesGridifyAll +
 * DumpFields if due, AdvanceVelocityExp(dt/2); AdvanceVelocity otherwise.
 * Arguments as picard_gpu_run. */
PICARD_API int picard_gpu_run_io(picard_ctx* ctx, int32_t iter_start, int32_t iter_end, int32_t log_interval,
                                 picard_log_fn log_fn, void* user, picard_io* io, int64_t* sweeps_total);

#ifdef __cplusplus
}
#endif

#endif /* PICARD_IO_H */
