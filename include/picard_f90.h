/*
 * picard_f90.h -- the reference's subroutine signatures over the device state.
 *
 * Every subroutine that `program picard` calls on its main path has one entry
 * point here whose argument list is the reference subroutine's, in the same
 * order and with the same meaning, every argument passed by reference as
 * Fortran passes it.  A Fortran host keeps its call lines as they are and
 * replaces the reference's .f90 sources with the interface module of this
 * header (each subroutine bound with bind(C, name="picard_f90_...")).
 *
 * Types: Fortran `integer` -> int32_t, `real*8` -> double, default-kind
 * `logical` -> picard_f90_logical (4 bytes; nonzero is .true., which covers
 * both the 1 of gfortran and the -1 of other compilers).  Arrays are the
 * reference's column-major arrays, passed as a pointer to their first
 * element.
 *
 * State.  The calls run on the device state of one context (picard_gpu.h),
 * registered once with picard_f90_attach.  The device copy of every array is
 * authoritative: the host arrays passed to the calls are neither read nor
 * written (they stay as the host left them) and are synchronised only when
 * the host asks: picard_f90_get_particles / picard_f90_get_fields copy the
 * device state into them in the reference layouts, picard_f90_set_particles
 * uploads host particles (a restart).  num_local, the one scalar the
 * reference returns, is written back by every routine that changes it.
 *
 * Scalar arguments are checked against the attached context: grid sizes,
 * species, max_per_proc, the flow flags, the rank grid (iprocs = jprocs =
 * kprocs = 1, myid = 0: one device-resident domain), num_local, and the
 * physical parameters (within 1e-12 relative).  Per-call values are taken
 * from the arguments: dt of AdvancePosition and AdvanceVelocity, deltat and
 * dt of AdvanceVelocityExp / AdvanceVelocityImp, maxerr and maxit of
 * CalcEpotential.
 *
 * Iteration.  BCinflow and ParticlesProduce draw from counter-based random
 * streams keyed by the iteration; the reference's signatures do not carry it.
 * The layer counts it: each BCinflow call starts the next iteration (the first
 * after attach is iteration 1), and ParticlesProduce uses the current one.
 * picard_f90_set_iteration sets the count for a run that starts at
 * iter_start > 0.
 *
 * Errors.  The reference's subroutines report nothing, so these are
 * subroutines too.  A failure is printed to stderr, recorded, and the call
 * returns; picard_f90_status() gives the first recorded status (and clears
 * it).  picard_f90_set_abort(1) makes a failure abort the process instead.
 * CalcEpotential that reaches 2*maxit+1 sweeps prints the reference's
 * "Maximum iteration reached!" and is not a failure (CalcEpotential.f90:67-69).
 */
#ifndef PICARD_F90_H
#define PICARD_F90_H

#include <stdint.h>

#include "picard_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t picard_f90_logical;

/* ------------------------------------------------------------ registration */

/* Binds the calls below to ctx (created with picard_gpu_create) and sets the
 * iteration count to 0.  Returns a picard_status. */
PICARD_API int picard_f90_attach(picard_ctx* ctx);
/* Unbinds the context (it stays alive; destroy it with picard_gpu_destroy). */
PICARD_API int picard_f90_detach(void);
/* The next BCinflow call runs iteration `iteration` + 1. */
PICARD_API int picard_f90_set_iteration(int32_t iteration);
/* First status recorded by the subroutine calls since the previous query
 * (PICARD_OK if none); the query clears it. */
PICARD_API int picard_f90_status(void);
/* Message of the status picard_f90_status() last returned ("" if none). */
PICARD_API const char* picard_f90_status_message(void);
/* on != 0: a failing call aborts the process after printing its message. */
PICARD_API int picard_f90_set_abort(int32_t on);
/* Directory that DumpParticles / DumpFields write under (the reference's
 * "save"; default "save"). */
PICARD_API int picard_f90_set_dump_root(const char* root);

/* ----------------------------------------------- host copies of the state */

/* real_particles(8, max_per_proc), int_particles(max_per_proc) and num_local
 * from the device (picard.f90:74-92 layouts).  PICARD_ERR_CAPACITY if the
 * device holds more than *max_per_proc particles. */
PICARD_API int picard_f90_get_particles(double* real_particles, int32_t* int_particles, const int32_t* max_per_proc,
                                        int32_t* num_local);
/* Uploads num_local host particles (a restart); the device count becomes
 * *num_local. */
PICARD_API int picard_f90_set_particles(const double* real_particles, const int32_t* int_particles,
                                        const int32_t* num_local);
/* U(Nx+2,Ny+2,Nz+2), E(3,...), N(species,...), C(...) from the device; any
 * of them may be NULL. */
PICARD_API int picard_f90_get_fields(double* U, double* E, double* N, double* C);
/* The sums of picard.f90:651-665 on the device (un-normalised uP, uE, uB)
 * and num_local, for the diagnostics block without a host copy. */
PICARD_API int picard_f90_energy(double* uP, double* uE, double* uB, int32_t* num_local);

/* ------------------------------- the reference's subroutines, same arguments */

/* CalcDistance.f90:1 */
PICARD_API void picard_f90_calc_distance(double* D, const int32_t* Nx, const int32_t* Ny, const int32_t* Nz,
                                         const double* dxyz, const picard_f90_logical* xflow,
                                         const picard_f90_logical* yflow, const picard_f90_logical* zflow);

/* ParticlesInitialize.f90:2-3 */
PICARD_API void picard_f90_particles_initialize(double* real_particles, int32_t* int_particles, const double* Lx_min,
                                                const double* Ly_min, const double* Lz_min, const double* dxyz,
                                                const double* kelvin, const double* mass, const double* v0,
                                                const double* ve, const double* tB, const int32_t* max_per_proc,
                                                int32_t* num_local, const int32_t* ppc, const int32_t* epp,
                                                const int32_t* hpp, const int32_t* ipp, const int32_t* species,
                                                const int32_t* Nx_local, const int32_t* Ny_local,
                                                const int32_t* Nz_local);

/* BCinflow.f90:2-4 */
PICARD_API void picard_f90_bc_inflow(double* real_particles, int32_t* int_particles, const double* Lx_min,
                                     const double* Ly_min, const double* Lz_min, const double* Lx_max,
                                     const double* Ly_max, const double* Lz_max, const double* dxyz,
                                     const double* kelvin, const double* mass, const double* v0, const double* ve,
                                     const int32_t* max_per_proc, int32_t* num_local, const int32_t* ppc,
                                     const int32_t* epp, const int32_t* hpp, const int32_t* ipp,
                                     const int32_t* species, const int32_t* Nx_local, const int32_t* Ny_local,
                                     const int32_t* Nz_local, const double* xmin, const double* xmax,
                                     const double* ymin, const double* ymax, const double* zmin, const double* zmax,
                                     const double* tB, const picard_f90_logical* xflow,
                                     const picard_f90_logical* yflow, const picard_f90_logical* zflow);

/* AdvancePosition.f90:4 */
PICARD_API void picard_f90_advance_position(double* real_particles, const double* dt, const int32_t* max_per_proc,
                                            const int32_t* num_local);

/* ParticlesProduce.f90:1-2 */
PICARD_API void picard_f90_particles_produce(double* real_particles, int32_t* int_particles, const double* Lx_min,
                                             const double* Ly_min, const double* Lz_min, const double* dxyz,
                                             const double* kelvin, const double* mass, const double* nu_d,
                                             const double* nu_i, const double* Ek, const double* Qn,
                                             const double* vn, const double* v0, const double* ve,
                                             const int32_t* max_per_proc, int32_t* num_local, const int32_t* ppc,
                                             const int32_t* epp, const int32_t* hpp, const int32_t* ipp,
                                             const int32_t* species, const int32_t* Nx_local,
                                             const int32_t* Ny_local, const int32_t* Nz_local, const double* dt,
                                             const double* n2p);

/* BCoutflow.f90:5-6 (removal in the reference's order) */
PICARD_API void picard_f90_bc_outflow(double* real_particles, int32_t* int_particles, const double* Lx_min,
                                      const double* Lx_max, const double* Ly_min, const double* Ly_max,
                                      const double* Lz_min, const double* Lz_max, const double* xmin,
                                      const double* xmax, const double* ymin, const double* ymax, const double* zmin,
                                      const double* zmax, const int32_t* max_per_proc, int32_t* num_local,
                                      const picard_f90_logical* xflow, const picard_f90_logical* yflow,
                                      const picard_f90_logical* zflow);

/* ParticlesTransfer.f90:2-3 (one domain: the periodic wrap) */
PICARD_API void picard_f90_particles_transfer(double* real_particles, int32_t* int_particles, const double* Lx_min,
                                              const double* Lx_max, const double* Ly_min, const double* Ly_max,
                                              const double* Lz_min, const double* Lz_max, const double* xmin,
                                              const double* xmax, const double* ymin, const double* ymax,
                                              const double* zmin, const double* zmax, const int32_t* max_per_proc,
                                              int32_t* num_local, const int32_t* iprocs, const int32_t* jprocs,
                                              const int32_t* kprocs, const int32_t* myid);

/* ParticlesGridify.f90:1-3 */
PICARD_API void picard_f90_particles_gridify(double* N, double* C, const double* real_particles,
                                             const int32_t* int_particles, const double* Lx_min, const double* Lx_max,
                                             const double* Ly_min, const double* Ly_max, const double* Lz_min,
                                             const double* Lz_max, const double* dxyz, const double* xmin,
                                             const double* xmax, const double* ymin, const double* ymax,
                                             const double* zmin, const double* zmax, const int32_t* species,
                                             const int32_t* Nx_local, const int32_t* Ny_local,
                                             const int32_t* Nz_local, const int32_t* max_per_proc,
                                             const int32_t* num_local, const picard_f90_logical* xflow,
                                             const picard_f90_logical* yflow, const picard_f90_logical* zflow,
                                             const int32_t* iprocs, const int32_t* jprocs, const int32_t* kprocs,
                                             const double* charge, const double* n2p, const int32_t* myid);

/* ParticlesGridifyAll.f90:1-3 */
PICARD_API void picard_f90_particles_gridify_all(double* F, double* N, double* C, const double* real_particles,
                                                 const int32_t* int_particles, const double* Lx_min,
                                                 const double* Lx_max, const double* Ly_min, const double* Ly_max,
                                                 const double* Lz_min, const double* Lz_max, const double* dxyz,
                                                 const double* xmin, const double* xmax, const double* ymin,
                                                 const double* ymax, const double* zmin, const double* zmax,
                                                 const int32_t* species, const int32_t* Nx_local,
                                                 const int32_t* Ny_local, const int32_t* Nz_local,
                                                 const int32_t* max_per_proc, const int32_t* num_local,
                                                 const picard_f90_logical* xflow, const picard_f90_logical* yflow,
                                                 const picard_f90_logical* zflow, const int32_t* iprocs,
                                                 const int32_t* jprocs, const int32_t* kprocs, const double* charge,
                                                 const double* n2p, const int32_t* myid);

/* BCpotentials.f90:1-2 */
PICARD_API void picard_f90_bc_potentials(double* U, const double* C, const double* D, const double* xmin,
                                         const double* xmax, const double* ymin, const double* ymax,
                                         const double* zmin, const double* zmax, const int32_t* Nx_local,
                                         const int32_t* Ny_local, const int32_t* Nz_local, const int32_t* Nx,
                                         const int32_t* Ny, const int32_t* Nz, const picard_f90_logical* xflow,
                                         const picard_f90_logical* yflow, const picard_f90_logical* zflow,
                                         const int32_t* species, const int32_t* iprocs, const int32_t* jprocs,
                                         const int32_t* kprocs, const int32_t* myid);

/* CalcEpotential.f90:4-5 */
PICARD_API void picard_f90_calc_epotential(double* U, const double* C, const int32_t* Nx_local,
                                           const int32_t* Ny_local, const int32_t* Nz_local, const double* Lx_min,
                                           const double* Lx_max, const double* Ly_min, const double* Ly_max,
                                           const double* Lz_min, const double* Lz_max,
                                           const picard_f90_logical* xflow, const picard_f90_logical* yflow,
                                           const picard_f90_logical* zflow, const double* xmin, const double* xmax,
                                           const double* ymin, const double* ymax, const double* zmin,
                                           const double* zmax, const double* dxyz, const double* maxerr,
                                           const int32_t* maxit, const int32_t* iprocs, const int32_t* jprocs,
                                           const int32_t* kprocs, const int32_t* species, const int32_t* myid);

/* CalcEfield.f90:3 */
PICARD_API void picard_f90_calc_efield(double* E, const double* U, const int32_t* Nx_local, const int32_t* Ny_local,
                                       const int32_t* Nz_local, const double* dxyz, const picard_f90_logical* xflow,
                                       const picard_f90_logical* yflow, const picard_f90_logical* zflow,
                                       const int32_t* iprocs, const int32_t* jprocs, const int32_t* kprocs,
                                       const int32_t* myid);

/* BCfields.f90:3 */
PICARD_API void picard_f90_bc_fields(double* E, const double* U, const double* B0, const double* E0,
                                     const int32_t* Nx_local, const int32_t* Ny_local, const int32_t* Nz_local,
                                     const picard_f90_logical* xflow, const picard_f90_logical* yflow,
                                     const picard_f90_logical* zflow, const int32_t* iprocs, const int32_t* jprocs,
                                     const int32_t* kprocs, const int32_t* myid);

/* AdvanceVelocity.f90:6-7 */
PICARD_API void picard_f90_advance_velocity(double* real_particles, const int32_t* int_particles, const double* E,
                                            const double* B0, const double* Lx_min, const double* Ly_min,
                                            const double* Lz_min, const double* dxyz, const double* dt,
                                            const double* v0, const double* ve, const double* eta, const double* tB,
                                            const double* sB, const int32_t* num_local, const int32_t* max_per_proc,
                                            const int32_t* species, const int32_t* Nx_local,
                                            const int32_t* Ny_local, const int32_t* Nz_local,
                                            const picard_f90_logical* fluid, const picard_f90_logical* gyration);

/* AdvanceVelocity.f90:128-129 */
PICARD_API void picard_f90_advance_velocity_exp(double* real_particles, const int32_t* int_particles,
                                                const double* E, const double* B0, const double* Lx_min,
                                                const double* Ly_min, const double* Lz_min, const double* dxyz,
                                                const double* deltat, const double* dt, const double* v0,
                                                const double* ve, const double* eta, const double* tB,
                                                const int32_t* num_local, const int32_t* max_per_proc,
                                                const int32_t* species, const int32_t* Nx_local,
                                                const int32_t* Ny_local, const int32_t* Nz_local,
                                                const picard_f90_logical* fluid, const picard_f90_logical* gyration);

/* AdvanceVelocity.f90:239-240 */
PICARD_API void picard_f90_advance_velocity_imp(double* real_particles, const int32_t* int_particles,
                                                const double* E, const double* B0, const double* Lx_min,
                                                const double* Ly_min, const double* Lz_min, const double* dxyz,
                                                const double* deltat, const double* dt, const double* v0,
                                                const double* ve, const double* eta, const double* tB,
                                                const int32_t* num_local, const int32_t* max_per_proc,
                                                const int32_t* species, const int32_t* Nx_local,
                                                const int32_t* Ny_local, const int32_t* Nz_local,
                                                const picard_f90_logical* fluid, const picard_f90_logical* gyration);

/* Write.f90:2 (the dump of the device particles under the dump root) */
PICARD_API void picard_f90_dump_particles(double* real_particles, const int32_t* int_particles,
                                          const int32_t* num_local, const int32_t* max_per_proc,
                                          int32_t* writeParticles_iteration, const int32_t* myid);

/* Write.f90:34 (the dump of the device fields under the dump root) */
PICARD_API void picard_f90_dump_fields(const double* U, const double* N, const double* F, const double* E,
                                       const int32_t* Nx_local, const int32_t* Ny_local, const int32_t* Nz_local,
                                       int32_t* writeFields_iteration, const int32_t* species, const int32_t* myid);

#ifdef __cplusplus
}
#endif

#endif /* PICARD_F90_H */
