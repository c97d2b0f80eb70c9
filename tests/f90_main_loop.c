/*
 * The main loop of program picard (picard.f90:505-509 and 554-631, write
 * step off) driven through include/picard_f90.h: every call line keeps the
 * reference's argument list, with the main program's own variable names.
 * A test program, built and run by tests/test_gpu_f90.py.
 *
 * usage: f90_main_loop PARAMS_FILE ITER_END OUT_FILE
 *   PARAMS_FILE  one picard_params block (inputs set; derived here)
 *   OUT_FILE     num_local, real_particles(8, num_local),
 *                int_particles(num_local), U, E, N, C, then the status
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "picard_f90.h"
#include "picard_gpu.h"

static int die(const char* what) {
  fprintf(stderr, "f90_main_loop: %s: %s\n", what, picard_gpu_last_error());
  return 1;
}

int main(int argc, char** argv) {
  if (argc != 4) {
    fprintf(stderr, "usage: %s PARAMS_FILE ITER_END OUT_FILE\n", argv[0]);
    return 2;
  }
  picard_params prm;
  FILE* f = fopen(argv[1], "rb");
  if (!f || fread(&prm, sizeof prm, 1, f) != 1) return 2;
  fclose(f);
  const int iter_end = atoi(argv[2]);
  if (picard_params_derive(&prm) != PICARD_OK) return die("picard_params_derive");

  /* the main program's variables (picard.f90:41-302, 333-467), one rank */
  int32_t Nx_local = prm.nx, Ny_local = prm.ny, Nz_local = prm.nz;
  int32_t Nx = Nx_local, Ny = Ny_local, Nz = Nz_local;
  int32_t iprocs = 1, jprocs = 1, kprocs = 1, myid = 0;
  int32_t species = prm.species, max_per_proc = prm.max_per_proc, maxit = prm.maxit;
  picard_f90_logical xflow = prm.xflow != 0, yflow = prm.yflow != 0, zflow = prm.zflow != 0;
  picard_f90_logical fluid[8], gyration[8];
  for (int s = 0; s < 8; ++s) {
    fluid[s] = prm.fluid[s] != 0;
    gyration[s] = prm.gyration[s] != 0;
  }
  double xmin = prm.xmin, xmax = prm.xmax, ymin = prm.ymin, ymax = prm.ymax, zmin = prm.zmin, zmax = prm.zmax;
  double Lx_min = prm.Lx_min, Lx_max = prm.Lx_max, Ly_min = prm.Ly_min, Ly_max = prm.Ly_max;
  double Lz_min = prm.Lz_min, Lz_max = prm.Lz_max;
  double dt = prm.dt, maxerr = prm.maxerr;
  double* dxyz = prm.dxyz;
  double *kelvin = prm.kelvin, *mass = prm.mass, *charge = prm.charge, *n2p = prm.n2p, *eta = prm.eta;
  double *nu_d = prm.nu_d, *nu_i = prm.nu_i, *Ek = prm.Ek, *Qn = prm.Qn, *vn = prm.vn;
  double *v0 = &prm.v0[0][0], *ve = prm.ve, *tB = &prm.tB[0][0], *sB = &prm.sB[0][0];
  double *B0 = prm.B0, *E0 = prm.E0;
  int32_t *ppc = prm.ppc, *epp = prm.epp, *hpp = prm.hpp, *ipp = prm.ipp;

  /* the state arrays (picard.f90:74-113) */
  const size_t nodes = (size_t)(Nx_local + 2) * (Ny_local + 2) * (Nz_local + 2);
  double* real_particles = calloc((size_t)8 * max_per_proc, sizeof(double));
  int32_t* int_particles = calloc((size_t)max_per_proc, sizeof(int32_t));
  double* U = calloc(nodes, sizeof(double));
  double* E = calloc(3 * nodes, sizeof(double));
  double* N = calloc((size_t)species * nodes, sizeof(double));
  double* C = calloc(nodes, sizeof(double));
  double* D = calloc((size_t)(2 * Nx + 1) * (2 * Ny + 1) * (2 * Nz + 1), sizeof(double));
  if (!real_particles || !int_particles || !U || !E || !N || !C || !D) return 2;
  int32_t num_local = 0;

  picard_ctx* ctx = NULL;
  if (picard_gpu_create(&prm, PICARD_LAYOUT_F64, PICARD_SOLVER_F64, &ctx) != PICARD_OK) return die("create");
  if (picard_f90_attach(ctx) != PICARD_OK) return die("attach");

  picard_f90_calc_distance(D, &Nx, &Ny, &Nz, dxyz, &xflow, &yflow, &zflow);
  picard_f90_particles_initialize(real_particles, int_particles, &Lx_min, &Ly_min, &Lz_min, dxyz, kelvin, mass, v0,
                                  ve, tB, &max_per_proc, &num_local, ppc, epp, hpp, ipp, &species, &Nx_local,
                                  &Ny_local, &Nz_local);

  for (int iteration = 1; iteration <= iter_end; ++iteration) {
    picard_f90_bc_inflow(real_particles, int_particles, &Lx_min, &Ly_min, &Lz_min, &Lx_max, &Ly_max, &Lz_max, dxyz,
                         kelvin, mass, v0, ve, &max_per_proc, &num_local, ppc, epp, hpp, ipp, &species, &Nx_local,
                         &Ny_local, &Nz_local, &xmin, &xmax, &ymin, &ymax, &zmin, &zmax, tB, &xflow, &yflow, &zflow);
    picard_f90_advance_position(real_particles, &dt, &max_per_proc, &num_local);
    picard_f90_particles_produce(real_particles, int_particles, &Lx_min, &Ly_min, &Lz_min, dxyz, kelvin, mass, nu_d,
                                 nu_i, Ek, Qn, vn, v0, ve, &max_per_proc, &num_local, ppc, epp, hpp, ipp, &species,
                                 &Nx_local, &Ny_local, &Nz_local, &dt, n2p);
    picard_f90_bc_outflow(real_particles, int_particles, &Lx_min, &Lx_max, &Ly_min, &Ly_max, &Lz_min, &Lz_max, &xmin,
                          &xmax, &ymin, &ymax, &zmin, &zmax, &max_per_proc, &num_local, &xflow, &yflow, &zflow);
    picard_f90_particles_transfer(real_particles, int_particles, &Lx_min, &Lx_max, &Ly_min, &Ly_max, &Lz_min,
                                  &Lz_max, &xmin, &xmax, &ymin, &ymax, &zmin, &zmax, &max_per_proc, &num_local,
                                  &iprocs, &jprocs, &kprocs, &myid);
    picard_f90_particles_gridify(N, C, real_particles, int_particles, &Lx_min, &Lx_max, &Ly_min, &Ly_max, &Lz_min,
                                 &Lz_max, dxyz, &xmin, &xmax, &ymin, &ymax, &zmin, &zmax, &species, &Nx_local,
                                 &Ny_local, &Nz_local, &max_per_proc, &num_local, &xflow, &yflow, &zflow, &iprocs,
                                 &jprocs, &kprocs, charge, n2p, &myid);
    picard_f90_bc_potentials(U, C, D, &xmin, &xmax, &ymin, &ymax, &zmin, &zmax, &Nx_local, &Ny_local, &Nz_local, &Nx,
                             &Ny, &Nz, &xflow, &yflow, &zflow, &species, &iprocs, &jprocs, &kprocs, &myid);
    picard_f90_calc_epotential(U, C, &Nx_local, &Ny_local, &Nz_local, &Lx_min, &Lx_max, &Ly_min, &Ly_max, &Lz_min,
                               &Lz_max, &xflow, &yflow, &zflow, &xmin, &xmax, &ymin, &ymax, &zmin, &zmax, dxyz,
                               &maxerr, &maxit, &iprocs, &jprocs, &kprocs, &species, &myid);
    picard_f90_calc_efield(E, U, &Nx_local, &Ny_local, &Nz_local, dxyz, &xflow, &yflow, &zflow, &iprocs, &jprocs,
                           &kprocs, &myid);
    picard_f90_bc_fields(E, U, B0, E0, &Nx_local, &Ny_local, &Nz_local, &xflow, &yflow, &zflow, &iprocs, &jprocs,
                         &kprocs, &myid);
    picard_f90_advance_velocity(real_particles, int_particles, E, B0, &Lx_min, &Ly_min, &Lz_min, dxyz, &dt, v0, ve,
                                eta, tB, sB, &num_local, &max_per_proc, &species, &Nx_local, &Ny_local, &Nz_local,
                                fluid, gyration);
  }
  const int status = picard_f90_status();

  /* the host copies, synchronised once at the end */
  if (picard_f90_get_particles(real_particles, int_particles, &max_per_proc, &num_local) != PICARD_OK)
    return die("get_particles");
  if (picard_f90_get_fields(U, E, N, C) != PICARD_OK) return die("get_fields");
  FILE* o = fopen(argv[3], "wb");
  if (!o) return 2;
  fwrite(&num_local, sizeof num_local, 1, o);
  fwrite(real_particles, sizeof(double), (size_t)8 * num_local, o);
  fwrite(int_particles, sizeof(int32_t), (size_t)num_local, o);
  fwrite(U, sizeof(double), nodes, o);
  fwrite(E, sizeof(double), 3 * nodes, o);
  fwrite(N, sizeof(double), (size_t)species * nodes, o);
  fwrite(C, sizeof(double), nodes, o);
  fwrite(&status, sizeof status, 1, o);
  fclose(o);
  picard_f90_detach();
  picard_gpu_destroy(ctx);
  printf("f90_main_loop: %d iterations, num_local %d, status %d\n", iter_end, num_local, status);
  return status == PICARD_OK ? 0 : 3;
}
