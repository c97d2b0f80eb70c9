/*
 * picard_oracle.c -- CPU FP64 restatement of Picard's per-timestep PIC loop.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the oracle the CUDA path is compared
 * against, and the CPU baseline that bench.py times.  Nothing in the product
 * (picard_b200/) links, loads or calls it.
 *
 * PARITY UNPINNED.  The reference is Fortran 90 + MPI and no Fortran compiler
 * or MPI exists on these machines, and the reference ships no tests, fixtures
 * or golden vectors.  This restatement is pinned instead by physics
 * known-answer tests (tests/test_oracle_kat.py) and by the published
 * Philox4x32-10 test vectors.
 *
 * Conventions kept from the reference (each routine cites the lines it follows):
 *  - arrays are column-major with a 1-cell ghost layer; the macros below take
 *    the reference's 1-based indices;
 *  - idint = truncation toward zero ((int) cast), dmod = fmod;
 *  - operations are evaluated in the reference's left-to-right order and the
 *    file is compiled with -ffp-contract=off (no fused multiply-add), so the
 *    FP64 results are the IEEE results of the reference's expressions;
 *  - particle loops run from the last particle to the first like the
 *    reference's `do pp = num_local, 1, -1`.
 *
 * Stochastic steps.  The reference draws from the compiler's random_number
 * with an uninitialised seed (picard.f90:136-138), so its streams cannot be
 * reproduced.  Here every draw comes from Philox4x32-10 (Salmon, Moraes, Dror,
 * Shaw, "Parallel random numbers: as easy as 1, 2, 3", SC'11), keyed by the
 * run seed, with one counter per draw site:
 *     counter = (a, b, iteration, tag << 24 | block)
 *     a   = 0-based index of the cell in the padded (Nx+2)(Ny+2)(Nz+2) box
 *     b   = (species << 24) | (pp << 8) | member   (init, inflow; member 0 is
 *           the ion, 1..epp its electrons, epp+1.. its protons)
 *           species                                 (produce: count draw)
 *           (species << 24) | pp                    (produce: particle draw)
 *     tag = 1 init, 2 inflow, 3 produce count, 4 produce particle
 * Uniform n of a site uses block n/2, words 2(n%2), 2(n%2)+1 -> 53-bit double
 * in [0,1).  The CUDA path implements the same specification, so both sides
 * generate the same particles.
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "picard_gpu.h"

/* physical constants, picard.f90:56-66 */
#define TAU 6.2831853071795864769252867665590
#define EC 1.60217646e-19
#define MP 1.6726216e-27
#define ME 9.1093819e-31
#define EPS0 8.854187817e-12
#define KB 1.380650e-23
#define MU0 1.25663706143591729538505735331180e-6

#define EXPORT __attribute__((visibility("default")))

/* ------------------------------------------------------------------ Philox */

static inline void mulhilo32(uint32_t a, uint32_t b, uint32_t* hi, uint32_t* lo) {
  uint64_t p = (uint64_t)a * (uint64_t)b;
  *hi = (uint32_t)(p >> 32);
  *lo = (uint32_t)p;
}

/* Philox4x32 with 10 rounds, SC'11 paper section 2.2 / Random123. */
EXPORT void orc_philox4x32_10(const uint32_t ctr_in[4], const uint32_t key_in[2], uint32_t out[4]) {
  uint32_t c0 = ctr_in[0], c1 = ctr_in[1], c2 = ctr_in[2], c3 = ctr_in[3];
  uint32_t k0 = key_in[0], k1 = key_in[1];
  for (int r = 0; r < 10; ++r) {
    uint32_t hi0, lo0, hi1, lo1;
    mulhilo32(0xD2511F53u, c0, &hi0, &lo0);
    mulhilo32(0xCD9E8D57u, c2, &hi1, &lo1);
    uint32_t n0 = hi1 ^ c1 ^ k0;
    uint32_t n2 = hi0 ^ c3 ^ k1;
    c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

typedef struct {
  uint32_t ctr[4];
  uint32_t key[2];
  uint32_t cached_blk;
  uint32_t words[4];
} site_rng;

static void site_init(site_rng* s, uint64_t seed, uint32_t a, uint32_t b, uint32_t it, uint32_t tag) {
  s->key[0] = (uint32_t)seed;
  s->key[1] = (uint32_t)(seed >> 32);
  s->ctr[0] = a;
  s->ctr[1] = b;
  s->ctr[2] = it;
  s->ctr[3] = tag << 24;
  s->cached_blk = 0xFFFFFFFFu;
}

/* uniform n of the site, in [0, 1) */
static double site_u(site_rng* s, uint32_t n) {
  uint32_t blk = n >> 1;
  if (blk != s->cached_blk) {
    uint32_t c[4] = {s->ctr[0], s->ctr[1], s->ctr[2], s->ctr[3] | blk};
    orc_philox4x32_10(c, s->key, s->words);
    s->cached_blk = blk;
  }
  uint32_t w0 = s->words[2 * (n & 1)], w1 = s->words[2 * (n & 1) + 1];
  return ((double)(w0 >> 5) * 67108864.0 + (double)(w1 >> 6)) * (1.0 / 9007199254740992.0);
}

EXPORT double orc_site_uniform(uint64_t seed, uint32_t a, uint32_t b, uint32_t it, uint32_t tag, uint32_t n) {
  site_rng s;
  site_init(&s, seed, a, b, it, tag);
  return site_u(&s, n);
}

/* Tools.f90:30-48 normal(): Box-Muller, r1 for the angle, r2 > 0 for the
 * radius.  r2 = 1 - u lies in (0, 1], so the reference's retry never fires. */
static double normal_from(site_rng* s, uint32_t n) {
  double r1 = site_u(s, n);
  double r2 = 1.0 - site_u(s, n + 1);
  return sqrt(-2.0 * log(r2)) * sin(TAU * r1);
}

/* Tools.f90:2-28 Gaussian(): drifting Maxwellian, uniforms n .. n+5 */
static void gaussian_from(site_rng* s, uint32_t n, double u[3], const double v[3], double t, double m) {
  if (t > 0.0 && m > 0.0) {
    double a = m / (2.0 * KB * t);
    double pw = sqrt(1.0 / a);
    for (int c = 0; c < 3; ++c) u[c] = normal_from(s, n + 2 * c);
    for (int c = 0; c < 3; ++c) u[c] = u[c] * pw / sqrt(2.0);
    for (int c = 0; c < 3; ++c) u[c] = u[c] + v[c];
  } else {
    for (int c = 0; c < 3; ++c) u[c] = v[c];
  }
}

/* The -dt/2 rotation with |v - ve| restored, as written out in
 * ParticlesInitialize.f90:73-80 and BCinflow.f90:74-81. */
static void half_rotate(double v[3], const double ve[4], const double tB[4]) {
  double vmin[3], vmid[3];
  for (int c = 0; c < 3; ++c) vmin[c] = v[c] - ve[c];
  vmid[0] = vmin[0] + vmin[1] * tB[2] - vmin[2] * tB[1];
  vmid[1] = vmin[1] + vmin[2] * tB[0] - vmin[0] * tB[2];
  vmid[2] = vmin[2] + vmin[0] * tB[1] - vmin[1] * tB[0];
  double smid = vmid[0] * vmid[0] + vmid[1] * vmid[1] + vmid[2] * vmid[2];
  if (smid > 0.0) {
    double smin = vmin[0] * vmin[0] + vmin[1] * vmin[1] + vmin[2] * vmin[2];
    double f = sqrt(smin / smid);
    for (int c = 0; c < 3; ++c) vmid[c] = vmid[c] * f;
  }
  for (int c = 0; c < 3; ++c) v[c] = vmid[c] + ve[c];
}

/* ------------------------------------------------------------ indexing */

#define NXP (p->nx + 2)
#define NYP (p->ny + 2)
#define NZP (p->nz + 2)
/* 1-based (i, j, k) node of a (Nx+2, Ny+2, Nz+2) array */
#define G3(i, j, k) ((size_t)((i)-1) + (size_t)NXP * ((size_t)((j)-1) + (size_t)NYP * (size_t)((k)-1)))
#define RP(q, pp) rp[(size_t)8 * (size_t)((pp)-1) + (size_t)((q)-1)]
#define IP(pp) ip[(pp)-1]

EXPORT void orc_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

EXPORT int orc_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

/* ------------------------------------------------ parameters (a2) */

/* picard.f90:333-467 on one rank (myid = 0, iprocs = jprocs = kprocs = 1). */
EXPORT void orc_derive_params(picard_params* p) {
  double Lx = p->xmax - p->xmin, Ly = p->ymax - p->ymin, Lz = p->zmax - p->zmin;
  double Lx_local = Lx / 1.0, Ly_local = Ly / 1.0, Lz_local = Lz / 1.0;
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

  p->vn[0] = 0.0; p->Qn[0] = 0.0; p->Ek[0] = 0.0; p->nu_i[0] = 0.0; p->nu_d[0] = 0.0;
  p->charge[0] = -EC;
  p->charge[1] = EC;
  for (int s = 1; s < 8; ++s) {
    int mx = p->ppc[s] > 1 ? p->ppc[s] : 1;
    p->density[s] = p->density[s] * (double)p->ppc[s] / (double)mx;
  }
  double acc = 0.0;
  for (int s = 1; s < 8; ++s) acc += -p->density[s] * p->charge[s];
  p->density[0] = acc * (1.0 / p->charge[0]);
  for (int s = 0; s < 8; ++s) {
    if (p->density[s] <= 0.0 || p->species < s + 1) {
      p->ppc[s] = 0;
      p->density[s] = 0.0;
    }
  }
  acc = 0.0;
  for (int s = 1; s < 8; ++s) acc += -p->density[s] * p->charge[s] / p->charge[0];
  p->density[0] = acc;

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

  for (int s = 0; s < 8; ++s) p->n2p[s] = 0.0;
  for (int s = 0; s < 8; ++s) {
    if (p->ppc[s] > 0)
      p->n2p[s] = p->dV * p->density[s] * (1.0 / (double)p->ppc[s]);
    else
      p->n2p[s] = p->n2p[0];
  }
  for (int s = 0; s < 8; ++s) p->eta[s] = p->charge[s] / p->mass[s];

  for (int c = 0; c < 3; ++c) {
    double num = 0.0, den = 0.0;
    for (int s = 0; s < 8; ++s) {
      double w = (double)p->ipp[s] *
                 (p->n2p[s] * p->mass[s] + (double)p->epp[s] * p->n2p[0] * p->mass[0] +
                  (double)p->hpp[s] * p->n2p[1] * p->mass[1]);
      num += w * p->v0[s][c];
      den += w;
    }
    p->ve[c] = num / den;
  }
  for (int s = 0; s < 8; ++s)
    p->v0[s][3] = sqrt(p->v0[s][0] * p->v0[s][0] + p->v0[s][1] * p->v0[s][1] + p->v0[s][2] * p->v0[s][2]);
  p->ve[3] = sqrt(p->ve[0] * p->ve[0] + p->ve[1] * p->ve[1] + p->ve[2] * p->ve[2]);
  p->B0[3] = sqrt(p->B0[0] * p->B0[0] + p->B0[1] * p->B0[1] + p->B0[2] * p->B0[2]);
  p->E0[0] = p->ve[2] * p->B0[1] - p->ve[1] * p->B0[2];
  p->E0[1] = p->ve[0] * p->B0[2] - p->ve[2] * p->B0[0];
  p->E0[2] = p->ve[1] * p->B0[0] - p->ve[0] * p->B0[1];
  p->E0[3] = sqrt(p->E0[0] * p->E0[0] + p->E0[1] * p->E0[1] + p->E0[2] * p->E0[2]);

  for (int s = 0; s < 8; ++s) {
    for (int c = 0; c < 4; ++c) p->tB[s][c] = p->gyration[s] ? 0.5 * p->dt * p->B0[c] * p->eta[s] : 0.0;
  }
  for (int s = 0; s < 8; ++s) {
    double d = 1.0 + p->tB[s][3] * p->tB[s][3];
    for (int c = 0; c < 4; ++c) p->sB[s][c] = 2.0 * p->tB[s][c] / d;
  }
  double vol = Lx * Ly * Lz;
  double uE0 = 0.5 * (p->E0[3] * p->E0[3] * EPS0) * vol;
  double uB0 = 0.5 * (p->B0[3] * p->B0[3] / MU0) * vol;
  double up = 0.0;
  for (int s = 0; s < 8; ++s)
    up += p->density[s] * (p->mass[s] * p->v0[s][3] * p->v0[s][3] + 3.0 * KB * p->kelvin[s]);
  double uP0 = 0.5 * up * vol;
  p->u0 = uE0 + uB0 + uP0;
}

/* ----------------------------------------------- CalcDistance (a8) */

/* CalcDistance.f90:28-87 */
EXPORT void orc_calc_distance(const picard_params* p, double* D) {
  const int Nx = p->nx, Ny = p->ny, Nz = p->nz;
  const int DX = 2 * Nx + 1, DY = 2 * Ny + 1;
  const double* dxyz = p->dxyz;
  const int xf = p->xflow != 0, yf = p->yflow != 0, zf = p->zflow != 0;
#define DD(i, j, k) D[(size_t)((i)-1) + (size_t)DX * ((size_t)((j)-1) + (size_t)DY * (size_t)((k)-1))]
  memset(D, 0, sizeof(double) * (size_t)DX * DY * (2 * Nz + 1));
#pragma omp parallel for schedule(static)
  for (int kk = 1; kk <= Nz + 1; ++kk)
    for (int jj = 1; jj <= Ny + 1; ++jj)
      for (int ii = 1; ii <= Nx + 1; ++ii) {
        int pi = Nx + 1 + (ii - 1), pj = Ny + 1 + (jj - 1), pk = Nz + 1 + (kk - 1);
        int ni = Nx + 1 - (ii - 1), nj = Ny + 1 - (jj - 1), nk = Nz + 1 - (kk - 1);
        double di = (double)(ii - 1), dj = (double)(jj - 1), dk = (double)(kk - 1);
        double a = di * dxyz[0], b = dj * dxyz[1], c = dk * dxyz[2];
        double an = (Nx - di) * dxyz[0], bn = (Ny - dj) * dxyz[1], cn = (Nz - dk) * dxyz[2];
#define INV(x, y, z) (1.0 / sqrt((x) * (x) + (y) * (y) + (z) * (z)))
        double t;
        if (ii == 1 && jj == 1 && kk == 1)
          t = 0.0;
        else
          t = INV(a, b, c);
        if (xf) {
          if (!yf && !zf) {
            t = t + INV(a, bn, c);
            t = t + INV(a, b, cn);
            t = t + INV(a, bn, cn);
          } else if (!yf) {
            t = t + INV(a, bn, c);
          } else if (!zf) {
            t = t + INV(a, b, cn);
          }
        } else if (yf) {
          if (!zf) {
            t = t + INV(an, b, c);
            t = t + INV(a, b, cn);
            t = t + INV(an, b, cn);
          } else {
            t = t + INV(an, b, c);
          }
        } else if (zf) {
          t = t + INV(an, b, c);
          t = t + INV(a, bn, c);
          t = t + INV(an, bn, c);
        } else {
          t = t + INV(an, b, c);
          t = t + INV(a, bn, c);
          t = t + INV(a, b, cn);
          t = t + INV(an, bn, c);
          t = t + INV(a, bn, cn);
          t = t + INV(an, b, cn);
          t = t + INV(an, bn, cn);
        }
#undef INV
        DD(pi, pj, pk) = t; DD(ni, pj, pk) = t; DD(pi, nj, pk) = t; DD(pi, pj, nk) = t;
        DD(ni, nj, pk) = t; DD(pi, nj, nk) = t; DD(ni, pj, nk) = t; DD(ni, nj, nk) = t;
      }
#undef DD
}

/* ---------------------------------------- ParticlesInitialize (a17) */

static int append_guard(int num_local, int add, int max_per_proc) {
  if (num_local + add > max_per_proc) {
    fprintf(stderr, "oracle: particle capacity %d exceeded\n", max_per_proc);
    return 0;
  }
  return 1;
}

/* Creates the ion of a site plus its epp electrons and hpp protons, each with
 * its own velocity, as in ParticlesInitialize.f90:65-113 and
 * BCinflow.f90:66-114.  Returns the number of particles written. */
static int create_group(const picard_params* p, uint64_t seed, uint32_t tag, uint32_t it, uint32_t cell_a,
                        int ss /*1-based*/, int pp /*1-based*/, double x0, double y0, double z0, double* rp,
                        int32_t* ip, int base /*0-based slot of the ion*/) {
  const double* dxyz = p->dxyz;
  int s0 = ss - 1;
  site_rng r;
  site_init(&r, seed, cell_a, ((uint32_t)ss << 24) | ((uint32_t)pp << 8), it, tag);
  double* ion = rp + (size_t)8 * base;
  ip[base] = ss;
  ion[0] = x0 + dxyz[0] * site_u(&r, 0);
  ion[1] = y0 + dxyz[1] * site_u(&r, 1);
  ion[2] = z0 + dxyz[2] * site_u(&r, 2);
  ion[6] = 0.0; ion[7] = 0.0;
  gaussian_from(&r, 3, ion + 3, p->v0[s0], p->kelvin[s0], p->mass[s0]);
  half_rotate(ion + 3, p->ve, p->tB[s0]);
  int n = 1;
  for (int ee = 1; ee <= p->epp[s0]; ++ee, ++n) {
    double* q = rp + (size_t)8 * (base + n);
    memcpy(q, ion, sizeof(double) * 8);
    ip[base + n] = 1;
    site_rng re;
    site_init(&re, seed, cell_a, ((uint32_t)ss << 24) | ((uint32_t)pp << 8) | (uint32_t)ee, it, tag);
    gaussian_from(&re, 0, q + 3, p->v0[s0], p->kelvin[0], p->mass[0]);
    half_rotate(q + 3, p->ve, p->tB[0]);
  }
  for (int ee = 1; ee <= p->hpp[s0]; ++ee, ++n) {
    double* q = rp + (size_t)8 * (base + n);
    memcpy(q, ion, sizeof(double) * 8);
    ip[base + n] = 2;
    site_rng re;
    site_init(&re, seed, cell_a, ((uint32_t)ss << 24) | ((uint32_t)pp << 8) | (uint32_t)(p->epp[s0] + ee), it,
              tag);
    gaussian_from(&re, 0, q + 3, p->v0[s0], p->kelvin[1], p->mass[1]);
    half_rotate(q + 3, p->ve, p->tB[1]);
  }
  return n;
}

/* particles created per cell by one ParticlesInitialize / BCinflow cell loop */
static int per_cell_count(const picard_params* p) {
  int c = 0;
  for (int s = 0; s < p->species; ++s) c += p->ipp[s] * (1 + p->epp[s] + p->hpp[s]);
  return c;
}

/* ParticlesInitialize.f90:54-119.  Every cell creates the same number of
 * particles, so cell (ii, jj, kk) owns a fixed block of slots in the
 * reference's append order and the cells can be filled in parallel. */
EXPORT int orc_particles_initialize(const picard_params* p, double* rp, int32_t* ip, int32_t* num_local) {
  const double* dxyz = p->dxyz;
  const int n0 = *num_local;
  const long long per_cell = per_cell_count(p);
  const long long cells = (long long)p->nx * p->ny * p->nz;
  if (!append_guard(n0, (int)(cells * per_cell), p->max_per_proc) || n0 + cells * per_cell > 2147483647LL) return 2;
#pragma omp parallel for collapse(2) schedule(static)
  for (int kk = 2; kk <= p->nz + 1; ++kk)
    for (int jj = 2; jj <= p->ny + 1; ++jj)
      for (int ii = 2; ii <= p->nx + 1; ++ii) {
        double x0 = p->Lx_min + dxyz[0] * (ii - 2);
        double y0 = p->Ly_min + dxyz[1] * (jj - 2);
        double z0 = p->Lz_min + dxyz[2] * (kk - 2);
        uint32_t a = (uint32_t)G3(ii, jj, kk);
        long long cell = (ii - 2) + (long long)p->nx * ((jj - 2) + (long long)p->ny * (kk - 2));
        int n = (int)(n0 + cell * per_cell);
        for (int ss = 1; ss <= p->species; ++ss)
          for (int pp = 1; pp <= p->ipp[ss - 1]; ++pp) n += create_group(p, p->seed, 1, 0, a, ss, pp, x0, y0, z0, rp, ip, n);
      }
  *num_local = (int)(n0 + cells * per_cell);
  return 0;
}

/* ---------------------------------------------------- BCinflow (a3) */

/* One face of BCinflow: `outer` x `inner` loop over guard cells in the
 * reference's order.  Every guard cell creates the same number of particles,
 * so each owns a fixed block of slots and the cells run in parallel.
 * axis 0: (outer kk, inner jj) at ii = fixed; axis 1: (outer kk, inner ii) at
 * jj = fixed; axis 2: (outer jj, inner ii) at kk = fixed.  `edge` is the
 * lower edge of the guard layer along the face normal. */
static void inflow_face(const picard_params* p, int iteration, int axis, int fixed, int o_lo, int o_hi, int i_lo,
                        int i_hi, double edge, double* rp, int32_t* ip, int* n) {
  const double* dxyz = p->dxyz;
  const long long per_cell = per_cell_count(p);
  const int o_n = o_hi - o_lo + 1, i_n = i_hi - i_lo + 1;
  if (o_n <= 0 || i_n <= 0) return;
  const int n0 = *n;
#pragma omp parallel for collapse(2) schedule(static)
  for (int o = o_lo; o <= o_hi; ++o)
    for (int in = i_lo; in <= i_hi; ++in) {
      int ii, jj, kk;
      double x0, y0, z0;
      if (axis == 0) {
        ii = fixed, kk = o, jj = in;
        x0 = edge, y0 = p->Ly_min + dxyz[1] * (jj - 2), z0 = p->Lz_min + dxyz[2] * (kk - 2);
      } else if (axis == 1) {
        jj = fixed, kk = o, ii = in;
        x0 = p->Lx_min + dxyz[0] * (ii - 2), y0 = edge, z0 = p->Lz_min + dxyz[2] * (kk - 2);
      } else {
        kk = fixed, jj = o, ii = in;
        x0 = p->Lx_min + dxyz[0] * (ii - 2), y0 = p->Ly_min + dxyz[1] * (jj - 2), z0 = edge;
      }
      uint32_t a = (uint32_t)G3(ii, jj, kk);
      int slot = (int)(n0 + ((long long)(o - o_lo) * i_n + (in - i_lo)) * per_cell);
      for (int ss = 1; ss <= p->species; ++ss)
        for (int pp = 1; pp <= p->ipp[ss - 1]; ++pp)
          slot += create_group(p, p->seed, 2, (uint32_t)iteration, a, ss, pp, x0, y0, z0, rp, ip, slot);
    }
  *n = (int)(n0 + (long long)o_n * i_n * per_cell);
}

/* BCinflow.f90:23-476 on one rank.  Each guard cell of the open faces is
 * filled once: x faces span the extended y and z range, y faces extend z on
 * the +z side (+y face) or the -z side (-y face), z faces extend y on the -y
 * side (+z face) or the +y side (-z face).  The x faces loop over species
 * 1..S and the y and z faces over 2..S (BCinflow.f90:63, 204); ipp(1) = 0
 * makes the two the same. */
EXPORT int orc_bc_inflow(const picard_params* p, int iteration, double* rp, int32_t* ip, int32_t* num_local) {
  const double* dxyz = p->dxyz;
  const int Nx = p->nx, Ny = p->ny, Nz = p->nz;
  int ypos = (p->yflow && (p->Ly_max + 0.5 * dxyz[1] > p->ymax)) ? 1 : 0;
  int yneg = (p->yflow && (p->Ly_min - 0.5 * dxyz[1] < p->ymin)) ? 1 : 0;
  int zpos = (p->zflow && (p->Lz_max + 0.5 * dxyz[2] > p->zmax)) ? 1 : 0;
  int zneg = (p->zflow && (p->Lz_min - 0.5 * dxyz[2] < p->zmin)) ? 1 : 0;
  int xpos = (p->xflow && (p->Lx_max + 0.5 * dxyz[0] > p->xmax)) ? 1 : 0;
  int xneg = (p->xflow && (p->Lx_min - 0.5 * dxyz[0] < p->xmin)) ? 1 : 0;
  long long per_cell = per_cell_count(p);
  long long cells = (long long)(xpos + xneg) * (Nz + zneg + zpos) * (Ny + yneg + ypos) +
                    (long long)ypos * (Nz + zpos) * Nx + (long long)yneg * (Nz + zneg) * Nx +
                    (long long)zpos * (Ny + yneg) * Nx + (long long)zneg * (Ny + ypos) * Nx;
  int n = *num_local;
  if ((long long)n + cells * per_cell > p->max_per_proc) {
    fprintf(stderr, "oracle: particle capacity %d exceeded\n", p->max_per_proc);
    return 2;
  }
  if (xpos) inflow_face(p, iteration, 0, Nx + 2, 2 - zneg, Nz + 1 + zpos, 2 - yneg, Ny + 1 + ypos, p->Lx_max, rp, ip, &n);
  if (xneg)
    inflow_face(p, iteration, 0, 1, 2 - zneg, Nz + 1 + zpos, 2 - yneg, Ny + 1 + ypos, p->Lx_min - dxyz[0], rp, ip, &n);
  if (ypos) inflow_face(p, iteration, 1, Ny + 2, 2, Nz + 1 + zpos, 2, Nx + 1, p->Ly_max, rp, ip, &n);
  if (yneg) inflow_face(p, iteration, 1, 1, 2 - zneg, Nz + 1, 2, Nx + 1, p->Ly_min - dxyz[1], rp, ip, &n);
  if (zpos) inflow_face(p, iteration, 2, Nz + 2, 2 - yneg, Ny + 1, 2, Nx + 1, p->Lz_max, rp, ip, &n);
  if (zneg) inflow_face(p, iteration, 2, 1, 2, Ny + 1 + ypos, 2, Nx + 1, p->Lz_min - dxyz[2], rp, ip, &n);
  *num_local = n;
  return 0;
}

/* --------------------------------------------- AdvancePosition (a4) */

/* AdvancePosition.f90:15 */
EXPORT void orc_advance_position(double* rp, double dt, int32_t num_local) {
#pragma omp parallel for schedule(static)
  for (int pp = num_local; pp >= 1; --pp) {
    RP(1, pp) = RP(1, pp) + RP(4, pp) * dt;
    RP(2, pp) = RP(2, pp) + RP(5, pp) * dt;
    RP(3, pp) = RP(3, pp) + RP(6, pp) * dt;
  }
}

/* -------------------------------------------- ParticlesProduce (a18) */

/* ParticlesProduce.f90:21-108 */
EXPORT int orc_particles_produce(const picard_params* p, int iteration, double* rp, int32_t* ip, int32_t* num_local) {
  const double* dxyz = p->dxyz;
  const double dV = dxyz[0] * dxyz[1] * dxyz[2];
  const double dt = p->dt;
  double ue[8], uh[8], ui[8];
  for (int s = 0; s < 8; ++s) ue[s] = uh[s] = ui[s] = 0.0;
  const double* m = p->mass;
  for (int s = 0; s < p->species; ++s) {
    ue[s] = sqrt(2.0 * m[s] * p->Ek[s] * (1.0 / (m[0] * (m[s] + m[0]))));
    uh[s] = sqrt(2.0 * m[s] * p->Ek[s] * (1.0 / (m[1] * (m[s] + m[1]))));
    if (p->epp[s] > 0)
      ui[s] = sqrt(2.0 * m[0] * p->Ek[s] * (1.0 / (m[s] * (m[s] + m[0]))));
    else if (p->hpp[s] > 0)
      ui[s] = sqrt(2.0 * m[1] * p->Ek[s] * (1.0 / (m[s] * (m[s] + m[1]))));
    else
      ui[s] = 0.0;
  }
  int n = *num_local;
  for (int kk = 2; kk <= p->nz + 1; ++kk)
    for (int jj = 2; jj <= p->ny + 1; ++jj)
      for (int ii = 2; ii <= p->nx + 1; ++ii) {
        double x0 = p->Lx_min + dxyz[0] * (ii - 2);
        double y0 = p->Ly_min + dxyz[1] * (jj - 2);
        double z0 = p->Lz_min + dxyz[2] * (kk - 2);
        double xc = x0 + 0.5 * dxyz[0], yc = y0 + 0.5 * dxyz[1], zc = z0 + 0.5 * dxyz[2];
        double r2 = xc * xc + yc * yc + zc * zc;
        double r1 = sqrt(r2);
        double r1c = 4.0 * r1;
        if (r1c * r1c * r1c < dV) {
          double s = 0.0;
          const double fa[8][3] = {{0.25, 0.25, 0.25}, {0.25, 0.25, 0.75}, {0.25, 0.75, 0.25}, {0.75, 0.25, 0.25},
                                   {0.25, 0.75, 0.75}, {0.75, 0.25, 0.75}, {0.75, 0.75, 0.25}, {0.75, 0.75, 0.75}};
          for (int q = 0; q < 8; ++q) {
            double a = x0 + fa[q][0] * dxyz[0], b = y0 + fa[q][1] * dxyz[1], c = z0 + fa[q][2] * dxyz[2];
            s = s + sqrt(a * a + b * b + c * c);
          }
          r1 = s * 0.125;
          r2 = r1 * r1;
        }
        uint32_t acell = (uint32_t)G3(ii, jj, kk);
        for (int ss = 1; ss <= p->species; ++ss) {
          int s0 = ss - 1;
          double nden;
          if (p->vn[s0] > 0.0)
            nden = p->Qn[s0] / (2.0 * TAU * r2 * p->vn[s0]) * exp(-p->nu_d[s0] * r1 / p->vn[s0]);
          else
            nden = 0.0;
          int num_create;
          if (p->n2p[s0] > 0.0) {
            double rnd = orc_site_uniform(p->seed, acell, (uint32_t)ss, (uint32_t)iteration, 3, 0);
            double rate = p->nu_i[s0] * nden * dV / p->n2p[s0];
            if (p->produce_dt_scaled) rate = rate * dt;
            num_create = (int)(rate + rnd);
          } else {
            num_create = 0;
          }
          for (int pp = 1; pp <= num_create; ++pp) {
            int add = 1 + p->epp[s0] + p->hpp[s0];
            if (!append_guard(n, add, p->max_per_proc)) return 2;
            site_rng r;
            site_init(&r, p->seed, acell, ((uint32_t)ss << 24) | (uint32_t)pp, (uint32_t)iteration, 4);
            double rnd7[7];
            for (int q = 0; q < 7; ++q) rnd7[q] = site_u(&r, (uint32_t)q);
            double* ion = rp + (size_t)8 * n;
            ip[n] = ss;
            ion[0] = x0 + dxyz[0] * rnd7[0];
            ion[1] = y0 + dxyz[1] * rnd7[1];
            ion[2] = z0 + dxyz[2] * rnd7[2];
            ion[6] = 0.0; ion[7] = 0.0;
            double rn = sqrt(ion[0] * ion[0] + ion[1] * ion[1] + ion[2] * ion[2]);
            double un = sqrt(rnd7[3] * rnd7[3] + rnd7[4] * rnd7[4] + rnd7[5] * rnd7[5]);
            for (int c = 0; c < 3; ++c) ion[3 + c] = p->vn[s0] * ion[c] / rn + ui[s0] * rnd7[3 + c] / un;
            for (int c = 0; c < 3; ++c) ion[c] = ion[c] + ion[3 + c] * dt * rnd7[6];
            int k = 1;
            for (int ee = 1; ee <= p->epp[s0]; ++ee, ++k) {
              double* q = rp + (size_t)8 * (n + k);
              ip[n + k] = 1;
              q[6] = 0.0; q[7] = 0.0;
              for (int c = 0; c < 3; ++c) q[3 + c] = ion[3 + c] - (ue[s0] + ui[s0]) * rnd7[3 + c] / un;
              for (int c = 0; c < 3; ++c) q[c] = ion[c] - ion[3 + c] * dt * rnd7[6] + q[3 + c] * dt * rnd7[6];
            }
            for (int ee = 1; ee <= p->hpp[s0]; ++ee, ++k) {
              double* q = rp + (size_t)8 * (n + k);
              ip[n + k] = 2;
              q[6] = 0.0; q[7] = 0.0;
              for (int c = 0; c < 3; ++c) q[3 + c] = ion[3 + c] - (uh[s0] + ui[s0]) * rnd7[3 + c] / un;
              for (int c = 0; c < 3; ++c) q[c] = ion[c] - ion[3 + c] * dt * rnd7[6] + q[3 + c] * dt * rnd7[6];
            }
            n += k;
          }
        }
      }
  *num_local = n;
  return 0;
}

/* ------------------------------------------------ BCoutflow (a5) */

/* BCoutflow.f90:24-83 */
EXPORT void orc_bc_outflow(const picard_params* p, double* rp, int32_t* ip, int32_t* num_local) {
  int n = *num_local;
  for (int pp = n; pp >= 1; --pp) {
    int del = 0;
    double x = RP(1, pp), y = RP(2, pp), z = RP(3, pp);
    if (p->xflow && (x < p->xmin || x > p->xmax)) del = 1;
    if (p->yflow && (y < p->ymin || y > p->ymax)) del = 1;
    if (p->zflow && (z < p->zmin || z > p->zmax)) del = 1;
    if (x < 2.0 * p->Lx_min - p->Lx_max || x > 2.0 * p->Lx_max - p->Lx_min) del = 1;
    if (y < 2.0 * p->Ly_min - p->Ly_max || y > 2.0 * p->Ly_max - p->Ly_min) del = 1;
    if (z < 2.0 * p->Lz_min - p->Lz_max || z > 2.0 * p->Lz_max - p->Lz_min) del = 1;
    if (del) {
      if (pp != n) {
        memcpy(&RP(1, pp), &RP(1, n), sizeof(double) * 8);
        IP(pp) = IP(n);
      }
      n = n - 1;
    }
  }
  *num_local = n;
}

/* ----------------------------------------- ParticlesTransfer (a6) */

/* ParticlesTransfer.f90:494-519: with one rank every neighbour is the rank
 * itself, the MPI blocks are skipped and all three axes are wrapped. */
EXPORT void orc_particles_transfer(const picard_params* p, double* rp, int32_t num_local) {
  const double Lx = p->xmax - p->xmin, Ly = p->ymax - p->ymin, Lz = p->zmax - p->zmin;
#pragma omp parallel for schedule(static)
  for (int pp = num_local; pp >= 1; --pp) {
    if (RP(3, pp) < p->zmin) RP(3, pp) = RP(3, pp) + Lz;
    if (RP(3, pp) > p->zmax) RP(3, pp) = RP(3, pp) - Lz;
    if (RP(2, pp) < p->ymin) RP(2, pp) = RP(2, pp) + Ly;
    if (RP(2, pp) > p->ymax) RP(2, pp) = RP(2, pp) - Ly;
    if (RP(1, pp) < p->xmin) RP(1, pp) = RP(1, pp) + Lx;
    if (RP(1, pp) > p->xmax) RP(1, pp) = RP(1, pp) - Lx;
  }
}

/* ----------------------------------------- CIC weights (a7, a13) */

typedef struct {
  int i, j, k;      /* 1-based base node (index_local) */
  double F[8];      /* F1..F8 of the reference, not yet divided by dV */
  double rest[3];
} cic_t;

/* ParticlesGridify.f90:70-77 / AdvanceVelocity.f90:44-51, 65-72 */
static inline void cic_weights(const picard_params* p, const double* x, cic_t* w) {
  const double* d = p->dxyz;
  double rest[3], drest[3];
  rest[0] = fmod(x[0] - p->Lx_min + 0.5 * d[0], d[0]);
  rest[1] = fmod(x[1] - p->Ly_min + 0.5 * d[1], d[1]);
  rest[2] = fmod(x[2] - p->Lz_min + 0.5 * d[2], d[2]);
  for (int c = 0; c < 3; ++c) drest[c] = d[c] - rest[c];
  w->i = 1 + (int)((x[0] - p->Lx_min) / d[0] + 0.5);
  w->j = 1 + (int)((x[1] - p->Ly_min) / d[1] + 0.5);
  w->k = 1 + (int)((x[2] - p->Lz_min) / d[2] + 0.5);
  w->F[0] = drest[0] * drest[1] * drest[2];
  w->F[1] = rest[0] * drest[1] * drest[2];
  w->F[2] = drest[0] * rest[1] * drest[2];
  w->F[3] = drest[0] * drest[1] * rest[2];
  w->F[4] = rest[0] * rest[1] * drest[2];
  w->F[5] = drest[0] * rest[1] * rest[2];
  w->F[6] = rest[0] * drest[1] * rest[2];
  w->F[7] = rest[0] * rest[1] * rest[2];
  for (int c = 0; c < 3; ++c) w->rest[c] = rest[c];
}

/* offsets of F1..F8 (ParticlesGridify.f90:98-121) */
static const int OFF[8][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {1, 1, 0}, {0, 1, 1}, {1, 0, 1}, {1, 1, 1}};

/* Base node indices of one particle (1-based), for the bit-exact cell test. */
EXPORT void orc_cell_indices(const picard_params* p, const double* rp, int32_t num_local, int32_t* ijk) {
  for (int pp = 1; pp <= num_local; ++pp) {
    cic_t w;
    cic_weights(p, &RP(1, pp), &w);
    ijk[3 * (pp - 1) + 0] = w.i;
    ijk[3 * (pp - 1) + 1] = w.j;
    ijk[3 * (pp - 1) + 2] = w.k;
  }
}

/* Ghost-layer folds of ParticlesGridify.f90:149-171 (z), 203-225 (y),
 * 256-278 (x) on one rank, for an array with `ncomp` leading components. */
static void fold_ghosts(const picard_params* p, double* A, int ncomp) {
  const int Nx = p->nx, Ny = p->ny, Nz = p->nz;
  const size_t nxp = NXP, nyp = NYP, nzp = NZP;
#define AA(c, i, j, k) A[(size_t)(c) + (size_t)ncomp * (((size_t)(i)-1) + nxp * (((size_t)(j)-1) + nyp * ((size_t)(k)-1)))]
  /* z */
  for (size_t j = 1; j <= nyp; ++j)
    for (size_t i = 1; i <= nxp; ++i)
      for (int c = 0; c < ncomp; ++c) {
        if (p->zflow) {
          AA(c, i, j, 2) = AA(c, i, j, 2) + AA(c, i, j, 1);
          AA(c, i, j, 1) = 0.0;
          AA(c, i, j, Nz + 1) = AA(c, i, j, Nz + 1) + AA(c, i, j, Nz + 2);
          AA(c, i, j, Nz + 2) = 0.0;
        } else {
          double n1 = AA(c, i, j, 1), n2 = AA(c, i, j, 2), m1 = AA(c, i, j, Nz + 1), m2 = AA(c, i, j, Nz + 2);
          AA(c, i, j, 1) = n1 + m1;
          AA(c, i, j, 2) = n2 + m2;
          AA(c, i, j, Nz + 1) = m1 + n1;
          AA(c, i, j, Nz + 2) = m2 + n2;
        }
      }
  /* y */
  for (size_t k = 1; k <= nzp; ++k)
    for (size_t i = 1; i <= nxp; ++i)
      for (int c = 0; c < ncomp; ++c) {
        if (p->yflow) {
          AA(c, i, 2, k) = AA(c, i, 2, k) + AA(c, i, 1, k);
          AA(c, i, 1, k) = 0.0;
          AA(c, i, Ny + 1, k) = AA(c, i, Ny + 1, k) + AA(c, i, Ny + 2, k);
          AA(c, i, Ny + 2, k) = 0.0;
        } else {
          double n1 = AA(c, i, 1, k), n2 = AA(c, i, 2, k), m1 = AA(c, i, Ny + 1, k), m2 = AA(c, i, Ny + 2, k);
          AA(c, i, 1, k) = n1 + m1;
          AA(c, i, 2, k) = n2 + m2;
          AA(c, i, Ny + 1, k) = m1 + n1;
          AA(c, i, Ny + 2, k) = m2 + n2;
        }
      }
  /* x */
  for (size_t k = 1; k <= nzp; ++k)
    for (size_t j = 1; j <= nyp; ++j)
      for (int c = 0; c < ncomp; ++c) {
        if (p->xflow) {
          AA(c, 2, j, k) = AA(c, 2, j, k) + AA(c, 1, j, k);
          AA(c, 1, j, k) = 0.0;
          AA(c, Nx + 1, j, k) = AA(c, Nx + 1, j, k) + AA(c, Nx + 2, j, k);
          AA(c, Nx + 2, j, k) = 0.0;
        } else {
          double n1 = AA(c, 1, j, k), n2 = AA(c, 2, j, k), m1 = AA(c, Nx + 1, j, k), m2 = AA(c, Nx + 2, j, k);
          AA(c, 1, j, k) = n1 + m1;
          AA(c, 2, j, k) = n2 + m2;
          AA(c, Nx + 1, j, k) = m1 + n1;
          AA(c, Nx + 2, j, k) = m2 + n2;
        }
      }
#undef AA
}

/* ------------------------------------------ ParticlesGridify (a7) */

/* ParticlesGridify.f90:56-123 (deposit), 149-278 (folds), 288-293 (C) */
EXPORT void orc_particles_gridify(const picard_params* p, const double* rp, const int32_t* ip, int32_t num_local,
                                  double* N, double* C) {
  const int S = p->species;
  const size_t nn = (size_t)NXP * NYP * NZP;
  const double dV = p->dxyz[0] * p->dxyz[1] * p->dxyz[2];
  memset(N, 0, sizeof(double) * nn * S);
  memset(C, 0, sizeof(double) * nn);
  for (int pp = num_local; pp >= 1; --pp) {
    cic_t w;
    cic_weights(p, &RP(1, pp), &w);
    int s = IP(pp);
    double n2p = p->n2p[s - 1];
    for (int q = 0; q < 8; ++q) {
      size_t g = G3(w.i + OFF[q][0], w.j + OFF[q][1], w.k + OFF[q][2]);
      N[(size_t)(s - 1) + (size_t)S * g] = N[(size_t)(s - 1) + (size_t)S * g] + w.F[q] / dV * n2p;
    }
  }
  fold_ghosts(p, N, S);
  for (int s = 0; s < S; ++s)
    for (size_t g = 0; g < nn; ++g) C[g] = C[g] + N[(size_t)s + (size_t)S * g] * p->charge[s];
}

/* ------------------------------------- ParticlesGridifyAll (a15) */

/* ParticlesGridifyAll.f90:60-202 (deposit of N and flux F), folds, C */
EXPORT void orc_particles_gridify_all(const picard_params* p, const double* rp, const int32_t* ip, int32_t num_local,
                                      double* F, double* N, double* C) {
  const int S = p->species;
  const size_t nn = (size_t)NXP * NYP * NZP;
  const double dV = p->dxyz[0] * p->dxyz[1] * p->dxyz[2];
  memset(N, 0, sizeof(double) * nn * S);
  memset(F, 0, sizeof(double) * nn * S * 3);
  memset(C, 0, sizeof(double) * nn);
  for (int pp = num_local; pp >= 1; --pp) {
    cic_t w;
    cic_weights(p, &RP(1, pp), &w);
    int s = IP(pp);
    double n2p = p->n2p[s - 1];
    for (int q = 0; q < 8; ++q) {
      size_t g = G3(w.i + OFF[q][0], w.j + OFF[q][1], w.k + OFF[q][2]);
      N[(size_t)(s - 1) + (size_t)S * g] = N[(size_t)(s - 1) + (size_t)S * g] + w.F[q] / dV * n2p;
    }
    for (int c = 0; c < 3; ++c)
      for (int q = 0; q < 8; ++q) {
        size_t g = G3(w.i + OFF[q][0], w.j + OFF[q][1], w.k + OFF[q][2]);
        size_t f = (size_t)(s - 1) + (size_t)S * ((size_t)c + 3 * g);
        F[f] = F[f] + w.F[q] / dV * n2p * RP(4 + c, pp);
      }
  }
  fold_ghosts(p, N, S);
  fold_ghosts(p, F, 3 * S);
  for (int s = 0; s < S; ++s)
    for (size_t g = 0; g < nn; ++g) C[g] = C[g] + N[(size_t)s + (size_t)S * g] * p->charge[s];
}

/* -------------------------------------------- BCpotentials (a9) */

/* BCpotentials.f90:36-139 on one rank (bi = bj = bk = 0, Nx = Nx_local).
 * stride > 1 computes only every stride-th node of each face (in the face's
 * loop order) -- a bounded sample for timing the CPU baseline. */
static void bc_potentials_core(const picard_params* p, double* U, const double* C, const double* D, int stride) {
  const int Nx = p->nx, Ny = p->ny, Nz = p->nz;
  const size_t nn = (size_t)NXP * NYP * NZP;
  const int DX = 2 * Nx + 1, DY = 2 * Ny + 1;
  const double scale = 1.0 / (2.0 * TAU * EPS0);
#define DD(i, j, k) D[(size_t)((i)-1) + (size_t)DX * ((size_t)((j)-1) + (size_t)DY * (size_t)((k)-1))]
  memset(U, 0, sizeof(double) * nn);
  /* sum(C(2:N+1,2:N+1,2:N+1) * D(di:di+Nx-1, dj:dj+Ny-1, dk:dk+Nz-1)) in array order */
#define WINDOW_SUM(di, dj, dk, out)                                   \
  do {                                                                \
    double s_ = 0.0;                                                  \
    for (int k_ = 1; k_ <= Nz; ++k_)                                  \
      for (int j_ = 1; j_ <= Ny; ++j_)                                \
        for (int i_ = 1; i_ <= Nx; ++i_)                              \
          s_ += C[G3(i_ + 1, j_ + 1, k_ + 1)] *                       \
                DD((di) + i_ - 1, (dj) + j_ - 1, (dk) + k_ - 1);      \
    (out) = s_;                                                       \
  } while (0)
  if (p->xflow) {
#pragma omp parallel for collapse(2) schedule(dynamic)
    for (int kk = 1; kk <= Nz; ++kk)
      for (int jj = 1; jj <= Ny; ++jj) {
        if (stride > 1 && ((jj - 1) + Ny * (kk - 1)) % stride) continue;
        int dj = Ny + 1 + (1 - jj), dk = Nz + 1 + (1 - kk);
        double u0, u1;
        WINDOW_SUM(Nx + 2, dj, dk, u0);
        WINDOW_SUM(Nx + 1 - Nx, dj, dk, u1);
        U[G3(1, jj + 1, kk + 1)] = u0 * scale;
        U[G3(Nx + 2, jj + 1, kk + 1)] = u1 * scale;
      }
  }
  if (p->yflow) {
#pragma omp parallel for collapse(2) schedule(dynamic)
    for (int kk = 1; kk <= Nz; ++kk)
      for (int ii = 1; ii <= Nx; ++ii) {
        if (stride > 1 && ((ii - 1) + Nx * (kk - 1)) % stride) continue;
        int di = Nx + 1 + (1 - ii), dk = Nz + 1 + (1 - kk);
        double u0, u1;
        WINDOW_SUM(di, Ny + 2, dk, u0);
        WINDOW_SUM(di, Ny + 1 - Ny, dk, u1);
        U[G3(ii + 1, 1, kk + 1)] = u0 * scale;
        U[G3(ii + 1, Ny + 2, kk + 1)] = u1 * scale;
      }
  }
  if (p->zflow) {
#pragma omp parallel for collapse(2) schedule(dynamic)
    for (int jj = 1; jj <= Ny; ++jj)
      for (int ii = 1; ii <= Nx; ++ii) {
        if (stride > 1 && ((ii - 1) + Nx * (jj - 1)) % stride) continue;
        int di = Nx + 1 + (1 - ii), dj = Ny + 1 + (1 - jj);
        double u0, u1;
        WINDOW_SUM(di, dj, Nz + 2, u0);
        WINDOW_SUM(di, dj, Nz + 1 - Nz, u1);
        U[G3(ii + 1, jj + 1, 1)] = u0 * scale;
        U[G3(ii + 1, jj + 1, Nz + 2)] = u1 * scale;
      }
  }
#undef WINDOW_SUM
#undef DD
}

EXPORT void orc_bc_potentials(const picard_params* p, double* U, const double* C, const double* D) {
  bc_potentials_core(p, U, C, D, 1);
}

EXPORT void orc_bc_potentials_sampled(const picard_params* p, double* U, const double* C, const double* D,
                                      int stride) {
  bc_potentials_core(p, U, C, D, stride < 1 ? 1 : stride);
}

/* ----------------------------------------- CalcEpotential (a10) */

/* Ghost refresh of CalcEpotential.f90:100-239 on one rank: periodic axes copy
 * the opposite interior layer, open axes keep their boundary values. */
static void refresh_periodic_u(const picard_params* p, double* U) {
  const int Nx = p->nx, Ny = p->ny, Nz = p->nz;
  if (!p->zflow)
    for (int j = 1; j <= Ny + 2; ++j)
      for (int i = 1; i <= Nx + 2; ++i) {
        U[G3(i, j, 1)] = U[G3(i, j, Nz + 1)];
        U[G3(i, j, Nz + 2)] = U[G3(i, j, 2)];
      }
  if (!p->yflow)
    for (int k = 1; k <= Nz + 2; ++k)
      for (int i = 1; i <= Nx + 2; ++i) {
        U[G3(i, 1, k)] = U[G3(i, Ny + 1, k)];
        U[G3(i, Ny + 2, k)] = U[G3(i, 2, k)];
      }
  if (!p->xflow)
    for (int k = 1; k <= Nz + 2; ++k)
      for (int j = 1; j <= Ny + 2; ++j) {
        U[G3(1, j, k)] = U[G3(Nx + 1, j, k)];
        U[G3(Nx + 2, j, k)] = U[G3(2, j, k)];
      }
}

/* Sum of squares over interior nodes: per z-plane partial sums in (j, i)
 * order, then the planes in k order (independent of the thread count). */
static double interior_sumsq(const picard_params* p, const double* A, double* plane) {
  const int Nx = p->nx, Ny = p->ny, Nz = p->nz;
#pragma omp parallel for schedule(static)
  for (int k = 2; k <= Nz + 1; ++k) {
    double s = 0.0;
    for (int j = 2; j <= Ny + 1; ++j)
      for (int i = 2; i <= Nx + 1; ++i) {
        double v = A[G3(i, j, k)];
        s += v * v;
      }
    plane[k] = s;
  }
  double t = 0.0;
  for (int k = 2; k <= Nz + 1; ++k) t += plane[k];
  return t;
}

/* CalcEpotential.f90:44-242.  Returns the number of sweeps done; *converged
 * is 0 if the loop ran to 2*maxit+1. */
EXPORT int orc_calc_epotential(const picard_params* p, double* U, const double* C, double maxerr, int maxit,
                               int* converged, double* resid_out) {
  const int Nx = p->nx, Ny = p->ny, Nz = p->nz;
  const size_t nn = (size_t)NXP * NYP * NZP;
  const double* d = p->dxyz;
  const double dV = d[0] * d[1] * d[2];
  double* b = (double*)calloc(nn, sizeof(double));
  double* res = (double*)calloc(nn, sizeof(double));
  double* Un = (double*)malloc(nn * sizeof(double));
  double* plane = (double*)calloc((size_t)Nz + 3, sizeof(double));
  const double S = (d[0] * d[1]) * (d[0] * d[1]) + (d[0] * d[2]) * (d[0] * d[2]) + (d[1] * d[2]) * (d[1] * d[2]);
  const double ax = 0.5 * (1.0 / S) * ((d[1] * d[2]) * (d[1] * d[2]));
  const double ay = 0.5 * (1.0 / S) * ((d[0] * d[2]) * (d[0] * d[2]));
  const double az = 0.5 * (1.0 / S) * ((d[0] * d[1]) * (d[0] * d[1]));
  const double af = 0.5 * (1.0 / S) * ((d[0] * d[1] * d[2]) * (d[0] * d[1] * d[2]));
  const double idx2 = d[0] * d[0], idy2 = d[1] * d[1], idz2 = d[2] * d[2];
  const double binv = 1.0 / (dV * EPS0);
  for (size_t g = 0; g < nn; ++g) b[g] = -C[g] * binv;
  double b_global = interior_sumsq(p, b, plane);
  double b_sqrt = sqrt(b_global);
  double r_global = 1.0 * b_global;
  int ss, done = 0;
  memcpy(Un, U, nn * sizeof(double));
  for (ss = 1; ss <= 2 * maxit + 1; ++ss) {
    if (ss <= maxit) {
      if (sqrt(r_global) <= maxerr * b_sqrt) {
        done = 1;
        break;
      }
    }
#pragma omp parallel for schedule(static)
    for (int k = 2; k <= Nz + 1; ++k)
      for (int j = 2; j <= Ny + 1; ++j)
        for (int i = 2; i <= Nx + 1; ++i) {
          Un[G3(i, j, k)] = ax * (U[G3(i + 1, j, k)] + U[G3(i - 1, j, k)]) +
                            ay * (U[G3(i, j + 1, k)] + U[G3(i, j - 1, k)]) +
                            az * (U[G3(i, j, k + 1)] + U[G3(i, j, k - 1)]) - af * (b[G3(i, j, k)]);
        }
#pragma omp parallel for schedule(static)
    for (int k = 2; k <= Nz + 1; ++k)
      for (int j = 2; j <= Ny + 1; ++j)
        for (int i = 2; i <= Nx + 1; ++i) U[G3(i, j, k)] = Un[G3(i, j, k)];
#pragma omp parallel for schedule(static)
    for (int k = 2; k <= Nz + 1; ++k)
      for (int j = 2; j <= Ny + 1; ++j)
        for (int i = 2; i <= Nx + 1; ++i) {
          double u = U[G3(i, j, k)];
          res[G3(i, j, k)] = b[G3(i, j, k)] - ((U[G3(i + 1, j, k)] + U[G3(i - 1, j, k)] - 2.0 * u) / idx2 +
                                               (U[G3(i, j + 1, k)] + U[G3(i, j - 1, k)] - 2.0 * u) / idy2 +
                                               (U[G3(i, j, k + 1)] + U[G3(i, j, k - 1)] - 2.0 * u) / idz2);
        }
    r_global = interior_sumsq(p, res, plane);
    refresh_periodic_u(p, U);
  }
  if (resid_out) resid_out[0] = sqrt(r_global), resid_out[1] = b_sqrt;
  free(b);
  free(res);
  free(Un);
  free(plane);
  if (converged) *converged = done;
  return done ? ss - 1 : 2 * maxit + 1;
}

/* -------------------------------------- CalcEfield + BCfields (a11, a12) */

/* CalcEfield.f90:27-34 plus its halo exchange on one rank (periodic axes copy
 * the opposite interior layer). */
EXPORT void orc_calc_efield(const picard_params* p, double* E, const double* U) {
  const int Nx = p->nx, Ny = p->ny, Nz = p->nz;
  const size_t nn = (size_t)NXP * NYP * NZP;
  const double* d = p->dxyz;
  memset(E, 0, sizeof(double) * 3 * nn);
#pragma omp parallel for schedule(static)
  for (int k = 2; k <= Nz + 1; ++k)
    for (int j = 2; j <= Ny + 1; ++j)
      for (int i = 2; i <= Nx + 1; ++i) {
        size_t g = G3(i, j, k);
        E[3 * g + 2] = -(U[G3(i, j, k + 1)] - U[G3(i, j, k - 1)]) * 0.5 / d[2];
        E[3 * g + 1] = -(U[G3(i, j + 1, k)] - U[G3(i, j - 1, k)]) * 0.5 / d[1];
        E[3 * g + 0] = -(U[G3(i + 1, j, k)] - U[G3(i - 1, j, k)]) * 0.5 / d[0];
      }
  if (!p->zflow)
    for (int j = 1; j <= Ny + 2; ++j)
      for (int i = 1; i <= Nx + 2; ++i)
        for (int c = 0; c < 3; ++c) {
          E[3 * G3(i, j, 1) + c] = E[3 * G3(i, j, Nz + 1) + c];
          E[3 * G3(i, j, Nz + 2) + c] = E[3 * G3(i, j, 2) + c];
        }
  if (!p->yflow)
    for (int k = 1; k <= Nz + 2; ++k)
      for (int i = 1; i <= Nx + 2; ++i)
        for (int c = 0; c < 3; ++c) {
          E[3 * G3(i, 1, k) + c] = E[3 * G3(i, Ny + 1, k) + c];
          E[3 * G3(i, Ny + 2, k) + c] = E[3 * G3(i, 2, k) + c];
        }
  if (!p->xflow)
    for (int k = 1; k <= Nz + 2; ++k)
      for (int j = 1; j <= Ny + 2; ++j)
        for (int c = 0; c < 3; ++c) {
          E[3 * G3(1, j, k) + c] = E[3 * G3(Nx + 1, j, k) + c];
          E[3 * G3(Nx + 2, j, k) + c] = E[3 * G3(2, j, k) + c];
        }
}

/* BCfields.f90:31-90 on one rank: zero the outer ghost layer of open faces. */
EXPORT void orc_bc_fields(const picard_params* p, double* E) {
  const int Nx = p->nx, Ny = p->ny, Nz = p->nz;
  if (p->zflow)
    for (int j = 1; j <= Ny + 2; ++j)
      for (int i = 1; i <= Nx + 2; ++i)
        for (int c = 0; c < 3; ++c) E[3 * G3(i, j, Nz + 2) + c] = 0.0, E[3 * G3(i, j, 1) + c] = 0.0;
  if (p->yflow)
    for (int k = 1; k <= Nz + 2; ++k)
      for (int i = 1; i <= Nx + 2; ++i)
        for (int c = 0; c < 3; ++c) E[3 * G3(i, Ny + 2, k) + c] = 0.0, E[3 * G3(i, 1, k) + c] = 0.0;
  if (p->xflow)
    for (int k = 1; k <= Nz + 2; ++k)
      for (int j = 1; j <= Ny + 2; ++j)
        for (int c = 0; c < 3; ++c) E[3 * G3(Nx + 2, j, k) + c] = 0.0, E[3 * G3(1, j, k) + c] = 0.0;
}

/* ------------------------------------------ AdvanceVelocity (a13, a14) */

/* 8-node gather of AdvanceVelocity.f90:44-78 */
static inline void gather_e(const picard_params* p, const double* E, const double* x, double Ep[3]) {
  const double dV = p->dxyz[0] * p->dxyz[1] * p->dxyz[2];
  cic_t w;
  cic_weights(p, x, &w);
  for (int c = 0; c < 3; ++c) {
    double s = 0.0;
    for (int q = 0; q < 8; ++q) {
      double e = E[3 * G3(w.i + OFF[q][0], w.j + OFF[q][1], w.k + OFF[q][2]) + c];
      if (q == 0)
        s = e * w.F[0];
      else
        s = s + e * w.F[q];
    }
    Ep[c] = s / dV;
  }
}

/* mode 0: AdvanceVelocity (full Boris, AdvanceVelocity.f90:39-121)
 * mode 1: AdvanceVelocityExp (AdvanceVelocity.f90:154-232)
 * mode 2: AdvanceVelocityImp (AdvanceVelocity.f90:265-343) */
EXPORT void orc_advance_velocity(const picard_params* p, double* rp, const int32_t* ip, int32_t num_local,
                                 const double* E, double dt, double deltat, int mode) {
  double etadt2[8], tBt[8][4];
  for (int s = 0; s < 8; ++s) {
    if (mode == 0) {
      etadt2[s] = 0.5 * dt * p->eta[s];
      for (int c = 0; c < 4; ++c) tBt[s][c] = p->tB[s][c];
    } else {
      etadt2[s] = 0.5 * dt * p->eta[s] * 2.0 * deltat / dt;
      for (int c = 0; c < 4; ++c) tBt[s][c] = p->tB[s][c] * 2.0 * deltat / dt;
    }
  }
  const double* B = p->B0;
  const double* ve = p->ve;
#pragma omp parallel for schedule(static)
  for (int pp = num_local; pp >= 1; --pp) {
    double Ep[3];
    gather_e(p, E, &RP(1, pp), Ep);
    int s = IP(pp) - 1;
    double* v = &RP(4, pp);
    if (p->fluid[s]) {
      if (p->gyration[s]) {
        double vmin[3], vmid[3];
        double vb = v[0] * B[0] + v[1] * B[1] + v[2] * B[2];
        for (int c = 0; c < 3; ++c) vmin[c] = vb * B[c];
        vmid[0] = vmin[0] + (Ep[1] * B[2] - Ep[2] * B[1]);
        vmid[1] = vmin[1] + (Ep[2] * B[0] - Ep[0] * B[2]);
        vmid[2] = vmin[2] + (Ep[0] * B[1] - Ep[1] * B[0]);
        double ib = 1.0 / (B[0] * B[0] + B[1] * B[1] + B[2] * B[2]);
        for (int c = 0; c < 3; ++c) v[c] = vmid[c] * ib;
      }
      continue;
    }
    const double* tB = tBt[s];
    double vmin[3], vmid[3];
    if (mode == 0) {
      const double* sB = p->sB[s];
      double vplus[3];
      for (int c = 0; c < 3; ++c) vmin[c] = v[c] - ve[c] + etadt2[s] * Ep[c];
      vmid[0] = vmin[0] + vmin[1] * tB[2] - vmin[2] * tB[1];
      vmid[1] = vmin[1] + vmin[2] * tB[0] - vmin[0] * tB[2];
      vmid[2] = vmin[2] + vmin[0] * tB[1] - vmin[1] * tB[0];
      vplus[0] = vmin[0] + vmid[1] * sB[2] - vmid[2] * sB[1];
      vplus[1] = vmin[1] + vmid[2] * sB[0] - vmid[0] * sB[2];
      vplus[2] = vmin[2] + vmid[0] * sB[1] - vmid[1] * sB[0];
      for (int c = 0; c < 3; ++c) v[c] = vplus[c] + ve[c] + etadt2[s] * Ep[c];
    } else {
      if (mode == 1)
        for (int c = 0; c < 3; ++c) vmin[c] = v[c] - ve[c];
      else
        for (int c = 0; c < 3; ++c) vmin[c] = v[c] - ve[c] + etadt2[s] * Ep[c];
      vmid[0] = vmin[0] + vmin[1] * tB[2] - vmin[2] * tB[1];
      vmid[1] = vmin[1] + vmin[2] * tB[0] - vmin[0] * tB[2];
      vmid[2] = vmin[2] + vmin[0] * tB[1] - vmin[1] * tB[0];
      double smid = vmid[0] * vmid[0] + vmid[1] * vmid[1] + vmid[2] * vmid[2];
      if (smid > 0.0) {
        double smin = vmin[0] * vmin[0] + vmin[1] * vmin[1] + vmin[2] * vmin[2];
        double f = sqrt(smin / smid);
        for (int c = 0; c < 3; ++c) vmid[c] = vmid[c] * f;
      }
      if (mode == 1)
        for (int c = 0; c < 3; ++c) v[c] = vmid[c] + ve[c] + etadt2[s] * Ep[c];
      else
        for (int c = 0; c < 3; ++c) v[c] = vmid[c] + ve[c];
    }
  }
}

/* ------------------------------------------------ diagnostics (a16) */

/* picard.f90:653-664: out = {uP, uE, uB} */
EXPORT void orc_energy(const picard_params* p, const double* rp, const int32_t* ip, int32_t num_local,
                       const double* E, double out[3]) {
  const int Nx = p->nx, Ny = p->ny, Nz = p->nz;
  const double dV = p->dxyz[0] * p->dxyz[1] * p->dxyz[2];
  double sB = 0.0, sE = 0.0, sP = 0.0;
  for (int k = 2; k <= Nz + 1; ++k)
    for (int j = 2; j <= Ny + 1; ++j)
      for (int i = 2; i <= Nx + 1; ++i) {
        for (int c = 0; c < 3; ++c) sB += p->B0[c] * p->B0[c];
        size_t g = G3(i, j, k);
        double e0 = E[3 * g] + p->E0[0], e1 = E[3 * g + 1] + p->E0[1], e2 = E[3 * g + 2] + p->E0[2];
        sE += e0 * e0 + e1 * e1 + e2 * e2;
      }
  for (int pp = 1; pp <= num_local; ++pp) {
    int s = IP(pp) - 1;
    double v2 = RP(4, pp) * RP(4, pp) + RP(5, pp) * RP(5, pp) + RP(6, pp) * RP(6, pp);
    sP += p->n2p[s] * p->mass[s] * v2;
  }
  out[0] = sP * 0.5;
  out[1] = sE * 0.5 * EPS0 * dV;
  out[2] = sB * 0.5 / MU0 * dV;
}

/* --------------------------------------------------- one iteration (a1) */

typedef struct {
  double* D;
  double* U;
  double* E;
  double* N;
  double* C;
} orc_fields;

/* picard.f90:556-631 with writeFields = writeParticles = .false.  Returns the
 * number of Jacobi sweeps (negative on capacity overflow). */
EXPORT int orc_step(const picard_params* p, int iteration, double* rp, int32_t* ip, int32_t* num_local, double* D,
                    double* U, double* E, double* N, double* C) {
  if (orc_bc_inflow(p, iteration, rp, ip, num_local)) return -1;
  orc_advance_position(rp, p->dt, *num_local);
  if (orc_particles_produce(p, iteration, rp, ip, num_local)) return -1;
  orc_bc_outflow(p, rp, ip, num_local);
  orc_particles_transfer(p, rp, *num_local);
  orc_particles_gridify(p, rp, ip, *num_local, N, C);
  orc_bc_potentials(p, U, C, D);
  int conv = 0;
  int sweeps = orc_calc_epotential(p, U, C, p->maxerr, p->maxit, &conv, NULL);
  orc_calc_efield(p, E, U);
  orc_bc_fields(p, E);
  orc_advance_velocity(p, rp, ip, *num_local, E, p->dt, 0.0, 0);
  return sweeps;
}
