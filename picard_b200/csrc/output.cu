// output.cu -- Picard's output path on the host: the Fortran E edit
// descriptor, DumpParticles / DumpFields (Write.f90) and the plasma summary
// and warnings of WriteWarnings.f90.  Device state reaches the host through
// the reference-layout accessors (picard_gpu_get_particles / get_field).
#include <cuda_runtime.h>
#include <sys/stat.h>

#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "context.cuh"
#include "picard_gpu.h"
#include "picard_io.h"

using namespace picard;

namespace {

constexpr double kC0 = 2.99792458e8;  // WriteWarnings.f90:34

// The w characters of v under the Fortran edit descriptor Ew.d.
std::string format_e(double v, int w, int d) {
  std::string body;
  if (std::isnan(v)) {
    body = "NaN";
  } else if (std::isinf(v)) {
    body = w >= 9 ? (v < 0 ? "-Infinity" : "Infinity") : (v < 0 ? "-Inf" : "Inf");
  } else {
    const bool neg = std::signbit(v);
    const double a = std::fabs(v);
    std::string digits;
    int e10 = 0;
    if (a == 0.0) {
      digits.assign((size_t)d, '0');
    } else {
      // d significant digits, correctly rounded: x.xxxe+NN -> 0.xxxx * 10^(NN+1)
      char buf[96];
      std::snprintf(buf, sizeof buf, "%.*e", d - 1, a);
      const char* ep = std::strchr(buf, 'e');
      digits.push_back(buf[0]);
      if (d > 1) digits.append(buf + 2, (size_t)(d - 1));
      e10 = std::atoi(ep + 1) + 1;
    }
    char ex[16];
    const int ae = e10 < 0 ? -e10 : e10;
    if (ae <= 99)
      std::snprintf(ex, sizeof ex, "E%c%02d", e10 < 0 ? '-' : '+', ae);
    else if (ae <= 999)
      std::snprintf(ex, sizeof ex, "%c%03d", e10 < 0 ? '-' : '+', ae);
    else
      return std::string((size_t)w, '*');
    const std::string frac = "." + digits + ex;
    // the optional leading zero goes first when the width is short
    body = (neg ? "-" : "") + std::string("0") + frac;
    if ((int)body.size() > w) body = (neg ? "-" : "") + frac;
  }
  if ((int)body.size() > w) return std::string((size_t)w, '*');
  return std::string((size_t)(w - (int)body.size()), ' ') + body;
}

std::string i5(int v) {
  if (v < 0 || v > 99999) return "*****";
  char b[8];
  std::snprintf(b, sizeof b, "%05d", v);
  return b;
}

int make_dir(const std::string& path) {
  if (::mkdir(path.c_str(), 0777) == 0 || errno == EEXIST) return PICARD_OK;
  return fail(PICARD_ERR_BAD_ARG, "cannot create directory " + path);
}

// One E10.4 value per line (the fields files).
int write_column(const std::string& path, const double* v, long long n, long long stride) {
  FILE* f = std::fopen(path.c_str(), "w");
  if (!f) return fail(PICARD_ERR_BAD_ARG, "cannot open " + path);
  std::string buf;
  buf.reserve(1 << 20);
  for (long long g = 0; g < n; ++g) {
    buf += format_e(v[g * stride], 10, 4);
    buf += '\n';
    if (buf.size() > (1u << 20)) {
      std::fwrite(buf.data(), 1, buf.size(), f);
      buf.clear();
    }
  }
  std::fwrite(buf.data(), 1, buf.size(), f);
  const bool ok = std::fclose(f) == 0;
  return ok ? PICARD_OK : fail(PICARD_ERR_BAD_ARG, "write failed: " + path);
}

double max_nonnan(const double* v, int n) {
  double m = std::nan("");
  for (int k = 0; k < n; ++k)
    if (!std::isnan(v[k]) && (std::isnan(m) || v[k] > m)) m = v[k];
  return m;
}

const char* const kWarnText[PICARD_WARN_COUNT] = {
    "wp_e > 1/dt", "wp_i > 1/dt", "wc_e > 1/dt", "wc_i > 1/dt", "va > dx/dt",  "v_e > dx/dt",
    "v_i > dx/dt", "Ld_e < dx",   "Ld_i < dx",   "rL_e < dx",   "rL_i < dx",   "rPU_e < dx",
    "rPU_i < dx",  "Li_e < dx",   "Li_i < dx",   "Not a regular grid!", "You are ionizing incorrectly!"};

}  // namespace

extern "C" {

int picard_format_e(double value, int32_t w, int32_t d, char* out) {
  if (!out || w < 1 || w > 64 || d < 1 || d >= w) return fail(PICARD_ERR_BAD_ARG, "bad E edit descriptor");
  const std::string s = format_e(value, w, d);
  std::memcpy(out, s.data(), s.size());
  out[s.size()] = '\0';
  return PICARD_OK;
}

// Write.f90:1-31
int picard_gpu_dump_particles(picard_ctx* c, const char* root, int32_t* write_iteration) {
  if (!c || !root || !write_iteration) return fail(PICARD_ERR_BAD_ARG, "NULL argument");
  int32_t n = 0;
  PICARD_TRY(picard_gpu_get_num_local(c, &n));
  std::vector<double> real((size_t)8 * (n > 0 ? n : 1));
  std::vector<int32_t> sp((size_t)(n > 0 ? n : 1));
  int32_t got = 0;
  PICARD_TRY(picard_gpu_get_particles(c, real.data(), sp.data(), n, &got));
  const std::string dir = std::string(root) + "/particles";
  PICARD_TRY(make_dir(root));
  PICARD_TRY(make_dir(dir));
  const std::string path = dir + "/particles_" + i5(*write_iteration) + "_" + i5(0);
  FILE* f = std::fopen(path.c_str(), "w");
  if (!f) return fail(PICARD_ERR_BAD_ARG, "cannot open " + path);
  std::string buf;
  buf.reserve(1 << 20);
  for (int32_t q = 0; q < got; ++q) {
    // real_particles(7, :) = dble(int_particles) (Write.f90:14), then 7E10.4
    for (int k = 0; k < 6; ++k) buf += format_e(real[(size_t)8 * q + k], 10, 4);
    buf += format_e((double)sp[(size_t)q], 10, 4);
    buf += '\n';
    if (buf.size() > (1u << 20)) {
      std::fwrite(buf.data(), 1, buf.size(), f);
      buf.clear();
    }
  }
  std::fwrite(buf.data(), 1, buf.size(), f);
  if (std::fclose(f) != 0) return fail(PICARD_ERR_BAD_ARG, "write failed: " + path);
  *write_iteration += 1;
  return PICARD_OK;
}

// Write.f90:34-523
int picard_gpu_dump_fields(picard_ctx* c, const char* root, int32_t* write_iteration) {
  if (!c || !root || !write_iteration) return fail(PICARD_ERR_BAD_ARG, "NULL argument");
  const int S = c->prm.species;
  const long long nn = c->K.nodes;
  std::vector<double> U((size_t)nn), E((size_t)3 * nn), N((size_t)S * nn), F((size_t)3 * S * nn, 0.0);
  PICARD_TRY(picard_gpu_get_field(c, PICARD_FIELD_U, U.data()));
  PICARD_TRY(picard_gpu_get_field(c, PICARD_FIELD_E, E.data()));
  PICARD_TRY(picard_gpu_get_field(c, PICARD_FIELD_N, N.data()));
  if (c->F) PICARD_TRY(picard_gpu_get_field(c, PICARD_FIELD_F, F.data()));  // zero before any GridifyAll
  const std::string dir = std::string(root) + "/fields";
  PICARD_TRY(make_dir(root));
  PICARD_TRY(make_dir(dir));
  const std::string tail = "_" + i5(*write_iteration) + "_" + i5(0);
  PICARD_TRY(write_column(dir + "/UE" + tail, U.data(), nn, 1));
  PICARD_TRY(write_column(dir + "/Ex" + tail, E.data() + 0, nn, 3));
  PICARD_TRY(write_column(dir + "/Ey" + tail, E.data() + 1, nn, 3));
  PICARD_TRY(write_column(dir + "/Ez" + tail, E.data() + 2, nn, 3));
  for (int s = 0; s < S; ++s)
    PICARD_TRY(write_column(dir + "/N" + std::to_string(s + 1) + tail, N.data() + s, nn, S));
  // F(species, 3, i, j, k): flux component d of species s at node g is F[s + S (d + 3 g)]
  const char* comp[3] = {"X", "Y", "Z"};
  for (int d = 0; d < 3; ++d)
    for (int s = 0; s < S; ++s)
      PICARD_TRY(write_column(dir + "/" + comp[d] + std::to_string(s + 1) + tail, F.data() + s + (long long)S * d, nn,
                              3LL * S));
  *write_iteration += 1;
  return PICARD_OK;
}

// WriteWarnings.f90:40-115 and the tests of 261-496
int picard_params_plasma(const picard_params* p, picard_plasma* o) {
  if (!p || !o) return fail(PICARD_ERR_BAD_ARG, "NULL argument");
  if (!(p->dt > 0.0)) return fail(PICARD_ERR_BAD_ARG, "dt must be positive");
  std::memset(o, 0, sizeof(*o));
  for (int s = 0; s < 8; ++s) o->vth[s] = std::sqrt(2.0 * kKb * p->kelvin[s] / (p->mass[s] + 1.0e-99));
  o->freq = 1.0 / p->dt;
  double t[7];
  o->wp[0] = std::sqrt(p->density[0] * p->charge[0] * p->charge[0] / p->mass[0] / kEps0);
  for (int s = 1; s < 8; ++s) t[s - 1] = std::sqrt(p->density[s] * p->charge[s] * p->charge[s] / p->mass[s] / kEps0);
  o->wp[1] = max_nonnan(t, 7);
  o->wp[2] = std::sqrt(p->density[0] * kEc * kEc / kMe / kEps0);
  o->wc[0] = std::fabs(p->charge[0]) * p->B0[3] / p->mass[0];
  for (int s = 1; s < 8; ++s) t[s - 1] = std::fabs(p->charge[s]) * p->B0[3] / p->mass[s];
  o->wc[1] = max_nonnan(t, 7);
  o->wc[2] = kEc * p->B0[3] / kMe;
  double md = 0.0;
  for (int s = 0; s < 8; ++s) md += p->mass[s] * p->density[s];
  o->va = p->B0[3] / std::sqrt(kMu0 * md);
  o->vc[0] = o->vth[0] * std::sqrt(0.5);
  for (int s = 1; s < 8; ++s) t[s - 1] = o->vth[s] * std::sqrt(0.5);
  o->vc[1] = max_nonnan(t, 7);
  o->vc[2] = o->vth[0] * std::sqrt(0.5 * p->mass[0] / kMe);
  if (!p->gyration[0]) o->wc[0] = o->wc[1];
  for (int k = 0; k < 3; ++k) {
    o->Ld[k] = o->vc[k] / o->wp[k];
    o->rL[k] = o->vc[k] / o->wc[k];
    o->rPU[k] = p->v0[0][3] / o->wc[k];
    o->Li[k] = o->va / o->wc[k];
    o->rM[k] = o->va / o->wp[k];
  }
  o->sd = kC0 / o->wp[0];
  const double dx = p->dxyz[0];
  o->cfl = dx / p->dt;
  o->dt_c = 1.0 / std::sqrt(3.0) * dx / kC0;
  o->dt_opt_part = 1.0 / std::sqrt(3.0) * dx /
                   (std::fmax(2.0 * p->v0[0][3], 2.0 * p->v0[1][3]) +
                    std::sqrt(12.0 / kTau) * std::fmax(o->vc[0], o->vc[1]));
  o->dt_opt_wave = kTau / std::sqrt(12.0) / std::fmax(std::fmax(o->wc[0], o->wc[1]), std::fmax(o->wp[0], o->wp[1]));
  o->dt_opt = std::fmax(std::fmin(o->dt_opt_part, o->dt_opt_wave), o->dt_c);
  o->dt_rec = o->dt_opt * 0.75;
  uint32_t m = 0;
  auto set = [&](bool c, int k) {
    if (c) m |= 1u << k;
  };
  set(o->wp[0] > o->freq, PICARD_WARN_WP_E);
  set(o->wp[1] > o->freq, PICARD_WARN_WP_I);
  set(o->wc[0] > o->freq, PICARD_WARN_WC_E);
  set(o->wc[1] > o->freq, PICARD_WARN_WC_I);
  set(o->va > o->cfl, PICARD_WARN_VA);
  set(p->v0[0][3] + o->vth[0] > o->cfl, PICARD_WARN_V_E);
  set(p->v0[1][3] + o->vth[1] > o->cfl, PICARD_WARN_V_I);
  set(o->Ld[0] < dx, PICARD_WARN_LD_E);
  set(o->Ld[1] < dx, PICARD_WARN_LD_I);
  set(o->rL[0] < dx, PICARD_WARN_RL_E);
  set(o->rL[1] < dx, PICARD_WARN_RL_I);
  set(o->rPU[0] < dx, PICARD_WARN_RPU_E);
  set(o->rPU[1] < dx, PICARD_WARN_RPU_I);
  set(o->Li[0] < dx, PICARD_WARN_LI_E);
  set(o->Li[1] < dx, PICARD_WARN_LI_I);
  set(p->dxyz[0] != p->dxyz[1] || p->dxyz[1] != p->dxyz[2], PICARD_WARN_IRREGULAR);
  double qp = 0.0;
  for (int s = 0; s < 8; ++s) qp += p->Qn[s] * (double)p->ppc[s];
  set(qp > 0.0, PICARD_WARN_IONIZING);
  o->warnings = m;
  return PICARD_OK;
}

const char* picard_warning_text(int32_t k) { return k >= 0 && k < PICARD_WARN_COUNT ? kWarnText[k] : nullptr; }

// WriteWarnings.f90:129-255 (parameters.dat) and 258-496 (warnings.dat)
int picard_write_parameters(const picard_params* p, const char* root, uint32_t* warnings) {
  if (!p || !root) return fail(PICARD_ERR_BAD_ARG, "NULL argument");
  picard_plasma q;
  PICARD_TRY(picard_params_plasma(p, &q));
  PICARD_TRY(make_dir(root));
  const std::string dir(root);
  std::string s;
  auto e12 = [&](const std::string& name, double v) { s += name + " = " + format_e(v, 12, 6) + "\n"; };
  auto arr = [&](const char* name, const double* v) {
    for (int k = 0; k < 8; ++k) e12(std::string(name) + "_" + std::to_string(k + 1), v[k]);
  };
  auto i4 = [&](const char* name, int v) {
    char b[16];
    std::snprintf(b, sizeof b, "%4d", v);
    s += std::string(name) + " = " + (v > 9999 || v < -999 ? "****" : b) + "\n";
  };
  arr("n2p", p->n2p);
  arr("mass", p->mass);
  arr("charge", p->charge);
  arr("density", p->density);
  arr("kelvin", p->kelvin);
  arr("Qn", p->Qn);
  arr("vn", p->vn);
  arr("Ek", p->Ek);
  arr("nui", p->nu_i);
  arr("nud", p->nu_d);
  for (int k = 0; k < 8; ++k) {
    const std::string name = "ppc_" + std::to_string(k + 1);
    i4(name.c_str(), p->ppc[k]);
  }
  // list-directed logical (the plot scripts read T/F)
  for (int k = 0; k < 8; ++k) s += " gyration_" + std::to_string(k + 1) + " = " + (p->gyration[k] ? " T" : " F") + "\n";
  // the reference writes ve under the name v0 (WriteWarnings.f90:230-232)
  for (int k = 0; k < 3; ++k) e12("v0_" + std::to_string(k + 1), p->ve[k]);
  for (int k = 0; k < 3; ++k) e12("B0_" + std::to_string(k + 1), p->B0[k]);
  for (int k = 0; k < 3; ++k) e12("dxyz_" + std::to_string(k + 1), p->dxyz[k]);
  e12("xmin", p->xmin);
  e12("xmax", p->xmax);
  e12("ymin", p->ymin);
  e12("ymax", p->ymax);
  e12("zmin", p->zmin);
  e12("zmax", p->zmax);
  e12("dt", p->dt);
  i4("Nx", p->nx);
  i4("Ny", p->ny);
  i4("Nz", p->nz);
  i4("iprocs", 1);
  i4("jprocs", 1);
  i4("kprocs", 1);
  s += std::string(" xflow = ") + (p->xflow ? "T" : "F") + "\n";
  s += std::string(" yflow = ") + (p->yflow ? "T" : "F") + "\n";
  s += std::string(" zflow = ") + (p->zflow ? "T" : "F") + "\n";
  FILE* f = std::fopen((dir + "/parameters.dat").c_str(), "w");
  if (!f) return fail(PICARD_ERR_BAD_ARG, "cannot open " + dir + "/parameters.dat");
  std::fwrite(s.data(), 1, s.size(), f);
  std::fclose(f);
  // warnings.dat: one block per warning with the compared values
  const std::string bar = " ****************************************************************\n";
  std::string w;
  auto g = [](double v) {
    char b[40];
    std::snprintf(b, sizeof b, "%25.17E", v);
    return std::string(b);
  };
  const double vals[PICARD_WARN_COUNT][3] = {
      {q.wp[0], q.freq, NAN},        {q.wp[1], q.freq, NAN},        {q.wc[0], q.freq, NAN},
      {q.wc[1], q.freq, NAN},        {q.va, q.cfl, NAN},            {p->v0[0][3], q.vth[0], q.cfl},
      {p->v0[1][3], q.vth[1], q.cfl}, {q.Ld[0], p->dxyz[0], NAN},   {q.Ld[1], p->dxyz[0], NAN},
      {q.rL[0], p->dxyz[0], NAN},    {q.rL[1], p->dxyz[0], NAN},    {q.rPU[0], p->dxyz[0], NAN},
      {q.rPU[1], p->dxyz[0], NAN},   {q.Li[0], p->dxyz[0], NAN},    {q.Li[1], p->dxyz[0], NAN},
      {p->dxyz[0], p->dxyz[1], p->dxyz[2]}, {NAN, NAN, NAN}};
  for (int k = 0; k < PICARD_WARN_COUNT; ++k) {
    if (!(q.warnings >> k & 1u)) continue;
    w += "  \n" + bar + " " + kWarnText[k] + "\n";
    if (k == PICARD_WARN_IONIZING) {
      w += " Qn=";
      for (int s2 = 0; s2 < 8; ++s2) w += g(p->Qn[s2]);
      w += "  ppc";
      for (int s2 = 0; s2 < 8; ++s2) w += " " + std::to_string(p->ppc[s2]);
      w += "\n";
    } else if (k == PICARD_WARN_IRREGULAR) {
      w += " dx=" + g(vals[k][0]) + " dy=" + g(vals[k][1]) + " dz=" + g(vals[k][2]) + "\n";
    } else {
      for (int v = 0; v < 3 && !std::isnan(vals[k][v]); ++v) w += g(vals[k][v]);
      w += "\n";
    }
    w += bar;
  }
  f = std::fopen((dir + "/warnings.dat").c_str(), "w");
  if (!f) return fail(PICARD_ERR_BAD_ARG, "cannot open " + dir + "/warnings.dat");
  std::fwrite(w.data(), 1, w.size(), f);
  std::fclose(f);
  if (warnings) *warnings = q.warnings;
  return PICARD_OK;
}

}  // extern "C"
