// f90.cu -- the reference's subroutine signatures (include/picard_f90.h) over
// the device state of one attached context.
//
// Each entry point checks its scalar arguments against the context, runs the
// matching picard_gpu_* routine, and writes num_local back where the
// reference's routine changes it.  The host arrays in the argument lists are
// not touched: the device copy is authoritative until the host asks for it.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <mutex>
#include <string>

#include "context.cuh"
#include "picard_f90.h"
#include "picard_gpu.h"
#include "picard_io.h"

namespace {

std::mutex g_mu;
picard_ctx* g_ctx = nullptr;
int32_t g_iteration = 0;  // the iteration BCinflow last started
int g_status = PICARD_OK;
std::string g_message;    // message of the first recorded failure
std::string g_reported;   // message of the status last returned by picard_f90_status
int g_abort = 0;
std::string g_root = "save";

bool close_to(double a, double b) {
  if (a == b) return true;
  const double m = std::fmax(std::fabs(a), std::fabs(b));
  return std::fabs(a - b) <= 1e-12 * m;
}

// One subroutine call: the attached context, the first argument that does not
// match it, and the recording of the outcome.
struct Call {
  const char* name;
  picard_ctx* c;
  const picard_params* p = nullptr;
  std::string err;

  explicit Call(const char* n) : name(n) {
    std::lock_guard<std::mutex> lk(g_mu);
    c = g_ctx;
    if (!c)
      err = "no context attached (picard_f90_attach)";
    else
      p = &c->prm;
  }
  bool ok() const { return err.empty(); }
  bool null(const char* arg, const void* v) {
    if (ok() && !v) err = std::string(arg) + " is NULL";
    return !ok();
  }
  void i(const char* arg, const int32_t* v, long long want) {
    if (null(arg, v)) return;
    if (*v != want) err = std::string(arg) + " = " + std::to_string(*v) + ", the context has " + std::to_string(want);
  }
  void ia(const char* arg, const int32_t* v, const int32_t* want, int n) {
    if (null(arg, v)) return;
    for (int k = 0; k < n && ok(); ++k)
      if (v[k] != want[k])
        err = std::string(arg) + "(" + std::to_string(k + 1) + ") = " + std::to_string(v[k]) + ", the context has " +
              std::to_string(want[k]);
  }
  void l(const char* arg, const picard_f90_logical* v, int want) {
    if (null(arg, v)) return;
    if ((*v != 0) != (want != 0))
      err = std::string(arg) + " = " + (*v ? ".true." : ".false.") + ", the context has " +
            (want ? ".true." : ".false.");
  }
  void la(const char* arg, const picard_f90_logical* v, const int32_t* want, int n) {
    if (null(arg, v)) return;
    for (int k = 0; k < n && ok(); ++k)
      if ((v[k] != 0) != (want[k] != 0)) err = std::string(arg) + "(" + std::to_string(k + 1) + ") differs from the context";
  }
  void d(const char* arg, const double* v, double want) {
    if (null(arg, v)) return;
    if (!close_to(*v, want)) {
      char b[160];
      std::snprintf(b, sizeof b, "%s = %.17g, the context has %.17g", arg, *v, want);
      err = b;
    }
  }
  void da(const char* arg, const double* v, const double* want, int n) {
    if (null(arg, v)) return;
    for (int k = 0; k < n && ok(); ++k)
      if (!close_to(v[k], want[k])) {
        char b[160];
        std::snprintf(b, sizeof b, "%s(%d) = %.17g, the context has %.17g", arg, k + 1, v[k], want[k]);
        err = b;
      }
  }
  // argument groups that recur in the reference's signatures
  void grid_local(const int32_t* nx, const int32_t* ny, const int32_t* nz) {
    if (!ok()) return;
    i("Nx_local", nx, p->nx);
    i("Ny_local", ny, p->ny);
    i("Nz_local", nz, p->nz);
  }
  void flows(const picard_f90_logical* x, const picard_f90_logical* y, const picard_f90_logical* z) {
    if (!ok()) return;
    l("xflow", x, p->xflow);
    l("yflow", y, p->yflow);
    l("zflow", z, p->zflow);
  }
  void ranks(const int32_t* ip, const int32_t* jp, const int32_t* kp, const int32_t* myid) {
    if (!ok()) return;
    i("iprocs", ip, 1);
    i("jprocs", jp, 1);
    i("kprocs", kp, 1);
    i("myid", myid, 0);
  }
  void local_min(const double* x, const double* y, const double* z) {
    if (!ok()) return;
    d("Lx_min", x, p->Lx_min);
    d("Ly_min", y, p->Ly_min);
    d("Lz_min", z, p->Lz_min);
  }
  void local_max(const double* x, const double* y, const double* z) {
    if (!ok()) return;
    d("Lx_max", x, p->Lx_max);
    d("Ly_max", y, p->Ly_max);
    d("Lz_max", z, p->Lz_max);
  }
  void domain(const double* x0, const double* x1, const double* y0, const double* y1, const double* z0,
              const double* z1) {
    if (!ok()) return;
    d("xmin", x0, p->xmin);
    d("xmax", x1, p->xmax);
    d("ymin", y0, p->ymin);
    d("ymax", y1, p->ymax);
    d("zmin", z0, p->zmin);
    d("zmax", z1, p->zmax);
  }
  void cells(const double* dxyz) { da("dxyz", dxyz, p->dxyz, 3); }
  void counts(const int32_t* ppc, const int32_t* epp, const int32_t* hpp, const int32_t* ipp) {
    if (!ok()) return;
    ia("ppc", ppc, p->ppc, 8);
    ia("epp", epp, p->epp, 8);
    ia("hpp", hpp, p->hpp, 8);
    ia("ipp", ipp, p->ipp, 8);
  }
  void capacity(const int32_t* max_per_proc) { i("max_per_proc", max_per_proc, p->max_per_proc); }
  // num_local passed in must equal the device count (the host's copy of the
  // count has not diverged from the device's)
  void count_in(const int32_t* num_local) {
    if (!ok() || null("num_local", num_local)) return;
    int32_t n = 0;
    if (picard_gpu_get_num_local(c, &n) != PICARD_OK) {
      err = picard_gpu_last_error();
      return;
    }
    i("num_local", num_local, n);
  }
  void count_out(int32_t* num_local) {
    if (!num_local || !c) return;
    int32_t n = 0;
    if (picard_gpu_get_num_local(c, &n) == PICARD_OK) *num_local = n;
  }
  // Records the outcome: an argument mismatch (PICARD_ERR_BAD_ARG) or the
  // status of the routine that ran.
  void finish(int rc) {
    std::string msg;
    if (!ok()) {
      rc = PICARD_ERR_BAD_ARG;
      msg = std::string(name) + ": " + err;
    } else if (rc != PICARD_OK) {
      msg = std::string(name) + ": " + picard_gpu_last_error();
    }
    if (rc == PICARD_OK) return;
    std::fprintf(stderr, "picard_f90: %s\n", msg.c_str());
    int abort_now = 0;
    {
      std::lock_guard<std::mutex> lk(g_mu);
      if (g_status == PICARD_OK) {
        g_status = rc;
        g_message = msg;
      }
      abort_now = g_abort;
    }
    if (abort_now) std::abort();
  }
};

}  // namespace

extern "C" {

// ------------------------------------------------------------ registration

int picard_f90_attach(picard_ctx* ctx) {
  if (!ctx) return picard::fail(PICARD_ERR_BAD_ARG, "ctx is NULL");
  std::lock_guard<std::mutex> lk(g_mu);
  g_ctx = ctx;
  g_iteration = 0;
  g_status = PICARD_OK;
  g_message.clear();
  return PICARD_OK;
}

int picard_f90_detach(void) {
  std::lock_guard<std::mutex> lk(g_mu);
  g_ctx = nullptr;
  return PICARD_OK;
}

int picard_f90_set_iteration(int32_t iteration) {
  if (iteration < 0) return picard::fail(PICARD_ERR_BAD_ARG, "iteration must be >= 0");
  std::lock_guard<std::mutex> lk(g_mu);
  g_iteration = iteration;
  return PICARD_OK;
}

int picard_f90_status(void) {
  std::lock_guard<std::mutex> lk(g_mu);
  const int s = g_status;
  g_reported = g_message;
  g_status = PICARD_OK;
  g_message.clear();
  return s;
}

const char* picard_f90_status_message(void) { return g_reported.c_str(); }

int picard_f90_set_abort(int32_t on) {
  std::lock_guard<std::mutex> lk(g_mu);
  g_abort = on != 0;
  return PICARD_OK;
}

int picard_f90_set_dump_root(const char* root) {
  if (!root || !*root) return picard::fail(PICARD_ERR_BAD_ARG, "dump root is empty");
  std::lock_guard<std::mutex> lk(g_mu);
  g_root = root;
  return PICARD_OK;
}

// ----------------------------------------------- host copies of the state

int picard_f90_get_particles(double* real_particles, int32_t* int_particles, const int32_t* max_per_proc,
                             int32_t* num_local) {
  Call k("picard_f90_get_particles");
  if (!k.ok()) return picard::fail(PICARD_ERR_STATE, k.err);
  if (!max_per_proc || !num_local) return picard::fail(PICARD_ERR_BAD_ARG, "NULL argument");
  return picard_gpu_get_particles(k.c, real_particles, int_particles, *max_per_proc, num_local);
}

int picard_f90_set_particles(const double* real_particles, const int32_t* int_particles, const int32_t* num_local) {
  Call k("picard_f90_set_particles");
  if (!k.ok()) return picard::fail(PICARD_ERR_STATE, k.err);
  if (!num_local) return picard::fail(PICARD_ERR_BAD_ARG, "num_local is NULL");
  return picard_gpu_set_particles(k.c, real_particles, int_particles, *num_local);
}

int picard_f90_get_fields(double* U, double* E, double* N, double* C) {
  Call k("picard_f90_get_fields");
  if (!k.ok()) return picard::fail(PICARD_ERR_STATE, k.err);
  if (U) PICARD_TRY(picard_gpu_get_field(k.c, PICARD_FIELD_U, U));
  if (E) PICARD_TRY(picard_gpu_get_field(k.c, PICARD_FIELD_E, E));
  if (N) PICARD_TRY(picard_gpu_get_field(k.c, PICARD_FIELD_N, N));
  if (C) PICARD_TRY(picard_gpu_get_field(k.c, PICARD_FIELD_C, C));
  return PICARD_OK;
}

int picard_f90_energy(double* uP, double* uE, double* uB, int32_t* num_local) {
  Call k("picard_f90_energy");
  if (!k.ok()) return picard::fail(PICARD_ERR_STATE, k.err);
  double e[3];
  int32_t n = 0;
  PICARD_TRY(picard_gpu_energy(k.c, e, &n));
  if (uP) *uP = e[0];
  if (uE) *uE = e[1];
  if (uB) *uB = e[2];
  if (num_local) *num_local = n;
  return PICARD_OK;
}

// ------------------------------------------- the reference's subroutines

void picard_f90_calc_distance(double* D, const int32_t* Nx, const int32_t* Ny, const int32_t* Nz, const double* dxyz,
                              const picard_f90_logical* xflow, const picard_f90_logical* yflow,
                              const picard_f90_logical* zflow) {
  (void)D;
  Call k("CalcDistance");
  if (k.ok()) {
    k.i("Nx", Nx, k.p->nx);
    k.i("Ny", Ny, k.p->ny);
    k.i("Nz", Nz, k.p->nz);
    k.cells(dxyz);
    k.flows(xflow, yflow, zflow);
  }
  k.finish(k.ok() ? picard_gpu_calc_distance(k.c) : PICARD_ERR_BAD_ARG);
}

void picard_f90_particles_initialize(double* real_particles, int32_t* int_particles, const double* Lx_min,
                                     const double* Ly_min, const double* Lz_min, const double* dxyz,
                                     const double* kelvin, const double* mass, const double* v0, const double* ve,
                                     const double* tB, const int32_t* max_per_proc, int32_t* num_local,
                                     const int32_t* ppc, const int32_t* epp, const int32_t* hpp, const int32_t* ipp,
                                     const int32_t* species, const int32_t* Nx_local, const int32_t* Ny_local,
                                     const int32_t* Nz_local) {
  (void)real_particles, (void)int_particles;
  Call k("ParticlesInitialize");
  if (k.ok()) {
    k.local_min(Lx_min, Ly_min, Lz_min);
    k.cells(dxyz);
    k.da("kelvin", kelvin, k.p->kelvin, 8);
    k.da("mass", mass, k.p->mass, 8);
    k.da("v0", v0, &k.p->v0[0][0], 32);
    k.da("ve", ve, k.p->ve, 4);
    k.da("tB", tB, &k.p->tB[0][0], 32);
    k.capacity(max_per_proc);
    k.null("num_local", num_local);
    k.counts(ppc, epp, hpp, ipp);
    k.i("species", species, k.p->species);
    k.grid_local(Nx_local, Ny_local, Nz_local);
  }
  // the reference appends to num_local (ParticlesInitialize.f90:54-119); the
  // device starts from its own count, which must match
  k.count_in(num_local);
  k.finish(k.ok() ? picard_gpu_particles_initialize(k.c) : PICARD_ERR_BAD_ARG);
  k.count_out(num_local);
}

void picard_f90_bc_inflow(double* real_particles, int32_t* int_particles, const double* Lx_min, const double* Ly_min,
                          const double* Lz_min, const double* Lx_max, const double* Ly_max, const double* Lz_max,
                          const double* dxyz, const double* kelvin, const double* mass, const double* v0,
                          const double* ve, const int32_t* max_per_proc, int32_t* num_local, const int32_t* ppc,
                          const int32_t* epp, const int32_t* hpp, const int32_t* ipp, const int32_t* species,
                          const int32_t* Nx_local, const int32_t* Ny_local, const int32_t* Nz_local,
                          const double* xmin, const double* xmax, const double* ymin, const double* ymax,
                          const double* zmin, const double* zmax, const double* tB, const picard_f90_logical* xflow,
                          const picard_f90_logical* yflow, const picard_f90_logical* zflow) {
  (void)real_particles, (void)int_particles;
  Call k("BCinflow");
  if (k.ok()) {
    k.local_min(Lx_min, Ly_min, Lz_min);
    k.local_max(Lx_max, Ly_max, Lz_max);
    k.cells(dxyz);
    k.da("kelvin", kelvin, k.p->kelvin, 8);
    k.da("mass", mass, k.p->mass, 8);
    k.da("v0", v0, &k.p->v0[0][0], 32);
    k.da("ve", ve, k.p->ve, 4);
    k.capacity(max_per_proc);
    k.counts(ppc, epp, hpp, ipp);
    k.i("species", species, k.p->species);
    k.grid_local(Nx_local, Ny_local, Nz_local);
    k.domain(xmin, xmax, ymin, ymax, zmin, zmax);
    k.da("tB", tB, &k.p->tB[0][0], 32);
    k.flows(xflow, yflow, zflow);
  }
  k.count_in(num_local);
  int32_t it = 0;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    if (k.ok()) g_iteration += 1;  // BCinflow opens the next iteration
    it = g_iteration;
  }
  k.finish(k.ok() ? picard_gpu_bc_inflow(k.c, it) : PICARD_ERR_BAD_ARG);
  k.count_out(num_local);
}

void picard_f90_advance_position(double* real_particles, const double* dt, const int32_t* max_per_proc,
                                 const int32_t* num_local) {
  (void)real_particles;
  Call k("AdvancePosition");
  if (k.ok()) {
    k.null("dt", dt);
    k.capacity(max_per_proc);
  }
  k.count_in(num_local);
  k.finish(k.ok() ? picard_gpu_advance_position(k.c, *dt) : PICARD_ERR_BAD_ARG);
}

void picard_f90_particles_produce(double* real_particles, int32_t* int_particles, const double* Lx_min,
                                  const double* Ly_min, const double* Lz_min, const double* dxyz, const double* kelvin,
                                  const double* mass, const double* nu_d, const double* nu_i, const double* Ek,
                                  const double* Qn, const double* vn, const double* v0, const double* ve,
                                  const int32_t* max_per_proc, int32_t* num_local, const int32_t* ppc,
                                  const int32_t* epp, const int32_t* hpp, const int32_t* ipp, const int32_t* species,
                                  const int32_t* Nx_local, const int32_t* Ny_local, const int32_t* Nz_local,
                                  const double* dt, const double* n2p) {
  (void)real_particles, (void)int_particles;
  Call k("ParticlesProduce");
  if (k.ok()) {
    k.local_min(Lx_min, Ly_min, Lz_min);
    k.cells(dxyz);
    k.da("kelvin", kelvin, k.p->kelvin, 8);
    k.da("mass", mass, k.p->mass, 8);
    k.da("nu_d", nu_d, k.p->nu_d, 8);
    k.da("nu_i", nu_i, k.p->nu_i, 8);
    k.da("Ek", Ek, k.p->Ek, 8);
    k.da("Qn", Qn, k.p->Qn, 8);
    k.da("vn", vn, k.p->vn, 8);
    k.da("v0", v0, &k.p->v0[0][0], 32);
    k.da("ve", ve, k.p->ve, 4);
    k.capacity(max_per_proc);
    k.counts(ppc, epp, hpp, ipp);
    k.i("species", species, k.p->species);
    k.grid_local(Nx_local, Ny_local, Nz_local);
    k.d("dt", dt, k.p->dt);
    k.da("n2p", n2p, k.p->n2p, 8);
  }
  k.count_in(num_local);
  int32_t it = 0;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    it = g_iteration;
  }
  if (k.ok() && it < 1) k.err = "no iteration started (ParticlesProduce follows BCinflow; see picard_f90_set_iteration)";
  k.finish(k.ok() ? picard_gpu_particles_produce(k.c, it) : PICARD_ERR_BAD_ARG);
  k.count_out(num_local);
}

void picard_f90_bc_outflow(double* real_particles, int32_t* int_particles, const double* Lx_min, const double* Lx_max,
                           const double* Ly_min, const double* Ly_max, const double* Lz_min, const double* Lz_max,
                           const double* xmin, const double* xmax, const double* ymin, const double* ymax,
                           const double* zmin, const double* zmax, const int32_t* max_per_proc, int32_t* num_local,
                           const picard_f90_logical* xflow, const picard_f90_logical* yflow,
                           const picard_f90_logical* zflow) {
  (void)real_particles, (void)int_particles;
  Call k("BCoutflow");
  if (k.ok()) {
    k.local_min(Lx_min, Ly_min, Lz_min);
    k.local_max(Lx_max, Ly_max, Lz_max);
    k.domain(xmin, xmax, ymin, ymax, zmin, zmax);
    k.capacity(max_per_proc);
    k.flows(xflow, yflow, zflow);
  }
  k.count_in(num_local);
  k.finish(k.ok() ? picard_gpu_bc_outflow(k.c) : PICARD_ERR_BAD_ARG);
  k.count_out(num_local);
}

void picard_f90_particles_transfer(double* real_particles, int32_t* int_particles, const double* Lx_min,
                                   const double* Lx_max, const double* Ly_min, const double* Ly_max,
                                   const double* Lz_min, const double* Lz_max, const double* xmin, const double* xmax,
                                   const double* ymin, const double* ymax, const double* zmin, const double* zmax,
                                   const int32_t* max_per_proc, int32_t* num_local, const int32_t* iprocs,
                                   const int32_t* jprocs, const int32_t* kprocs, const int32_t* myid) {
  (void)real_particles, (void)int_particles;
  Call k("ParticlesTransfer");
  if (k.ok()) {
    k.local_min(Lx_min, Ly_min, Lz_min);
    k.local_max(Lx_max, Ly_max, Lz_max);
    k.domain(xmin, xmax, ymin, ymax, zmin, zmax);
    k.capacity(max_per_proc);
    k.ranks(iprocs, jprocs, kprocs, myid);
  }
  k.count_in(num_local);
  k.finish(k.ok() ? picard_gpu_particles_transfer(k.c) : PICARD_ERR_BAD_ARG);
  k.count_out(num_local);
}

namespace {
// The arguments ParticlesGridify and ParticlesGridifyAll share.
void gridify_args(Call& k, const double* Lx_min, const double* Lx_max, const double* Ly_min, const double* Ly_max,
                  const double* Lz_min, const double* Lz_max, const double* dxyz, const double* xmin,
                  const double* xmax, const double* ymin, const double* ymax, const double* zmin, const double* zmax,
                  const int32_t* species, const int32_t* Nx_local, const int32_t* Ny_local, const int32_t* Nz_local,
                  const int32_t* max_per_proc, const int32_t* num_local, const picard_f90_logical* xflow,
                  const picard_f90_logical* yflow, const picard_f90_logical* zflow, const int32_t* iprocs,
                  const int32_t* jprocs, const int32_t* kprocs, const double* charge, const double* n2p,
                  const int32_t* myid) {
  if (k.ok()) {
    k.local_min(Lx_min, Ly_min, Lz_min);
    k.local_max(Lx_max, Ly_max, Lz_max);
    k.cells(dxyz);
    k.domain(xmin, xmax, ymin, ymax, zmin, zmax);
    k.i("species", species, k.p->species);
    k.grid_local(Nx_local, Ny_local, Nz_local);
    k.capacity(max_per_proc);
    k.flows(xflow, yflow, zflow);
    k.ranks(iprocs, jprocs, kprocs, myid);
    k.da("charge", charge, k.p->charge, 8);
    k.da("n2p", n2p, k.p->n2p, 8);
  }
  k.count_in(num_local);
}
}  // namespace

void picard_f90_particles_gridify(double* N, double* C, const double* real_particles, const int32_t* int_particles,
                                  const double* Lx_min, const double* Lx_max, const double* Ly_min,
                                  const double* Ly_max, const double* Lz_min, const double* Lz_max,
                                  const double* dxyz, const double* xmin, const double* xmax, const double* ymin,
                                  const double* ymax, const double* zmin, const double* zmax, const int32_t* species,
                                  const int32_t* Nx_local, const int32_t* Ny_local, const int32_t* Nz_local,
                                  const int32_t* max_per_proc, const int32_t* num_local,
                                  const picard_f90_logical* xflow, const picard_f90_logical* yflow,
                                  const picard_f90_logical* zflow, const int32_t* iprocs, const int32_t* jprocs,
                                  const int32_t* kprocs, const double* charge, const double* n2p,
                                  const int32_t* myid) {
  (void)N, (void)C, (void)real_particles, (void)int_particles;
  Call k("ParticlesGridify");
  gridify_args(k, Lx_min, Lx_max, Ly_min, Ly_max, Lz_min, Lz_max, dxyz, xmin, xmax, ymin, ymax, zmin, zmax, species,
               Nx_local, Ny_local, Nz_local, max_per_proc, num_local, xflow, yflow, zflow, iprocs, jprocs, kprocs,
               charge, n2p, myid);
  k.finish(k.ok() ? picard_gpu_particles_gridify(k.c) : PICARD_ERR_BAD_ARG);
}

void picard_f90_particles_gridify_all(double* F, double* N, double* C, const double* real_particles,
                                      const int32_t* int_particles, const double* Lx_min, const double* Lx_max,
                                      const double* Ly_min, const double* Ly_max, const double* Lz_min,
                                      const double* Lz_max, const double* dxyz, const double* xmin,
                                      const double* xmax, const double* ymin, const double* ymax, const double* zmin,
                                      const double* zmax, const int32_t* species, const int32_t* Nx_local,
                                      const int32_t* Ny_local, const int32_t* Nz_local, const int32_t* max_per_proc,
                                      const int32_t* num_local, const picard_f90_logical* xflow,
                                      const picard_f90_logical* yflow, const picard_f90_logical* zflow,
                                      const int32_t* iprocs, const int32_t* jprocs, const int32_t* kprocs,
                                      const double* charge, const double* n2p, const int32_t* myid) {
  (void)F, (void)N, (void)C, (void)real_particles, (void)int_particles;
  Call k("ParticlesGridifyAll");
  gridify_args(k, Lx_min, Lx_max, Ly_min, Ly_max, Lz_min, Lz_max, dxyz, xmin, xmax, ymin, ymax, zmin, zmax, species,
               Nx_local, Ny_local, Nz_local, max_per_proc, num_local, xflow, yflow, zflow, iprocs, jprocs, kprocs,
               charge, n2p, myid);
  k.finish(k.ok() ? picard_gpu_particles_gridify_all(k.c) : PICARD_ERR_BAD_ARG);
}

void picard_f90_bc_potentials(double* U, const double* C, const double* D, const double* xmin, const double* xmax,
                              const double* ymin, const double* ymax, const double* zmin, const double* zmax,
                              const int32_t* Nx_local, const int32_t* Ny_local, const int32_t* Nz_local,
                              const int32_t* Nx, const int32_t* Ny, const int32_t* Nz,
                              const picard_f90_logical* xflow, const picard_f90_logical* yflow,
                              const picard_f90_logical* zflow, const int32_t* species, const int32_t* iprocs,
                              const int32_t* jprocs, const int32_t* kprocs, const int32_t* myid) {
  (void)U, (void)C, (void)D;
  Call k("BCpotentials");
  if (k.ok()) {
    k.domain(xmin, xmax, ymin, ymax, zmin, zmax);
    k.grid_local(Nx_local, Ny_local, Nz_local);
    k.i("Nx", Nx, k.p->nx);
    k.i("Ny", Ny, k.p->ny);
    k.i("Nz", Nz, k.p->nz);
    k.flows(xflow, yflow, zflow);
    k.i("species", species, k.p->species);
    k.ranks(iprocs, jprocs, kprocs, myid);
  }
  k.finish(k.ok() ? picard_gpu_bc_potentials(k.c) : PICARD_ERR_BAD_ARG);
}

void picard_f90_calc_epotential(double* U, const double* C, const int32_t* Nx_local, const int32_t* Ny_local,
                                const int32_t* Nz_local, const double* Lx_min, const double* Lx_max,
                                const double* Ly_min, const double* Ly_max, const double* Lz_min,
                                const double* Lz_max, const picard_f90_logical* xflow,
                                const picard_f90_logical* yflow, const picard_f90_logical* zflow, const double* xmin,
                                const double* xmax, const double* ymin, const double* ymax, const double* zmin,
                                const double* zmax, const double* dxyz, const double* maxerr, const int32_t* maxit,
                                const int32_t* iprocs, const int32_t* jprocs, const int32_t* kprocs,
                                const int32_t* species, const int32_t* myid) {
  (void)U, (void)C;
  Call k("CalcEpotential");
  if (k.ok()) {
    k.grid_local(Nx_local, Ny_local, Nz_local);
    k.local_min(Lx_min, Ly_min, Lz_min);
    k.local_max(Lx_max, Ly_max, Lz_max);
    k.flows(xflow, yflow, zflow);
    k.domain(xmin, xmax, ymin, ymax, zmin, zmax);
    k.cells(dxyz);
    k.null("maxerr", maxerr);
    k.null("maxit", maxit);
    k.ranks(iprocs, jprocs, kprocs, myid);
    k.i("species", species, k.p->species);
  }
  int rc = PICARD_ERR_BAD_ARG;
  if (k.ok()) {
    int32_t sweeps = 0;
    rc = picard_gpu_calc_epotential(k.c, *maxerr, *maxit, &sweeps);
    if (rc == PICARD_ERR_NOT_CONVERGED) {
      // the reference prints this and carries on (CalcEpotential.f90:67-69)
      std::printf(" Maximum iteration reached!\n");
      std::fflush(stdout);
      rc = PICARD_OK;
    }
  }
  k.finish(rc);
}

void picard_f90_calc_efield(double* E, const double* U, const int32_t* Nx_local, const int32_t* Ny_local,
                            const int32_t* Nz_local, const double* dxyz, const picard_f90_logical* xflow,
                            const picard_f90_logical* yflow, const picard_f90_logical* zflow, const int32_t* iprocs,
                            const int32_t* jprocs, const int32_t* kprocs, const int32_t* myid) {
  (void)E, (void)U;
  Call k("CalcEfield");
  if (k.ok()) {
    k.grid_local(Nx_local, Ny_local, Nz_local);
    k.cells(dxyz);
    k.flows(xflow, yflow, zflow);
    k.ranks(iprocs, jprocs, kprocs, myid);
  }
  k.finish(k.ok() ? picard_gpu_calc_efield(k.c) : PICARD_ERR_BAD_ARG);
}

void picard_f90_bc_fields(double* E, const double* U, const double* B0, const double* E0, const int32_t* Nx_local,
                          const int32_t* Ny_local, const int32_t* Nz_local, const picard_f90_logical* xflow,
                          const picard_f90_logical* yflow, const picard_f90_logical* zflow, const int32_t* iprocs,
                          const int32_t* jprocs, const int32_t* kprocs, const int32_t* myid) {
  (void)E, (void)U;
  Call k("BCfields");
  if (k.ok()) {
    k.da("B0", B0, k.p->B0, 4);
    k.da("E0", E0, k.p->E0, 4);
    k.grid_local(Nx_local, Ny_local, Nz_local);
    k.flows(xflow, yflow, zflow);
    k.ranks(iprocs, jprocs, kprocs, myid);
  }
  k.finish(k.ok() ? picard_gpu_bc_fields(k.c) : PICARD_ERR_BAD_ARG);
}

namespace {
// The arguments the three AdvanceVelocity variants share.
void velocity_args(Call& k, const double* B0, const double* Lx_min, const double* Ly_min, const double* Lz_min,
                   const double* dxyz, const double* v0, const double* ve, const double* eta, const double* tB,
                   const int32_t* num_local, const int32_t* max_per_proc, const int32_t* species,
                   const int32_t* Nx_local, const int32_t* Ny_local, const int32_t* Nz_local,
                   const picard_f90_logical* fluid, const picard_f90_logical* gyration) {
  if (k.ok()) {
    k.da("B0", B0, k.p->B0, 4);
    k.local_min(Lx_min, Ly_min, Lz_min);
    k.cells(dxyz);
    k.da("v0", v0, &k.p->v0[0][0], 32);
    k.da("ve", ve, k.p->ve, 4);
    k.da("eta", eta, k.p->eta, 8);
    k.da("tB", tB, &k.p->tB[0][0], 32);
    k.capacity(max_per_proc);
    k.i("species", species, k.p->species);
    k.grid_local(Nx_local, Ny_local, Nz_local);
    k.la("fluid", fluid, k.p->fluid, 8);
    k.la("gyration", gyration, k.p->gyration, 8);
  }
  k.count_in(num_local);
}
}  // namespace

void picard_f90_advance_velocity(double* real_particles, const int32_t* int_particles, const double* E,
                                 const double* B0, const double* Lx_min, const double* Ly_min, const double* Lz_min,
                                 const double* dxyz, const double* dt, const double* v0, const double* ve,
                                 const double* eta, const double* tB, const double* sB, const int32_t* num_local,
                                 const int32_t* max_per_proc, const int32_t* species, const int32_t* Nx_local,
                                 const int32_t* Ny_local, const int32_t* Nz_local, const picard_f90_logical* fluid,
                                 const picard_f90_logical* gyration) {
  (void)real_particles, (void)int_particles, (void)E;
  Call k("AdvanceVelocity");
  velocity_args(k, B0, Lx_min, Ly_min, Lz_min, dxyz, v0, ve, eta, tB, num_local, max_per_proc, species, Nx_local,
                Ny_local, Nz_local, fluid, gyration);
  if (k.ok()) {
    k.da("sB", sB, &k.p->sB[0][0], 32);
    k.null("dt", dt);
  }
  k.finish(k.ok() ? picard_gpu_advance_velocity(k.c, *dt) : PICARD_ERR_BAD_ARG);
}

void picard_f90_advance_velocity_exp(double* real_particles, const int32_t* int_particles, const double* E,
                                     const double* B0, const double* Lx_min, const double* Ly_min,
                                     const double* Lz_min, const double* dxyz, const double* deltat, const double* dt,
                                     const double* v0, const double* ve, const double* eta, const double* tB,
                                     const int32_t* num_local, const int32_t* max_per_proc, const int32_t* species,
                                     const int32_t* Nx_local, const int32_t* Ny_local, const int32_t* Nz_local,
                                     const picard_f90_logical* fluid, const picard_f90_logical* gyration) {
  (void)real_particles, (void)int_particles, (void)E;
  Call k("AdvanceVelocityExp");
  velocity_args(k, B0, Lx_min, Ly_min, Lz_min, dxyz, v0, ve, eta, tB, num_local, max_per_proc, species, Nx_local,
                Ny_local, Nz_local, fluid, gyration);
  if (k.ok()) {
    k.null("deltat", deltat);
    k.null("dt", dt);
  }
  k.finish(k.ok() ? picard_gpu_advance_velocity_exp(k.c, *deltat, *dt) : PICARD_ERR_BAD_ARG);
}

void picard_f90_advance_velocity_imp(double* real_particles, const int32_t* int_particles, const double* E,
                                     const double* B0, const double* Lx_min, const double* Ly_min,
                                     const double* Lz_min, const double* dxyz, const double* deltat, const double* dt,
                                     const double* v0, const double* ve, const double* eta, const double* tB,
                                     const int32_t* num_local, const int32_t* max_per_proc, const int32_t* species,
                                     const int32_t* Nx_local, const int32_t* Ny_local, const int32_t* Nz_local,
                                     const picard_f90_logical* fluid, const picard_f90_logical* gyration) {
  (void)real_particles, (void)int_particles, (void)E;
  Call k("AdvanceVelocityImp");
  velocity_args(k, B0, Lx_min, Ly_min, Lz_min, dxyz, v0, ve, eta, tB, num_local, max_per_proc, species, Nx_local,
                Ny_local, Nz_local, fluid, gyration);
  if (k.ok()) {
    k.null("deltat", deltat);
    k.null("dt", dt);
  }
  k.finish(k.ok() ? picard_gpu_advance_velocity_imp(k.c, *deltat, *dt) : PICARD_ERR_BAD_ARG);
}

void picard_f90_dump_particles(double* real_particles, const int32_t* int_particles, const int32_t* num_local,
                               const int32_t* max_per_proc, int32_t* writeParticles_iteration, const int32_t* myid) {
  (void)real_particles, (void)int_particles;
  Call k("DumpParticles");
  if (k.ok()) {
    k.capacity(max_per_proc);
    k.null("writeParticles_iteration", writeParticles_iteration);
    k.i("myid", myid, 0);
  }
  k.count_in(num_local);
  std::string root;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    root = g_root;
  }
  k.finish(k.ok() ? picard_gpu_dump_particles(k.c, root.c_str(), writeParticles_iteration) : PICARD_ERR_BAD_ARG);
}

void picard_f90_dump_fields(const double* U, const double* N, const double* F, const double* E,
                            const int32_t* Nx_local, const int32_t* Ny_local, const int32_t* Nz_local,
                            int32_t* writeFields_iteration, const int32_t* species, const int32_t* myid) {
  (void)U, (void)N, (void)F, (void)E;
  Call k("DumpFields");
  if (k.ok()) {
    k.grid_local(Nx_local, Ny_local, Nz_local);
    k.null("writeFields_iteration", writeFields_iteration);
    k.i("species", species, k.p->species);
    k.i("myid", myid, 0);
  }
  std::string root;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    root = g_root;
  }
  k.finish(k.ok() ? picard_gpu_dump_fields(k.c, root.c_str(), writeFields_iteration) : PICARD_ERR_BAD_ARG);
}

}  // extern "C"
