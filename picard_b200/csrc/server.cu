// server.cu -- the request loop of the serving workload: runs admitted by HBM
// budget, state resident on the device for the whole run, concurrent runs
// overlapping on the device, latencies reported per run.
//
// Each admitted request becomes a picard_ctx on its own CUDA stream, driven by
// one worker thread: CalcDistance, ParticlesInitialize, `steps` iterations of
// the fused loop, the energy diagnostics, release.  A request is admitted when
// a worker is free and its device footprint (picard_gpu_footprint) fits in
// what the budget has left; requests are admitted in arrival order, so a
// large request waits for memory instead of being overtaken forever.  While a
// run waits on its own stream for the host (the Jacobi stop test), the
// kernels of the other runs keep the device busy -- that overlap is the
// continuous batching of the loop.  Context memory comes from the
// stream-ordered allocator, so admitting or retiring a run does not
// synchronise the device.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "context.cuh"
#include "picard_gpu.h"
#include "picard_io.h"
#include "picard_server.h"

using namespace picard;

struct picard_server {
  uint64_t budget = 0;
  uint64_t in_use = 0;
  int device = 0;
  int max_slots = 1;
  int running = 0;
  bool stopping = false;
  bool batched = false;  // continuous batching: one cohort advanced by picard_batch_step
  int shard = 0;         // index of this server among the shards of a multi-device server
  std::vector<picard_server*> shards;  // multi-device server: one server per device
  std::deque<std::pair<picard_request, uint64_t>> queue;  // request, footprint
  std::vector<picard_result> done;
  std::mutex mu;
  std::condition_variable cv_work;  // a worker may be able to start a request
  std::condition_variable cv_done;  // a request finished
  std::condition_variable cv_ready;  // batched mode: a prepared run can join the cohort
  std::vector<std::thread> workers;
  std::chrono::steady_clock::time_point t0;
  int64_t submitted = 0, finished = 0;
  // batched mode
  struct Prepared {
    picard_ctx* c;
    picard_request rq;
    uint64_t fp;
    picard_result r;
  };
  std::deque<std::pair<picard_request, uint64_t>> admitted;  // waiting for a preparer
  std::vector<Prepared> ready;                               // prepared, waiting for a step boundary
};

namespace {

double now_ms(const picard_server* s) {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - s->t0).count();
}

// Context creation, CalcDistance and ParticlesInitialize of a request.
int prepare_run(const picard_request& rq, picard_ctx** out) {
  picard_ctx* c = nullptr;
  PICARD_TRY(picard_gpu_create(&rq.params, rq.layout, rq.solver, &c));
  int rc = picard_gpu_calc_distance(c);
  if (rc == PICARD_OK) rc = picard_gpu_particles_initialize(c);
  if (rc == PICARD_OK) rc = check_cuda(cudaStreamSynchronize(c->st), "prepare");
  if (rc != PICARD_OK) {
    picard_gpu_destroy(c);
    return rc;
  }
  *out = c;
  return PICARD_OK;
}

// Energies, particle count and checksums of the final potential; releases the context.
int finish_run(picard_ctx* c, picard_result* out) {
  int rc = picard_gpu_energy(c, out->energy, &out->num_local);
  picard_stats st;
  if (rc == PICARD_OK) rc = picard_gpu_get_stats(c, &st);
  if (rc == PICARD_OK) {
    out->sweeps = st.sweeps;
    out->particle_steps = st.particle_steps;
    const long long nn = c->K.nodes;
    std::vector<double> h((size_t)nn);
    rc = check_cuda(cudaMemcpyAsync(h.data(), c->U, sizeof(double) * nn, cudaMemcpyDeviceToHost, c->st), "U");
    if (rc == PICARD_OK) rc = check_cuda(cudaStreamSynchronize(c->st), "sync");
    double sm = 0.0, ab = 0.0;
    for (long long g = 0; g < nn; ++g) sm += h[(size_t)g], ab += std::fabs(h[(size_t)g]);
    out->u_sum = sm;
    out->u_abs_sum = ab;
  }
  picard_gpu_destroy(c);
  return rc;
}

int run_request(const picard_request& rq, picard_result* out) {
  picard_ctx* c = nullptr;
  PICARD_TRY(prepare_run(rq, &c));
  int64_t sweeps = 0;
  int rc = picard_gpu_run_fused(c, 0, rq.steps, &sweeps);
  if (rc == PICARD_ERR_NOT_CONVERGED) rc = PICARD_OK;  // the reference carries on too
  if (rc != PICARD_OK) {
    picard_gpu_destroy(c);
    return rc;
  }
  return finish_run(c, out);
}

// WriteWarnings.f90's mask of a request's parameters (0 if it cannot be formed).
uint32_t request_warnings(const picard_request& rq) {
  picard_plasma q;
  return picard_params_plasma(&rq.params, &q) == PICARD_OK ? q.warnings : 0u;
}

void worker_main(picard_server* s) {
  cudaSetDevice(s->device);
  for (;;) {
    std::pair<picard_request, uint64_t> job;
    {
      std::unique_lock<std::mutex> lk(s->mu);
      s->cv_work.wait(lk, [&] {
        if (s->stopping && s->queue.empty()) return true;
        return !s->queue.empty() && s->queue.front().second <= s->budget - s->in_use;
      });
      if (s->queue.empty()) return;
      job = s->queue.front();
      s->queue.pop_front();
      s->in_use += job.second;
      s->running += 1;
    }
    s->cv_work.notify_all();
    picard_result r;
    std::memset(&r, 0, sizeof(r));
    r.id = job.first.id;
    r.warnings = request_warnings(job.first);
    r.shard = s->shard;
    r.start_ms = now_ms(s);
    r.status = run_request(job.first, &r);
    r.finish_ms = now_ms(s);
    r.arrival_ms = job.first.arrival_ms;
    {
      std::lock_guard<std::mutex> lk(s->mu);
      s->in_use -= job.second;
      s->running -= 1;
      s->finished += 1;
      s->done.push_back(r);
    }
    s->cv_work.notify_all();
    s->cv_done.notify_all();
  }
}

// ------------------------------------------------ continuous batching
//
// Admission as in the stream mode (arrival order, slots and HBM budget).
// Admitted requests are prepared (context, CalcDistance, ParticlesInitialize)
// by preparer threads; a prepared run joins the cohort at the next step
// boundary.  The scheduler advances the whole cohort one iteration at a time
// with picard_batch_step -- all runs' Jacobi sweeps in one launch per tick --
// and retires each run after its last step.  A run's result is bit-identical
// to the same run alone: the batched step is.

// In this mode `running` counts the admitted runs that have not finished.
void admit_locked(picard_server* s) {
  while (s->running < s->max_slots && !s->queue.empty() && s->queue.front().second <= s->budget - s->in_use) {
    s->in_use += s->queue.front().second;
    s->running += 1;
    s->admitted.push_back(s->queue.front());
    s->queue.pop_front();
  }
}

void post_result(picard_server* s, const picard_result& r, uint64_t fp) {
  std::lock_guard<std::mutex> lk(s->mu);
  s->in_use -= fp;
  s->running -= 1;
  s->finished += 1;
  s->done.push_back(r);
  admit_locked(s);
  s->cv_work.notify_all();
  s->cv_done.notify_all();
}

void preparer_main(picard_server* s) {
  cudaSetDevice(s->device);
  for (;;) {
    std::pair<picard_request, uint64_t> job;
    {
      std::unique_lock<std::mutex> lk(s->mu);
      s->cv_work.wait(lk, [&] { return !s->admitted.empty() || (s->stopping && s->queue.empty()); });
      if (s->admitted.empty()) return;
      job = s->admitted.front();
      s->admitted.pop_front();
    }
    picard_result r;
    std::memset(&r, 0, sizeof(r));
    r.id = job.first.id;
    r.warnings = request_warnings(job.first);
    r.shard = s->shard;
    r.arrival_ms = job.first.arrival_ms;
    r.start_ms = now_ms(s);
    picard_ctx* c = nullptr;
    int rc = prepare_run(job.first, &c);
    if (rc != PICARD_OK) {
      r.status = rc;
      r.finish_ms = now_ms(s);
      post_result(s, r, job.second);
      continue;
    }
    {
      std::lock_guard<std::mutex> lk(s->mu);
      s->ready.push_back({c, job.first, job.second, r});
    }
    s->cv_ready.notify_all();
  }
}

void scheduler_main(picard_server* s) {
  cudaSetDevice(s->device);
  struct Active {
    picard_ctx* c;
    picard_request rq;
    uint64_t fp;
    picard_result r;
    int32_t iter;  // iterations done
  };
  std::vector<Active> act;
  for (;;) {
    {
      std::unique_lock<std::mutex> lk(s->mu);
      s->cv_ready.wait(lk, [&] {
        return !s->ready.empty() || !act.empty() ||
               (s->stopping && s->queue.empty() && s->running == 0);
      });
      for (auto& p : s->ready) act.push_back({p.c, p.rq, p.fp, p.r, 0});
      s->ready.clear();
      if (act.empty()) return;  // stopping and nothing left
    }
    std::vector<picard_ctx*> ctxs;
    std::vector<int32_t> its;
    for (auto& a : act) {
      ctxs.push_back(a.c);
      its.push_back(a.iter + 1);
    }
    int rc = picard_batch_step(ctxs.data(), int32_t(ctxs.size()), its.data(), nullptr);
    if (rc == PICARD_ERR_NOT_CONVERGED) rc = PICARD_OK;  // the reference carries on too
    std::vector<Active> keep;
    for (auto& a : act) {
      a.iter += 1;
      if (rc != PICARD_OK || a.iter >= a.rq.steps) {
        picard_result r = a.r;
        r.status = rc != PICARD_OK ? rc : finish_run(a.c, &r);
        if (rc != PICARD_OK) picard_gpu_destroy(a.c);
        r.finish_ms = now_ms(s);
        post_result(s, r, a.fp);
      } else {
        keep.push_back(a);
      }
    }
    act.swap(keep);
  }
}

// A server on `device` (its worker threads make it current), results timed
// from t0, reporting `shard` as the shard index.
picard_server* open_server(uint64_t budget, int slots, bool batched, int preparers, int device, int shard,
                           std::chrono::steady_clock::time_point t0) {
  picard_server* s = new picard_server();
  s->budget = budget;
  s->max_slots = slots;
  s->batched = batched;
  s->device = device;
  s->shard = shard;
  s->t0 = t0;
  // keep freed context memory in the pool between runs
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
    uint64_t keep = budget;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  if (batched) {
    for (int i = 0; i < preparers; ++i) s->workers.emplace_back(preparer_main, s);
    s->workers.emplace_back(scheduler_main, s);
  } else {
    for (int i = 0; i < slots; ++i) s->workers.emplace_back(worker_main, s);
  }
  return s;
}

// Footprint a shard holds or has queued, relative to its budget.
double shard_load(picard_server* s) {
  std::lock_guard<std::mutex> lk(s->mu);
  uint64_t q = s->in_use;
  for (const auto& e : s->queue) q += e.second;
  return (double)q / (double)s->budget;
}

}  // namespace

extern "C" {

int picard_server_create(uint64_t hbm_budget_bytes, int32_t max_slots, picard_server** out) {
  if (!out || max_slots < 1 || hbm_budget_bytes == 0) return fail(PICARD_ERR_BAD_ARG, "bad server arguments");
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return fail(PICARD_ERR_CUDA, "no CUDA device");
  *out = open_server(hbm_budget_bytes, max_slots, false, 0, dev, 0, std::chrono::steady_clock::now());
  return PICARD_OK;
}

int picard_server_create_batched(uint64_t hbm_budget_bytes, int32_t max_runs, int32_t preparers,
                                 picard_server** out) {
  if (!out || max_runs < 1 || preparers < 1 || hbm_budget_bytes == 0)
    return fail(PICARD_ERR_BAD_ARG, "bad server arguments");
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return fail(PICARD_ERR_CUDA, "no CUDA device");
  *out = open_server(hbm_budget_bytes, max_runs, true, preparers, dev, 0, std::chrono::steady_clock::now());
  return PICARD_OK;
}

int picard_server_create_multi(const int32_t* devices, int32_t ndev, uint64_t hbm_budget_per_device,
                               int32_t slots_per_device, int32_t batched, int32_t preparers, picard_server** out) {
  if (!out || !devices || ndev < 1 || ndev > 64 || slots_per_device < 1 || hbm_budget_per_device == 0 ||
      (batched && preparers < 1))
    return fail(PICARD_ERR_BAD_ARG, "bad server arguments");
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess) return fail(PICARD_ERR_CUDA, "no CUDA device");
  for (int k = 0; k < ndev; ++k)
    if (devices[k] < 0 || devices[k] >= count) return fail(PICARD_ERR_BAD_ARG, "device ordinal out of range");
  picard_server* m = new picard_server();
  m->budget = hbm_budget_per_device;
  m->max_slots = slots_per_device;
  m->batched = batched != 0;
  m->t0 = std::chrono::steady_clock::now();
  for (int k = 0; k < ndev; ++k)
    m->shards.push_back(open_server(hbm_budget_per_device, slots_per_device, batched != 0, preparers, devices[k], k,
                                    m->t0));
  *out = m;
  return PICARD_OK;
}

int picard_server_submit(picard_server* s, const picard_request* rq) {
  if (!s || !rq) return fail(PICARD_ERR_BAD_ARG, "NULL argument");
  if (rq->steps < 1) return fail(PICARD_ERR_BAD_ARG, "steps < 1");
  if (!s->shards.empty()) {
    // the least loaded shard (footprint held and queued over budget), the first on ties
    size_t best = 0;
    double lb = shard_load(s->shards[0]);
    for (size_t k = 1; k < s->shards.size(); ++k) {
      const double l = shard_load(s->shards[k]);
      if (l < lb) best = k, lb = l;
    }
    picard_request copy = *rq;
    if (copy.arrival_ms < 0) copy.arrival_ms = now_ms(s);
    return picard_server_submit(s->shards[best], &copy);
  }
  uint64_t fp = 0;
  PICARD_TRY(picard_gpu_footprint(&rq->params, rq->layout, rq->solver, &fp));
  if (fp > s->budget)
    return fail(PICARD_ERR_CAPACITY, "request needs " + std::to_string(fp) + " B, more than the whole HBM budget");
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stopping) return fail(PICARD_ERR_STATE, "server is shutting down");
    picard_request copy = *rq;
    if (copy.arrival_ms < 0) copy.arrival_ms = now_ms(s);
    s->queue.emplace_back(copy, fp);
    s->submitted += 1;
    if (s->batched) admit_locked(s);
  }
  s->cv_work.notify_all();
  return PICARD_OK;
}

int picard_server_now_ms(picard_server* s, double* ms) {
  if (!s || !ms) return fail(PICARD_ERR_BAD_ARG, "NULL argument");
  *ms = now_ms(s);
  return PICARD_OK;
}

int picard_server_poll(picard_server* s, picard_result* out, int32_t max, int32_t* n, int32_t wait_all) {
  if (!s || !n) return fail(PICARD_ERR_BAD_ARG, "NULL argument");
  if (!s->shards.empty()) {
    int32_t k = 0;
    for (picard_server* sh : s->shards) {
      int32_t got = 0;
      PICARD_TRY(picard_server_poll(sh, out + k, max - k, &got, wait_all));
      k += got;
    }
    std::stable_sort(out, out + k, [](const picard_result& a, const picard_result& b) { return a.finish_ms < b.finish_ms; });
    *n = k;
    return PICARD_OK;
  }
  std::unique_lock<std::mutex> lk(s->mu);
  if (wait_all) s->cv_done.wait(lk, [&] { return s->finished == s->submitted; });
  int32_t k = 0;
  while (k < max && !s->done.empty()) {
    out[k++] = s->done.front();
    s->done.erase(s->done.begin());
  }
  *n = k;
  return PICARD_OK;
}

int picard_server_load(picard_server* s, int32_t* running, int32_t* queued, uint64_t* bytes_in_use) {
  if (!s) return fail(PICARD_ERR_BAD_ARG, "NULL argument");
  if (!s->shards.empty()) {
    int32_t r = 0, q = 0;
    uint64_t b = 0;
    for (picard_server* sh : s->shards) {
      int32_t r1 = 0, q1 = 0;
      uint64_t b1 = 0;
      PICARD_TRY(picard_server_load(sh, &r1, &q1, &b1));
      r += r1, q += q1, b += b1;
    }
    if (running) *running = r;
    if (queued) *queued = q;
    if (bytes_in_use) *bytes_in_use = b;
    return PICARD_OK;
  }
  std::lock_guard<std::mutex> lk(s->mu);
  if (running) *running = s->running;
  if (queued) *queued = int32_t(s->queue.size());
  if (bytes_in_use) *bytes_in_use = s->in_use;
  return PICARD_OK;
}

int picard_server_destroy(picard_server* s) {
  if (!s) return PICARD_OK;
  if (!s->shards.empty()) {
    int rc = PICARD_OK;
    for (picard_server* sh : s->shards) {
      const int q = picard_server_destroy(sh);
      if (rc == PICARD_OK) rc = q;
    }
    delete s;
    return rc;
  }
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stopping = true;
  }
  s->cv_work.notify_all();
  s->cv_ready.notify_all();
  if (s->batched) {
    // the queue drains first: wait for every submitted run
    std::unique_lock<std::mutex> lk(s->mu);
    s->cv_done.wait(lk, [&] { return s->finished == s->submitted; });
    lk.unlock();
    s->cv_work.notify_all();
    s->cv_ready.notify_all();
  }
  for (auto& t : s->workers) t.join();
  delete s;
  return PICARD_OK;
}

}  // extern "C"
