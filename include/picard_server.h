/*
 * picard_server.h -- C ABI of the request loop that serves parameter-sweep
 * runs of Picard's main loop (picard.f90:554-674) on one device.
 *
 * The reference has no serving layer: one `program picard` process runs one
 * parameter set, hard-coded in picard.f90:42-52 and 145-302.  Here a request
 * carries its own picard_params block (the run's grid, plasma, source and
 * seed) and a step count; the server admits it when a worker slot is free and
 * its device footprint (picard_gpu_footprint) fits in the HBM budget, keeps
 * its particle and field state on the device for the whole run, and runs the
 * admitted requests concurrently, each on its own CUDA stream, so the kernels
 * of one run fill the gaps of another (a run waiting on the host for its
 * Jacobi stop test does not leave the device idle).  Requests are admitted in
 * arrival order.  A run's result does not depend on what else is running: every
 * kernel of a run touches only that run's buffers, and every reduction has a
 * fixed order.
 */
#ifndef PICARD_SERVER_H
#define PICARD_SERVER_H

#include <stdint.h>

#include "picard_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct picard_server picard_server;

typedef struct picard_request {
  int64_t id;            /* caller's tag, copied into the result              */
  picard_params params;  /* the run (picard_params_derive applied by the caller) */
  int32_t layout;        /* picard_layout                                     */
  int32_t solver;        /* picard_solver                                     */
  int32_t steps;         /* main-loop iterations 1..steps                     */
  double arrival_ms;     /* arrival time on the server clock; < 0: now        */
} picard_request;

typedef struct picard_result {
  int64_t id;
  int32_t status;          /* picard_status of the run                       */
  int32_t num_local;       /* live particles after the last step             */
  double arrival_ms;       /* server clock (ms since picard_server_create)   */
  double start_ms;         /* admission                                      */
  double finish_ms;        /* state released                                 */
  int64_t sweeps;          /* Jacobi sweeps over all steps                   */
  int64_t particle_steps;  /* live particles summed over the steps           */
  double energy[3];        /* kinetic, electric, magnetic (picard.f90:667-671) */
  double u_sum;            /* sum of the final potential over all nodes      */
  double u_abs_sum;        /* sum of its absolute values                     */
  uint32_t warnings;       /* WriteWarnings.f90 mask of the request's params
                              (picard_io.h picard_warning); the reference only
                              warns, so a run with warnings still runs       */
  int32_t shard;           /* index into the device list of picard_server_create_multi (0 otherwise) */
} picard_result;

/* hbm_budget_bytes: device memory the admitted runs may hold together.
 * max_slots: runs in flight at once (one host worker thread and one CUDA
 * stream each).  The server uses the calling thread's current device. */
PICARD_API int picard_server_create(uint64_t hbm_budget_bytes, int32_t max_slots, picard_server** out);
/* Continuous batching on the current device: at most max_runs runs admitted at
 * once (same admission rule), prepared (context, CalcDistance,
 * ParticlesInitialize) by `preparers` threads, and advanced together one
 * iteration at a time by picard_batch_step -- every run's Jacobi sweeps in
 * one launch per sweep -- joining and leaving the cohort between steps.  Each
 * run's result is bit-identical to the same run alone. */
PICARD_API int picard_server_create_batched(uint64_t hbm_budget_bytes, int32_t max_runs, int32_t preparers,
                                            picard_server** out);
/* Run placement over several devices: one server per entry of devices[ndev]
 * (stream mode, or continuous batching when `batched`), each with its own HBM
 * budget and slots.  A request goes to the shard whose admitted and queued
 * footprint is the smallest fraction of its budget (the first on ties); runs
 * are independent, so nothing crosses between devices.  submit, poll (results
 * of every shard, in finish order, tagged with their shard), load (summed) and
 * destroy work on the whole set.  An ordinal may appear more than once: two
 * shards then share that device. */
PICARD_API int picard_server_create_multi(const int32_t* devices, int32_t ndev, uint64_t hbm_budget_per_device,
                                          int32_t slots_per_device, int32_t batched, int32_t preparers,
                                          picard_server** out);
/* Queues a run.  PICARD_ERR_CAPACITY if its footprint exceeds the whole budget
 * (it could never be admitted), PICARD_ERR_BAD_ARG for invalid params. */
PICARD_API int picard_server_submit(picard_server* s, const picard_request* rq);
/* Milliseconds since picard_server_create, on the clock of the results. */
PICARD_API int picard_server_now_ms(picard_server* s, double* ms);
/* Moves up to max finished results into out (completion order).  wait_all != 0
 * first waits until every submitted run has finished. */
PICARD_API int picard_server_poll(picard_server* s, picard_result* out, int32_t max, int32_t* n,
                                  int32_t wait_all);
/* Runs in flight and queued, and the HBM budget they hold. */
PICARD_API int picard_server_load(picard_server* s, int32_t* running, int32_t* queued, uint64_t* bytes_in_use);
/* Finishes the queued and running requests, then joins the workers. */
PICARD_API int picard_server_destroy(picard_server* s);

#ifdef __cplusplus
}
#endif

#endif /* PICARD_SERVER_H */
