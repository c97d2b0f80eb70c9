"""Particle-steps/s of Picard's per-timestep PIC loop on B200.

One "step" is one iteration of picard.f90:554-674 (inflow, position advance,
Haser production, outflow, wrap, CIC deposit, open-boundary potential, Jacobi
solve, E-field, Boris push) over the whole run.  The default workload is the
at-scale plain configuration: 256x128x128 cells of 1 km, 32 H+ and 32
electrons per cell (268,435,456 particles), drifting solar-wind Maxwellian,
Haser source at the centre, CELL32 particles (32-bit fixed-point in-cell
offsets, FP32 velocities), BCpotentials as FP64 FFT convolutions, and the
Jacobi iterate of the reference's stopping sweep (tolerance 1e-6) in closed
form (--solver spectral; --solver refine runs the FP32 sweeps under FP64
anchors instead).  Inputs are synthetic (seeded Philox, seed = rank); the
particle arrays (7.8 GB) are far larger than L2.

Arms:
  --impl picard     the sm_100a kernels through the C ABI (default)
  --impl reference  the CPU oracle (the FP64 restatement of the reference;
                    the Fortran+MPI reference cannot be built on these
                    machines) with every host thread, one bounded sample of a
                    full-size step per timed step.
Multi-GPU (torchrun): every rank advances its own independent run of the same
workload (weak scaling, no data-path collective); value = particle-steps of
all ranks / the slowest rank's device time.
"""
from __future__ import annotations

import argparse
import datetime
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "particle-steps/s"
UNIT = "particle-steps/s"


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["picard", "reference"], default="picard")
    ap.add_argument("--workload", choices=["scale", "plain32", "poisson", "serving", "precision", "batch",
                                           "bcpot", "deposit"], default="scale")
    ap.add_argument("--runs", type=int, default=64, help="batch workload: runs in the parameter sweep")
    ap.add_argument("--precision-n", type=int, default=512, help="precision workload: box edge in cells")
    ap.add_argument("--precision-sweeps", type=int, default=4001, help="precision workload: Jacobi sweeps compared")
    ap.add_argument("--requests", type=int, default=12, help="serving workload: runs in the arrival stream")
    ap.add_argument("--rate", type=float, default=20.0, help="serving workload: mean arrivals per second")
    ap.add_argument("--run-steps", type=int, default=200, help="serving workload: iterations per run")
    ap.add_argument("--slots", type=int, default=8, help="serving workload: runs in flight at once")
    ap.add_argument("--batch-slots", type=int, default=8,
                    help="serving workload, continuous batching: runs in the cohort at once")
    ap.add_argument("--preparers", type=int, default=3,
                    help="serving workload, continuous batching: threads preparing admitted runs")
    ap.add_argument("--budget-gb", type=float, default=150.0, help="serving workload: HBM budget of admitted runs")
    ap.add_argument("--poisson-n", type=int, default=256)
    ap.add_argument("--poisson-dims", type=str, default=None, help="poisson workload: nx,ny,nz (default n^3)")
    ap.add_argument("--poisson-sweeps", type=int, default=400)
    ap.add_argument("--deposit-dims", type=str, default=None,
                    help="deposit workload: nx,ny,nz (default 256,128,128)")
    ap.add_argument("--layout", choices=["cell32", "f64"], default="cell32")
    ap.add_argument("--solver", choices=["refine", "f64", "spectral"], default="spectral")
    ap.add_argument("--sort-every", type=int, default=0,
                    help="fused loop: sort the particles by CIC stencil every k iterations (0: never)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-phi", action="store_true", help="skip the FP64 check of the timed run's potential")
    ap.add_argument("--no-sweep", action="store_true",
                    help="skip the FP32 sweep solve of the timed run's charge (the jacobi_sweep block)")
    ap.add_argument("--no-served", action="store_true",
                    help="skip the served and batched blocks of the default (N=1) line")
    ap.add_argument("--served-requests", type=int, default=16, help="default line: runs in the serving stream")
    ap.add_argument("--served-steps", type=int, default=200, help="default line: iterations per served run")
    ap.add_argument("--batched-runs", type=int, default=64, help="default line: runs of the batched sweep")
    ap.add_argument("--batched-steps", type=int, default=20, help="default line: iterations per batched run")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=25.0, help="rough budget of the CPU baseline sample")
    ap.add_argument("--ppc", type=int, default=None,
                    help="ions per cell of the at-scale workload (default 32; smaller for profiling runs)")
    return ap.parse_args()


def workload(name: str, seed: int, ppc: int | None = None):
    from picard_b200 import params as P

    if name == "scale":
        p = P.config_plain_scale(seed=seed) if ppc is None else P.config_plain_scale(seed=seed, ppc_ion=ppc)
        desc = {"workload": "plain-at-scale 256x128x128 cells, 64 ppc (32 H+ + 32 e-), Haser source Q=1e27/s",
                "grid": [256, 128, 128], "ppc_total": 64, "species": 3,
                "l2": "particle arrays (7.8 GB) exceed L2; the Jacobi working set (52 MB) is L2-resident"}
    else:
        p = P.config_plain_32(seed=seed)
        desc = {"workload": "plain 32^3 cells, 16 ppc per species (H+, e-)", "grid": [32, 32, 32],
                "ppc_total": 32, "species": 2, "l2": "every working set fits in L2"}
    return p, desc


def env_rank():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms while the
    timed region runs."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu_index = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(prefix="clocks_", suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.gpu_index)],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        with open(self.path) as f:
            for line in f:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(rows)}


def combine_ranks(ms: float, work: float, dist=None, device: str = "cpu"):
    """Whole-job timing of independent runs, one per rank: the slowest rank's
    device time and the work summed over ranks (every rank takes part)."""
    if dist is None:
        return ms, work
    import torch

    t = torch.tensor([ms, work], dtype=torch.float64, device=device)
    tmax = t.clone()
    dist.all_reduce(tmax, op=dist.ReduceOp.MAX)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(tmax[0]), float(t[1])


# ---------------------------------------------------------------- GPU arm

SOLVERS = {"f64": 0, "refine": 1, "spectral": 2}  # picard_solver (include/picard_gpu.h)
SOLVER_WORDS = {"f64": "f64 Jacobi sweeps", "refine": "f32 Jacobi sweeps with f64 anchors",
                "spectral": "f64 closed-form Jacobi iterate (sine-basis transforms)"}


def dtype_of(args) -> str:
    parts = "cell32 particles (32-bit fixed-point offsets, f32 velocities)" if args.layout == "cell32" else "f64 particles"
    return f"{parts}, {SOLVER_WORDS[args.solver]}"


def run_picard(args, rank, world, local_rank):
    import torch

    from picard_b200 import capi
    from picard_b200.simulation import Simulation

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist
    layout = capi.LAYOUT_CELL32 if args.layout == "cell32" else capi.LAYOUT_F64
    solver = SOLVERS[args.solver]
    p, desc = workload(args.workload, seed=rank, ppc=args.ppc)
    if args.ppc is not None:
        desc = dict(desc, ppc_total=2 * args.ppc, workload=desc["workload"] + f" (ppc override {args.ppc})")
    W, K = args.warmup, args.steps

    sim = Simulation(p, layout=layout, solver=solver)
    if args.sort_every:
        sim.set_option(capi.OPT_SORT_EVERY, args.sort_every)
    sim.calc_distance()
    sim.particles_initialize()
    sim.run_fused(0, W)
    sim.reset_stats()
    ext = torch.cuda.ExternalStream(sim.stream_handle)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    visible = os.environ.get("CUDA_VISIBLE_DEVICES")
    gpu_index = int(visible.split(",")[local_rank]) if visible else local_rank
    clocks = ClockSampler(gpu_index)
    clocks.start()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record(ext)
    sim.run_fused(W, W + K)
    t1.record(ext)
    t1.synchronize()
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = t0.elapsed_time(t1)
    st = sim.stats()
    particle_steps = st["particle_steps"]
    sweeps_per_step = st["sweeps"] / max(st["solves"], 1)
    # dominant kernel: the CIC deposit (ParticlesGridify), timed on its own
    # right after the timed region on the run's final particles, K launches
    # of the entry point (deposit kernel + fixed-point finish) on the
    # library's stream; algorithmic bytes = the particle stream it reads
    dep_ms = deposit_launch_ms(sim, ext, K, torch)
    n_dep = sim.num_local
    alg_bytes = DEPOSIT_BYTES_PER_PARTICLE * n_dep
    achieved = alg_bytes / (dep_ms * 1e-3) / 1e9
    sweep = sweep_roofline(sim, p, torch) if not args.no_sweep else None
    num_final = sim.num_local
    phi = None
    if not args.no_phi:
        phi = phi_check(sim, p, desc)
    sim.close()
    del sim
    torch.cuda.synchronize()

    # end to end through the reference-facing entry points (picard_gpu_run:
    # the per-subroutine call sequence of picard.f90), from the host-side
    # parameter block: context creation, CalcDistance, ParticlesInitialize,
    # K iterations with the energy log read back every iteration.
    e2e = None
    if not args.no_e2e:
        logged = []
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        ea = torch.cuda.Event(enable_timing=True)
        e0.record()
        s2 = Simulation(p, layout=layout, solver=solver)
        s2.calc_distance()
        s2.particles_initialize()
        s2.synchronize()
        ea.record()
        s2.reset_stats()
        s2.run(0, K, log_interval=1, log=lambda *row: logged.append(row))
        torch.cuda.synchronize()
        e1.record()
        e1.synchronize()
        e_ms = e0.elapsed_time(e1)
        setup_ms = e0.elapsed_time(ea)
        st2 = s2.stats()
        s2.close()
        import ctypes

        from picard_b200.params import PicardParams

        params_bytes = ctypes.sizeof(PicardParams)
        e2e = {"value": st2["particle_steps"] / (e_ms * 1e-3), "unit": UNIT,
               "h2d_bytes_per_step": int(round((params_bytes + st2.get("h2d_bytes", 0)) / K)),
               "d2h_bytes_per_step": int(round(st2.get("d2h_bytes", 0) / K)),
               "path": "picard_gpu_run (per-subroutine C-ABI calls) incl. context creation and initialisation",
               "ms": e_ms, "setup_ms": setup_ms, "loop_ms_per_step": (e_ms - setup_ms) / K}

    ms_max, total_ps = combine_ranks(ms, float(particle_steps), dist, "cuda")
    value = total_ps / (ms_max * 1e-3)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baseline(args, sweeps_per_step=sweeps_per_step)
    served = batched = None
    if rank == 0 and world == 1 and not args.no_served and args.workload == "scale":
        # the headline comparison on one GPU: the same runs served, batched
        # and run one after another through the per-subroutine loop
        served = serving_measure(args, local_rank, args.served_requests, args.served_steps)
        batched = batch_measure(args, local_rank, args.batched_runs, args.batched_steps)

    if rank == 0:
        peak, peak_kind = measured_peaks()
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
            "ms_per_step": ms_max / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": dtype_of(args),
            "data": "synthetic (seeded Philox plasma, seed = rank)",
            "config": line_config(desc, world),
            "impl": "picard",
            "layout": args.layout, "solver": args.solver, "sort_every": args.sort_every,
            "gpu_launches": st["kernel_launches"],
            "jacobi_sweeps_per_step": sweeps_per_step,
            "phase_ms_per_step": {k: round(v / K, 3) for k, v in st["phase_ms"].items()},
            "particles_final": num_final,
            "roofline": {"bound": "hbm",
                         "kernel": "deposit_tile_c32_kernel" if args.layout == "cell32" else "deposit_f64_kernel",
                         "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_kind": peak_kind,
                         "alg_bytes_per_launch": alg_bytes, "launch_ms": dep_ms,
                         "alg_bytes_rule": f"{DEPOSIT_BYTES_PER_PARTICLE} B per particle read (cell word, three "
                                           "32-bit offsets, species) x the live particles",
                         "traffic": (DEPOSIT_DRAM_BYTES_PER_PARTICLE * n_dep
                                     if DEPOSIT_DRAM_BYTES_PER_PARTICLE and args.layout == "cell32" else None),
                         "traffic_source": "dram__bytes_read.sum + dram__bytes_write.sum per particle (17.49 B) of "
                                           "one ncu capture of the deposit at 128x64x64 x 64 ppc (the default "
                                           "workload's density), scaled by the particles",
                         "note": "launch_ms is the ParticlesGridify entry point (deposit kernel and the "
                                 "fixed-point finish) timed with CUDA events on the library stream, K launches on "
                                 "the timed run's final particles; the step's other phases are in "
                                 "phase_ms_per_step"},
            "jacobi_sweep": sweep,
            "clocks": clk,
            "e2e": e2e,
            "cpu_baseline": cpu,
            "phi_check": phi,
        }
        if served is not None:
            line["served"] = compact_serving(served)
        if batched is not None:
            line["batched"] = compact_batch(batched)
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()


# CELL32 ParticlesGridify reads the cell word, the three 32-bit offsets and
# the species of every particle.
DEPOSIT_BYTES_PER_PARTICLE = 17
# DRAM bytes per particle of one deposit launch (dram__bytes_read.sum +
# dram__bytes_write.sum over the particles): 581.7 + 5.1 MB over 33,556,485
# particles in an ncu capture at 128x64x64 with 32 + 32 ppc, the density of
# the default workload (the node arrays' share per particle depends on the
# density, not on the grid).
DEPOSIT_DRAM_BYTES_PER_PARTICLE = 17.49


def deposit_launch_ms(sim, ext, reps: int, torch) -> float:
    """Device time of one ParticlesGridify call on the run's particles: reps
    calls between CUDA events on the library's stream, after one untimed call."""
    sim.particles_gridify()
    sim.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(ext)
    for _ in range(max(1, reps)):
        sim.particles_gridify()
    e1.record(ext)
    e1.synchronize()
    return e0.elapsed_time(e1) / max(1, reps)


def sweep_roofline(sim, p, torch) -> dict:
    """The FP32 Jacobi sweep kernel on the timed run's grid: one solve of the
    run's last charge density with the F32_REFINE solver (the sweeps the
    closed form replaces), its sweep launches timed with CUDA events on the
    library's stream; 12 B per interior node per sweep against the measured
    HBM copy rate and a device copy whose buffers stay in L2 (the 52 MB
    working set is L2-resident)."""
    from picard_b200 import capi
    from picard_b200.simulation import Simulation

    C = sim.field(capi.FIELD_C)
    st = sim.stats()
    q = p.copy()
    q.max_per_proc = 1024
    ref = Simulation(q, layout=capi.LAYOUT_CELL32, solver=capi.SOLVER_F32_REFINE)
    ref.calc_distance()
    ref.set_field(capi.FIELD_C, C)
    ref.bc_potentials()
    ref.reset_stats()
    sweeps = ref.calc_epotential()
    ref.synchronize()
    s2 = ref.stats()
    ref.close()
    launch_ms = s2["sweep_ms"] / max(s2["sweep_launches"], 1)
    alg = 12 * p.nx * p.ny * p.nz
    achieved = alg / (launch_ms * 1e-3) / 1e9
    peak, kind = measured_peaks()
    l2 = l2_copy_gbs(torch)
    spec_ms = st["spectral_transform_ms"] / max(st["spectral_transforms"] / 2, 1)
    return {"kernel": "sweep_tma2_kernel" if p.xflow and p.yflow and p.zflow else "sweep_f32_kernel",
            "bound": "l2", "sweeps": sweeps, "launch_ms": launch_ms, "alg_bytes_per_launch": alg,
            "achieved": achieved, "unit": "GB/s", "frac_of_hbm_copy": achieved / peak, "peak_kind": kind,
            "l2_copy_gbs": l2, "l2_frac": achieved / l2 if l2 else None,
            "traffic": SWEEP_DRAM_BYTES.get((p.nx, p.ny, p.nz, 1)),
            "solve_ms_sweeps": s2["sweep_ms"] + s2["anchor_ms"],
            "solve_ms_closed_form_transforms": spec_ms,
            "note": "the FP32 sweep solve of the timed run's last charge density; the timed loop takes the same "
                    "iterate in closed form (two FP64 transforms + a few Parseval evaluations)"}


def phi_check(sim, p, desc) -> dict:
    """The timed run's last potential against an all-FP64 solve of the same
    charge density: FP64 BCpotentials (direct sum) and FP64 Jacobi sweeps
    (SOLVER_F64, whose sweeps and stopping rule equal the oracle's) from the
    run's C, with the reference's tolerance maxerr.  The bar is 1e-6 relative
    L2 (the potential's tolerance)."""
    import numpy as np

    from picard_b200 import capi
    from picard_b200.simulation import Simulation

    U = sim.field(capi.FIELD_U)
    Cd = sim.field(capi.FIELD_C)
    sweeps_run = sim.stats()["last_sweeps"]
    q = p.copy()
    q.max_per_proc = 1024
    ref = Simulation(q, layout=capi.LAYOUT_F64, solver=capi.SOLVER_F64)
    ref.calc_distance()
    ref.set_field(capi.FIELD_C, Cd)
    ref.set_option(capi.OPT_BCPOT_TENSOR, 0)
    t0 = time.perf_counter()
    ref.bc_potentials()
    sweeps64 = ref.calc_epotential()
    ref.synchronize()
    t64 = time.perf_counter() - t0
    U64 = ref.field(capi.FIELD_U)
    ref.close()
    d = U - U64
    rel = float(np.linalg.norm(d.ravel()) / np.linalg.norm(U64.ravel()))
    return {"rel_l2": rel, "max_rel": float(np.abs(d).max() / np.abs(U64).max()), "bar": 1e-6, "ok": rel <= 1e-6,
            "sweeps_fp64": sweeps64, "sweeps_timed_run_last_solve": sweeps_run, "fp64_solve_s": round(t64, 3),
            "what": "U after the last timed iteration (the run's BCpotentials method and solver) vs FP64 direct-sum "
                    "BCpotentials + FP64 Jacobi sweeps (SOLVER_F64) from the same C"}


def l2_copy_gbs(torch) -> float:
    """Device copy rate with both buffers resident in L2 (2 x 24 MiB, copied
    back and forth): read + write bytes over CUDA-event time.  The ceiling
    of a kernel whose working set stays in L2."""
    n = 24 * 2 ** 20 // 4
    a = torch.ones(n, dtype=torch.float32, device="cuda")
    b = torch.zeros_like(a)
    for _ in range(20):
        b.copy_(a)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    reps = 400
    e0.record()
    for i in range(reps):
        (b if i % 2 == 0 else a).copy_(a if i % 2 == 0 else b)
    e1.record()
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    del a, b
    return 2.0 * n * 4 * reps / (ms * 1e-3) / 1e9


def compact_serving(d: dict) -> dict:
    keys = ("config", "served", "batched_served", "plain", "served_over_plain", "batched_served_over_plain",
            "offered_load", "u_sum_max_rel_diff_served_vs_plain", "clocks")
    return {k: d[k] for k in keys if k in d}


def compact_batch(d: dict) -> dict:
    keys = ("config", "batched", "plain", "fused", "batched_over_plain", "batched_over_fused",
            "results_identical_to_fused", "jacobi_sweeps_total", "clocks")
    return {k: d[k] for k in keys if k in d}


# ----------------------------------------------------------- CPU baseline

# DRAM bytes of one Jacobi sweep launch, from an ncu capture of that launch
# (dram__bytes_read.sum + dram__bytes_write.sum), keyed by (nx, ny, nz, solver)
SWEEP_DRAM_BYTES = {(256, 128, 128, 1): 35.22e6}


def cpu_baseline(args, sweeps_per_step=None, steps: int = 1) -> dict:
    """Bounded samples of full-size iterations on the CPU oracle with every
    host thread.  Per iteration the particle phase (inflow, advance, produce,
    outflow, wrap, deposit, E-field, push) runs in full at full size; the
    field solve is sampled once: BCpotentials on a strided subset of face nodes
    (times the stride) and Jacobi timed over a few sweeps (times the sweeps an
    iteration takes: the count measured by the GPU arm on the same algorithm
    and stopping rule when available, else the slowest-mode estimate)."""
    from oracle import oracle as O

    threads = os.cpu_count() or 1
    O.set_threads(threads)
    p, desc = workload(args.workload, seed=0)
    p = O.derive(p)
    s = O.OracleState(p)
    s.calc_distance()
    s.initialize()

    def timed(fn):
        a = time.perf_counter()
        fn()
        return time.perf_counter() - a

    # field solve, sampled once
    faces = 2 * (p.ny * p.nz + p.nx * p.nz + p.nx * p.ny)
    stride = max(1, faces // 1536)
    s.gridify()
    t_bcpot = timed(lambda: s.bc_potentials_sampled(stride)) * stride
    maxit = 10
    t_sweep = timed(lambda: s.calc_epotential(maxerr=1e-300, maxit=maxit)) / (2 * maxit + 1)
    if sweeps_per_step is not None and sweeps_per_step > 0:
        n_sweeps, n_kind = sweeps_per_step, "measured by the GPU arm (same algorithm and stopping rule)"
    else:
        # slowest Jacobi mode: rho = sum_d 2 a_d cos(pi/(N_d+1)); residual 1e-6
        d = list(p.dxyz)
        S = (d[0] * d[1]) ** 2 + (d[0] * d[2]) ** 2 + (d[1] * d[2]) ** 2
        a_ = [0.5 / S * (d[1] * d[2]) ** 2, 0.5 / S * (d[0] * d[2]) ** 2, 0.5 / S * (d[0] * d[1]) ** 2]
        rho = sum(2 * a_[k] * math.cos(math.pi / (n + 1)) for k, n in enumerate((p.nx, p.ny, p.nz)))
        n_sweeps, n_kind = math.log(p.maxerr) / math.log(rho), "slowest-mode estimate ln(1e-6)/ln(rho_J)"
    t_jacobi = t_sweep * n_sweeps
    per_step = []
    phases = {}
    particle_steps = 0
    for it in range(1, steps + 1):
        t = {"inflow": timed(lambda: s.bc_inflow(it)), "advance": timed(lambda: s.advance_position()),
             "produce": timed(lambda: s.produce(it)), "outflow": timed(lambda: s.bc_outflow()),
             "transfer": timed(lambda: s.transfer()), "gridify": timed(lambda: s.gridify()),
             "efield": timed(lambda: s.calc_efield()), "velocity": timed(lambda: s.advance_velocity())}
        t["bcpot"] = t_bcpot
        t["jacobi"] = t_jacobi
        per_step.append(sum(t.values()))
        particle_steps += s.num_local
        phases = t
    total = sum(per_step)
    return {"value": particle_steps / total, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": (f"{steps} full-size iteration(s) ({s.num_local} particles) on the FP64 oracle: particle "
                       f"phase timed in full, BCpotentials on 1/{stride} of the face nodes x{stride}, Jacobi "
                       f"{2 * maxit + 1} sweeps timed ({t_sweep * 1e3:.2f} ms/sweep) x {n_sweeps:.0f} sweeps per "
                       f"iteration ({n_kind})"),
            "seconds_per_step": total / steps, "phase_seconds": {k: round(v, 4) for k, v in phases.items()}}


def blob_charge(n: int, seed: int, blobs: int = 32):
    """Charge of the standalone Poisson workload: `blobs` Gaussian blobs
    (centres uniform in the box, sigma uniform in [4, 16] cells, amplitudes
    N(0, 1) e per cell) plus 1% uniform noise, on an n^3 box with ghosts."""
    import numpy as np

    from picard_b200 import params as P

    rng = np.random.default_rng(seed)
    ax = np.arange(n + 2, dtype=np.float64)
    C = np.zeros((n + 2,) * 3)
    for _ in range(blobs):
        c = rng.uniform(1, n, 3)
        s = rng.uniform(4, 16)
        a = rng.standard_normal()
        gx, gy, gz = (np.exp(-0.5 * ((ax - c[d]) / s) ** 2) for d in range(3))
        C += a * gz[:, None, None] * gy[None, :, None] * gx[None, None, :]
    C += 0.01 * rng.uniform(-1, 1, C.shape)
    C[0, :, :] = C[-1, :, :] = 0
    C[:, 0, :] = C[:, -1, :] = 0
    C[:, :, 0] = C[:, :, -1] = 0
    return C * P.EC


def run_poisson(args, local_rank):
    """Jacobi-only workload: an n^3 open box, blob charge, zero boundary
    potential, `--poisson-sweeps` sweeps (maxit bounded, no stop).  Reports the
    sweep kernel's device time and roofline.  Used for kernel profiling on a
    working set larger than L2."""
    import torch

    from picard_b200 import capi
    from picard_b200 import params as P
    from picard_b200.simulation import Simulation

    import numpy as np

    torch.cuda.set_device(local_rank)
    n = args.poisson_n
    dims = [int(v) for v in args.poisson_dims.split(",")] if args.poisson_dims else [n, n, n]
    nx, ny, nz = dims
    p = P.config_plain_32(n=8, ppc=1, capacity=1024)
    p.nx, p.ny, p.nz = nx, ny, nz
    p.xmin, p.xmax = -500.0 * nx, 500.0 * nx
    p.ymin, p.ymax = -500.0 * ny, 500.0 * ny
    p.zmin, p.zmax = -500.0 * nz, 500.0 * nz
    solver = capi.SOLVER_F32_REFINE if args.solver == "refine" else capi.SOLVER_F64
    sim = Simulation(p, layout=capi.LAYOUT_F64, solver=solver)
    big = blob_charge(max(dims), seed=0)
    C = np.ascontiguousarray(big[: nz + 2, : ny + 2, : nx + 2])
    C[-1, :, :] = C[:, -1, :] = C[:, :, -1] = 0.0
    sim.set_field(capi.FIELD_C, C)
    sim.set_field(capi.FIELD_U, np.zeros_like(C))
    maxit = max(1, args.poisson_sweeps // 2)
    sim.calc_epotential(maxerr=1e-300, maxit=maxit)  # warm-up solve
    sim.reset_stats()
    sim.set_field(capi.FIELD_U, np.zeros_like(C))
    sim.calc_epotential(maxerr=1e-300, maxit=maxit)
    st = sim.stats()
    shape = (sim.get_option(capi.OPT_SWEEP_PAIRS), sim.get_option(capi.OPT_SWEEP_CTAS),
             sim.get_option(capi.OPT_SWEEP_PDL), sim.get_option(capi.OPT_SWEEP_STAGES),
             sim.get_option(capi.OPT_SWEEP_RESIDENT))
    sim.close()
    cells = nx * ny * nz
    bpn = 12 if solver == capi.SOLVER_F32_REFINE else 24
    ms = st["sweep_ms"] / max(st["sweep_launches"], 1)
    peak, kind = measured_peaks()
    ach = bpn * cells / (ms * 1e-3) / 1e9
    print(json.dumps({"workload": f"poisson {nx}x{ny}x{nz}", "sweep_shape": {
                          "pairs": shape[0], "ctas": shape[1], "pdl": shape[2], "stages": shape[3],
                          "resident": shape[4]}, "sweeps": st["sweep_launches"], "sweep_ms": ms,
                      "achieved_gbs": ach, "peak_gbs": peak, "frac": ach / peak, "peak_kind": kind,
                      "anchor_ms": st["anchor_ms"] / max(st["anchor_launches"], 1),
                      "gpu_launches": st["kernel_launches"]}), flush=True)


def run_serving(args, local_rank):
    print(json.dumps(serving_measure(args, local_rank, args.requests, args.run_steps)), flush=True)


def serving_measure(args, local_rank, requests: int, run_steps: int) -> dict:
    """Serving workload: a Poisson stream of `requests` parameter-sweep runs
    (cubic grids of 24..128 cells, 8..64 ppc, Haser Q log-uniform in
    [1e25, 1e28] s^-1, `run_steps` iterations each) served three ways on one
    GPU.
      plain:  one run after another through picard_gpu_run (the per-subroutine
              call sequence of picard.f90), the arrival stream replayed against
              the measured service times;
      served: the picard_server request loop -- admission under the HBM
              budget, --slots runs in flight on their own streams, requests
              submitted at their arrival times.
      batched: the continuous-batching request loop -- the same admission, up
              to --batch-slots runs advanced together one iteration at a time,
              all their Jacobi sweeps in one launch per sweep.
    All arms create, initialise, run and release every run inside the timed
    region.  Throughput = particle-steps of all runs / (last finish - first
    arrival); latency = finish - arrival."""
    import numpy as np
    import torch

    from picard_b200 import capi
    from picard_b200 import params as P
    from picard_b200.server import Server
    from picard_b200.simulation import Simulation

    torch.cuda.set_device(local_rank)
    stream = P.serving_stream(seed=0, count=requests, rate_per_s=args.rate)
    reqs = []
    for t, p, steps in stream:
        if run_steps != steps:
            p = P._size_capacity(p, run_steps, max(1, int(p.ppc[1])))
        reqs.append((t, capi.params_derive(p), run_steps))
    layout, solver = capi.LAYOUT_CELL32, SOLVERS[args.solver]

    # warm-up, untimed: load the kernels, and run the sweep launch tuner once per
    # grid shape (cached for the process) so that neither arm pays for tuning
    w = P.config_plain_scale(seed=99, nx=16, ny=16, nz=16, ppc_ion=2)
    sim = Simulation(w, layout=layout, solver=solver)
    sim.calc_distance()
    sim.particles_initialize()
    sim.run_fused(0, 2)
    sim.close()
    seen = set()
    for _, p, _ in reqs:
        if (p.nx, p.ny, p.nz) not in seen:
            seen.add((p.nx, p.ny, p.nz))
            Simulation(p, derive=False, layout=layout, solver=solver).close()
    torch.cuda.synchronize()

    visible = os.environ.get("CUDA_VISIBLE_DEVICES")
    clocks = ClockSampler(int(visible.split(",")[local_rank]) if visible else local_rank)
    clocks.start()
    plain = []
    for t, p, steps in reqs:
        a = time.perf_counter()
        sim = Simulation(p, derive=False, layout=layout, solver=solver)
        sim.calc_distance()
        sim.particles_initialize()
        sweeps = sim.run(0, steps)
        st = sim.stats()
        U = sim.field(capi.FIELD_U)
        sim.close()
        plain.append({"service_s": time.perf_counter() - a, "particle_steps": st["particle_steps"],
                      "sweeps": sweeps, "u_sum": float(U.sum())})
    clock = reqs[0][0]
    plain_lat = []
    for (t, _, _), r in zip(reqs, plain):
        start = max(clock, t)
        clock = start + r["service_s"]
        plain_lat.append(clock - t)
    plain_makespan = clock - reqs[0][0]

    def serve(srv):
        base = srv.now_ms()
        for i, (t, p, steps) in enumerate(reqs):
            wait = base + t * 1e3 - srv.now_ms()
            if wait > 0:
                time.sleep(wait * 1e-3)
            srv.submit(i, p, steps, layout=layout, solver=solver, arrival_ms=base + t * 1e3)
        res = sorted(srv.poll(wait_all=True), key=lambda r: r["id"])
        makespan = (max(r["finish_ms"] for r in res) - (base + reqs[0][0] * 1e3)) * 1e-3
        return res, makespan

    with Server(int(args.budget_gb * 1e9), args.slots) as srv:
        res, served_makespan = serve(srv)
    with Server(int(args.budget_gb * 1e9), args.batch_slots, batched=True, preparers=args.preparers) as srv:
        bres, batched_makespan = serve(srv)
    clk = clocks.stop()
    bad = [r for r in res + bres if r["status"] != capi.OK]
    served_lat = [(r["finish_ms"] - r["arrival_ms"]) * 1e-3 for r in res]
    batched_lat = [(r["finish_ms"] - r["arrival_ms"]) * 1e-3 for r in bres]
    ps_served = sum(r["particle_steps"] for r in res)
    ps_batched = sum(r["particle_steps"] for r in bres)
    ps_plain = sum(r["particle_steps"] for r in plain)
    u_diff = max(abs(r["u_sum"] - q["u_sum"]) / max(abs(q["u_sum"]), 1e-300) for r, q in zip(res, plain))
    b_mismatch = sum(1 for r, q in zip(bres, res)
                     if (r["u_sum"], r["u_abs_sum"], r["num_local"], r["sweeps"]) !=
                     (q["u_sum"], q["u_abs_sum"], q["num_local"], q["sweeps"]))

    def pct(v, q):
        return float(np.percentile(np.asarray(v), q))

    served_tput = ps_served / served_makespan
    batched_tput = ps_batched / batched_makespan
    plain_tput = ps_plain / plain_makespan
    line = {
        "metric": "particle-steps/s & run p50/p99 latency, served vs plain", "value": max(served_tput, batched_tput),
        "unit": UNIT, "n_gpus": 1, "higher_is_better": True, "impl": "picard",
        "workload": "serving", "vs_baseline": None,
        "dtype": dtype_of(args),
        "data": "synthetic (seeded Philox plasma, run seeds 0..requests-1)",
        "config": {"workload": f"serving stream: {len(reqs)} runs, Poisson arrivals {args.rate}/s, cubic grids "
                               f"24..128 cells, 8..64 ppc, Haser Q log-uniform [1e25, 1e28] s^-1, "
                               f"{run_steps} steps each",
                   "grids": [int(p.nx) for _, p, _ in reqs], "budget_gb": args.budget_gb, "slots": args.slots,
                   "batch_slots": args.batch_slots, "preparers": args.preparers},
        "served": {"particle_steps_per_s": served_tput, "makespan_s": served_makespan,
                   "p50_latency_s": pct(served_lat, 50), "p99_latency_s": pct(served_lat, 99),
                   "failed": len(bad)},
        "batched_served": {"particle_steps_per_s": batched_tput, "makespan_s": batched_makespan,
                           "p50_latency_s": pct(batched_lat, 50), "p99_latency_s": pct(batched_lat, 99),
                           "results_differing_from_stream_mode": b_mismatch},
        "plain": {"particle_steps_per_s": plain_tput, "makespan_s": plain_makespan,
                  "p50_latency_s": pct(plain_lat, 50), "p99_latency_s": pct(plain_lat, 99),
                  "busy_s": sum(r["service_s"] for r in plain)},
        "served_over_plain": served_tput / plain_tput,
        "batched_served_over_plain": batched_tput / plain_tput,
        "offered_load": {"arrivals_per_s": args.rate,
                         "plain_service_rate_per_s": len(reqs) / sum(r["service_s"] for r in plain)},
        "u_sum_max_rel_diff_served_vs_plain": u_diff,
        "clocks": clk,
    }
    return line


def run_precision(args, local_rank):
    """Precision study on an n^3 open box (default 512^3) with the blob charge
    (32 Gaussian blobs, sigma 4..16 cells, N(0,1) e per cell, 1% noise):
      boundary: the tensor-core BCpotentials (three-way BF16 split, FP32
                accumulation in TMEM folded on chip, FP64 partials) against the
                FP64 direct sum, over every face node (the full product, no
                coarsening of the charge);
      jacobi:   FP32 sweeps of the increment with FP64 anchors against all-FP64
                sweeps, the same number of sweeps from the same FP64 boundary
                potential;
      end to end: tensor-core boundary + FP32/FP64 Jacobi against FP64 boundary
                + FP64 Jacobi;
      and the FP64 methods of the default path: the FFT boundary against the
      direct sum, the closed-form iterate of the same sweep count against the
      FP64 sweeps, and FFT boundary + closed form end to end.
    Errors are relative L2 over the nodes compared, and the largest pointwise
    error relative to the largest |U|."""
    import numpy as np
    import torch

    from picard_b200 import capi
    from picard_b200 import params as P
    from picard_b200.simulation import Simulation

    torch.cuda.set_device(local_rank)
    n = args.precision_n
    p = P.config_plain_32(n=n, ppc=1, capacity=1024)
    C = blob_charge(n, seed=0)
    maxit = max(1, (args.precision_sweeps - 1) // 2)

    def rel(a, b, mask=None):
        if mask is not None:
            a, b = a[mask], b[mask]
        d = float(np.linalg.norm((a - b).ravel()))
        return {"rel_l2": d / max(float(np.linalg.norm(b.ravel())), 1e-300),
                "max_rel": float(np.abs(a - b).max()) / max(float(np.abs(b).max()), 1e-300)}

    def timed(fn, stream):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1)

    out = {"workload": f"precision {n}^3 open box, blob charge", "sweeps_compared": 2 * maxit + 1}
    g64 = Simulation(p, layout=capi.LAYOUT_F64, solver=capi.SOLVER_F64)
    s64 = torch.cuda.ExternalStream(g64.stream_handle)
    g64.calc_distance()
    g64.set_field(capi.FIELD_C, C)
    g64.set_option(capi.OPT_BCPOT_TENSOR, 0)
    out["bcpot_fp64_ms"] = timed(g64.bc_potentials, s64)
    Ub64 = g64.field(capi.FIELD_U)
    g64.set_option(capi.OPT_BCPOT_TENSOR, 1)
    out["bcpot_tensor_ms"] = timed(g64.bc_potentials, s64)
    Ubtc = g64.field(capi.FIELD_U)
    g64.set_option(capi.OPT_BCPOT_TENSOR, 2)
    g64.bc_potentials()  # the first call after CalcDistance also transforms the slices of D
    out["bcpot_fft_ms"] = timed(g64.bc_potentials, s64)
    Ubfft = g64.field(capi.FIELD_U)
    face = Ub64 != 0.0
    out["boundary"] = rel(Ubtc, Ub64, face)
    out["boundary_fft"] = rel(Ubfft, Ub64, face)
    out["face_nodes"] = int(face.sum())
    # FP64 Jacobi from the FP64 boundary potential
    g64.set_field(capi.FIELD_U, Ub64)
    out["jacobi_fp64_ms"] = timed(lambda: g64.calc_epotential(maxerr=1e-300, maxit=maxit), s64)
    U64 = g64.field(capi.FIELD_U)
    g64.close()
    g32 = Simulation(p, layout=capi.LAYOUT_F64, solver=capi.SOLVER_F32_REFINE)
    s32 = torch.cuda.ExternalStream(g32.stream_handle)
    g32.set_field(capi.FIELD_C, C)
    g32.set_field(capi.FIELD_U, Ub64)
    out["jacobi_fp32_refine_ms"] = timed(lambda: g32.calc_epotential(maxerr=1e-300, maxit=maxit), s32)
    U32 = g32.field(capi.FIELD_U)
    out["jacobi"] = rel(U32, U64)
    g32.set_field(capi.FIELD_U, Ubtc)
    g32.calc_epotential(maxerr=1e-300, maxit=maxit)
    Ue2e = g32.field(capi.FIELD_U)
    out["end_to_end"] = rel(Ue2e, U64)
    g32.close()
    gsp = Simulation(p, layout=capi.LAYOUT_F64, solver=capi.SOLVER_SPECTRAL)
    ssp = torch.cuda.ExternalStream(gsp.stream_handle)
    gsp.set_field(capi.FIELD_C, C)
    gsp.set_field(capi.FIELD_U, Ub64)
    out["jacobi_closed_form_ms"] = timed(lambda: gsp.calc_epotential(maxerr=1e-300, maxit=maxit), ssp)
    out["jacobi_closed_form"] = rel(gsp.field(capi.FIELD_U), U64)
    gsp.set_field(capi.FIELD_U, Ubfft)
    gsp.calc_epotential(maxerr=1e-300, maxit=maxit)
    out["end_to_end_fft_closed_form"] = rel(gsp.field(capi.FIELD_U), U64)
    gsp.close()
    print(json.dumps(out), flush=True)


def run_batch(args, local_rank):
    print(json.dumps(batch_measure(args, local_rank, args.runs, args.run_steps)), flush=True)


def batch_measure(args, local_rank, nruns: int, run_steps: int) -> dict:
    """Batched parameter sweep: `nruns` independent runs (cubic grids 16..96
    cells, 8..32 ppc, drift 300..800 km/s, |B| 1..10 nT in a random direction,
    `run_steps` iterations each, CELL32 / F32_REFINE) advanced two ways:
      plain:   one run after another through picard_gpu_run, the
               per-subroutine call sequence of picard.f90 (the drop-in loop);
      fused:   one run after another through picard_gpu_run_fused (the
               single-run loop the batch and the server build on);
      batched: all runs together through picard_batch_run_fused (one sweep
               launch per sweep for every run).
    Every arm creates, initialises, runs and releases every run inside its
    timed region (the sweep launch tuner runs at creation).  Reports
    particle-steps/s of each arm and checks that every batched run ends bit
    for bit where the fused loop ends it alone (the per-subroutine loop plans
    its FP32 rounds differently, so its potentials agree to the solver's
    tolerance, not bit for bit)."""
    import numpy as np
    import torch

    from picard_b200 import capi
    from picard_b200 import params as P
    from picard_b200.simulation import Simulation, batch_run_fused

    torch.cuda.set_device(local_rank)
    sets = P.batch_set(seed=0, count=nruns)
    runs = []
    for p, steps in sets:
        if run_steps != steps:
            p = P._size_capacity(p, run_steps, max(1, int(p.ppc[1])))
        runs.append(capi.params_derive(p))
    steps = run_steps
    layout, solver = capi.LAYOUT_CELL32, SOLVERS[args.solver]
    # warm-up, untimed: kernels loaded, and the sweep launch tuner run once per
    # grid shape (its choices are cached for the process), so that neither
    # arm pays for tuning
    w = Simulation(runs[0], derive=False, layout=layout, solver=solver)
    w.calc_distance()
    w.particles_initialize()
    w.run_fused(0, 1)
    w.close()
    seen = set()
    for p in runs:
        if (p.nx, p.ny, p.nz) not in seen:
            seen.add((p.nx, p.ny, p.nz))
            Simulation(p, derive=False, layout=layout, solver=solver).close()
    torch.cuda.synchronize()
    visible = os.environ.get("CUDA_VISIBLE_DEVICES")
    clocks = ClockSampler(int(visible.split(",")[local_rank]) if visible else local_rank)
    clocks.start()
    t0 = time.perf_counter()
    sub = []
    for p in runs:
        g = Simulation(p, derive=False, layout=layout, solver=solver)
        g.calc_distance()
        g.particles_initialize()
        g.run(0, steps)
        sub.append({"particle_steps": g.stats()["particle_steps"], "u": float(np.abs(g.field(capi.FIELD_U)).sum())})
        g.close()
    torch.cuda.synchronize()
    t_sub = time.perf_counter() - t0
    t0 = time.perf_counter()
    plain = []
    plain_phase = {}
    for p in runs:
        g = Simulation(p, derive=False, layout=layout, solver=solver)
        g.calc_distance()
        g.particles_initialize()
        sw = g.run_fused(0, steps)
        st = g.stats()
        for k, v in st["phase_ms"].items():
            plain_phase[k] = plain_phase.get(k, 0.0) + v
        plain.append({"sweeps": sw, "particle_steps": st["particle_steps"],
                      "u": float(np.abs(g.field(capi.FIELD_U)).sum()), "n": g.num_local})
        g.close()
    torch.cuda.synchronize()
    t_plain = time.perf_counter() - t0
    t0 = time.perf_counter()
    sims = []
    for p in runs:
        g = Simulation(p, derive=False, layout=layout, solver=solver)
        g.calc_distance()
        g.particles_initialize()
        sims.append(g)
    sweeps = batch_run_fused(sims, 0, steps)
    batched = []
    for g, sw in zip(sims, sweeps):
        batched.append({"sweeps": sw, "particle_steps": g.stats()["particle_steps"],
                        "u": float(np.abs(g.field(capi.FIELD_U)).sum()), "n": g.num_local})
        g.close()
    torch.cuda.synchronize()
    t_batch = time.perf_counter() - t0
    clk = clocks.stop()
    mism = [{"run": k, "grid": int(runs[k].nx), "sweeps": [a["sweeps"], b["sweeps"]], "n": [a["n"], b["n"]],
             "u_rel": abs(a["u"] - b["u"]) / max(abs(a["u"]), 1e-300)}
            for k, (a, b) in enumerate(zip(plain, batched))
            if not (a["u"] == b["u"] and a["n"] == b["n"] and a["sweeps"] == b["sweeps"])]
    same = not mism
    ps_plain = sum(r["particle_steps"] for r in plain)
    ps_batch = sum(r["particle_steps"] for r in batched)
    ps_sub = sum(r["particle_steps"] for r in sub)
    line = {
        "metric": "particle-steps/s, batched vs plain", "value": ps_batch / t_batch, "unit": UNIT, "n_gpus": 1,
        "higher_is_better": True, "impl": "picard", "workload": "batch", "vs_baseline": None,
        "dtype": dtype_of(args),
        "data": "synthetic (seeded Philox plasma, run seeds 0..runs-1)",
        "config": {"workload": f"batched parameter sweep: {len(runs)} runs, cubic grids 16..96 cells, 8..32 ppc, "
                               f"drift 300..800 km/s, |B| 1..10 nT random direction, {steps} steps each",
                   "grids": [int(p.nx) for p in runs]},
        "batched": {"particle_steps_per_s": ps_batch / t_batch, "seconds": t_batch},
        "plain": {"particle_steps_per_s": ps_sub / t_sub, "seconds": t_sub,
                  "loop": "picard_gpu_run (per-subroutine calls)",
                  "u_abs_sum_max_rel_diff_vs_batched": max(abs(a["u"] - b["u"]) / max(abs(b["u"]), 1e-300)
                                                            for a, b in zip(sub, batched))},
        "fused": {"particle_steps_per_s": ps_plain / t_plain, "seconds": t_plain,
                  "loop": "picard_gpu_run_fused", "phase_ms": {k: round(v, 1) for k, v in plain_phase.items()}},
        "batched_over_plain": (ps_batch / t_batch) / (ps_sub / t_sub),
        "batched_over_fused": (ps_batch / t_batch) / (ps_plain / t_plain),
        "jacobi_sweeps_total": sum(r["sweeps"] for r in batched),
        "jacobi_node_sweeps": sum(r["sweeps"] * int(p.nx) * int(p.ny) * int(p.nz) for r, p in zip(batched, runs)),
        "jacobi_sweeps_per_run": [r["sweeps"] for r in batched],
        "results_identical_to_fused": same,
        "mismatches": mism[:8],
        "clocks": clk,
    }
    return line


def run_bcpot(args, local_rank):
    """Tensor-core BCpotentials alone: one context on --poisson-dims (default
    256,128,128) with a random charge; device time per call (3 axes)."""
    import numpy as np
    import torch

    from picard_b200 import capi
    from picard_b200 import params as P
    from picard_b200.simulation import Simulation

    torch.cuda.set_device(local_rank)
    nx, ny, nz = [int(v) for v in (args.poisson_dims or "256,128,128").split(",")]
    p = P.config_plain_32(n=8, ppc=1, capacity=1024)
    p.nx, p.ny, p.nz = nx, ny, nz
    p.xmin, p.xmax = -500.0 * nx, 500.0 * nx
    p.ymin, p.ymax = -500.0 * ny, 500.0 * ny
    p.zmin, p.zmax = -500.0 * nz, 500.0 * nz
    sim = Simulation(p, layout=capi.LAYOUT_F64, solver=capi.SOLVER_F64)
    sim.calc_distance()
    rng = np.random.default_rng(0)
    C = np.zeros((nz + 2, ny + 2, nx + 2))
    C[1:-1, 1:-1, 1:-1] = rng.normal(size=(nz, ny, nx)) * 1e-15
    sim.set_field(capi.FIELD_C, C)
    sim.set_option(capi.OPT_BCPOT_TENSOR, 1)
    ext = torch.cuda.ExternalStream(sim.stream_handle)
    sim.bc_potentials()
    sim.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    reps = max(1, args.steps)
    e0.record(ext)
    for _ in range(reps):
        sim.bc_potentials()
    e1.record(ext)
    e1.synchronize()
    ms = e0.elapsed_time(e1) / reps
    faces = 2 * (ny * nz + nx * nz + nx * ny)
    flops = 2.0 * 6 * faces * nx * ny * nz  # six split products
    print(json.dumps({"workload": f"bcpot {nx}x{ny}x{nz}", "bcpot_tc_ms": ms,
                      "split_product_tflops": flops / (ms * 1e-3) / 1e12}), flush=True)
    sim.close()


def run_deposit(args, local_rank):
    """CELL32 ParticlesGridify alone on the at-scale grid (or --deposit-dims)
    with --ppc ions per cell (default 32), after two fused steps; device time
    per call."""
    import torch

    from picard_b200 import capi
    from picard_b200 import params as P
    from picard_b200.simulation import Simulation

    torch.cuda.set_device(local_rank)
    ppc = args.ppc or 32
    nx, ny, nz = (int(v) for v in (args.deposit_dims or "256,128,128").split(","))
    sim = Simulation(P.config_plain_scale(seed=0, nx=nx, ny=ny, nz=nz, ppc_ion=ppc), layout=capi.LAYOUT_CELL32,
                     solver=capi.SOLVER_SPECTRAL)
    sim.calc_distance()
    sim.particles_initialize()
    sim.run_fused(0, 2)
    ext = torch.cuda.ExternalStream(sim.stream_handle)
    sim.particles_gridify()
    sim.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    reps = max(1, args.steps)
    e0.record(ext)
    for _ in range(reps):
        sim.particles_gridify()
    e1.record(ext)
    e1.synchronize()
    ms = e0.elapsed_time(e1) / reps
    n = sim.num_local
    print(json.dumps({"workload": f"deposit {nx}x{ny}x{nz}, {ppc}+{ppc} ppc", "particles": n, "gridify_ms": ms,
                      "read_gbs": 17.0 * n / (ms * 1e-3) / 1e9}), flush=True)
    sim.close()


def run_reference(args, rank, world):
    """The reference arm: one complete full-size iteration of the loop
    (picard.f90:554-674) on the FP64 CPU oracle with every host thread --
    every phase in full (BCpotentials over every face node, Jacobi to the
    reference's stopping rule), nothing sampled or extrapolated.  The untimed
    warm-up is the oracle's setup (CalcDistance, ParticlesInitialize).  The
    K timed steps together perform that one iteration (each step is 1/K of
    its work), so ms_per_step = T/K and value = particles x 1 iteration / T.
    Under torchrun only rank 0 runs."""
    if rank != 0:
        return
    from oracle import oracle as O

    W, K = args.warmup, args.steps
    threads = os.cpu_count() or 1
    O.set_threads(threads)
    p, desc = workload(args.workload, seed=0)
    p = O.derive(p)
    s = O.OracleState(p)
    t0 = time.perf_counter()
    s.calc_distance()
    s.initialize()
    setup_s = time.perf_counter() - t0
    it = 1
    ph = {}

    def timed(name, fn):
        a = time.perf_counter()
        r = fn()
        ph[name] = time.perf_counter() - a
        return r

    timed("inflow", lambda: s.bc_inflow(it))
    timed("advance", lambda: s.advance_position())
    timed("produce", lambda: s.produce(it))
    timed("outflow", lambda: s.bc_outflow())
    timed("transfer", lambda: s.transfer())
    timed("gridify", lambda: s.gridify())
    timed("bcpot", lambda: s.bc_potentials())
    sweeps, conv, _ = timed("jacobi", lambda: s.calc_epotential())
    timed("efield", lambda: (s.calc_efield(), s.bc_fields()))
    timed("velocity", lambda: s.advance_velocity())
    total = sum(ph.values())
    particle_steps = s.num_local
    value = particle_steps / total
    sample = (f"one complete full-size iteration (iteration 1 after ParticlesInitialize, {particle_steps} "
              f"particles) on the FP64 oracle with {threads} threads: every phase in full, BCpotentials over all "
              f"face nodes, Jacobi {sweeps} sweeps to the reference's stopping rule (converged: {conv}); the "
              f"{K} timed steps together are that iteration (each 1/{K} of its work); warm-up = the oracle's "
              f"setup ({setup_s:.1f} s, untimed)")
    cpu = {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample,
           "seconds_per_iteration": total, "phase_seconds": {k: round(v, 4) for k, v in ph.items()},
           "jacobi_sweeps": sweeps}
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
        "ms_per_step": total * 1e3 / K, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded Philox plasma, seed 0)",
        "config": line_config(desc, world),
        "impl": "reference",
        "arithmetic": "FP64 particles (reference layout), FP64 BCpotentials and Jacobi",
        "cpu_baseline": cpu,
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def line_config(desc: dict, world: int) -> dict:
    """The workload named in both arms' lines (implementation choices such as
    the particle layout and the solver precision are reported beside it)."""
    return dict(desc, runs_per_gpu=1, parallelism=f"independent runs x{world}")


def main():
    args = parse_args()
    rank, world, local_rank = env_rank()
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    # every arm creates and releases contexts: let the stream-ordered pool keep
    # freed memory for reuse (as the serving loop does for its budget), so that
    # no arm maps memory afresh for each run
    from picard_b200 import capi

    capi.pool_keep(local_rank, int(args.budget_gb * 1e9))
    if args.workload == "poisson":
        run_poisson(args, local_rank)
        return
    if args.workload in ("bcpot", "deposit"):
        if rank == 0:
            (run_bcpot if args.workload == "bcpot" else run_deposit)(args, local_rank)
        return
    if args.workload == "batch":
        if rank == 0:
            run_batch(args, local_rank)
        return
    if args.workload == "precision":
        if rank == 0:
            run_precision(args, local_rank)
        return
    if args.workload == "serving":
        if rank == 0:
            run_serving(args, local_rank)
        return
    if world > 1:
        import torch
        import torch.distributed as dist

        backend = "nccl" if torch.cuda.is_available() else "gloo"
        dist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=300))
    try:
        run_picard(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
