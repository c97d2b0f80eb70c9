"""Host-side mirror of the reference's subroutine interface over the C ABI.

``Simulation`` owns one device context.  Its methods are the reference's
subroutines (picard.f90:554-674 calls them in this order) with the reference's
argument meaning; state arrays live on the device and are copied in the
reference layouts by ``particles()`` / ``set_particles()`` / ``field()`` /
``set_field()``.  numpy shapes: real_particles (8, n) column-major is returned
as (n, 8); U and C (Nx+2, Ny+2, Nz+2) as (Nz+2, Ny+2, Nx+2); E (3, ...) as
(Nz+2, Ny+2, Nx+2, 3); N (S, ...) as (Nz+2, Ny+2, Nx+2, S); F (S, 3, ...) as
(Nz+2, Ny+2, Nx+2, 3, S).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import capi
from .params import PicardParams


class Simulation:
    def __init__(self, params: PicardParams, layout: int = capi.LAYOUT_CELL32,
                 solver: int = capi.SOLVER_F32_REFINE, derive: bool = True):
        self.p = capi.params_derive(params) if derive else params.copy()
        self.layout = layout
        self.solver = solver
        h = C.c_void_p()
        capi.check(capi.lib().picard_gpu_create(C.byref(self.p), layout, solver, C.byref(h)), "picard_gpu_create")
        self._h = h
        self.last_sweeps = 0

    # ------------------------------------------------------------ lifecycle
    def close(self) -> None:
        if self._h is not None and self._h.value:
            capi.lib().picard_gpu_destroy(self._h)
        self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _call(self, name: str, *args, allow=(capi.OK,)) -> int:
        return capi.check(getattr(capi.lib(), name)(self._h, *args), name, allow)

    def set_option(self, option: int, value: int) -> None:
        self._call("picard_gpu_set_option", option, value)

    def get_option(self, option: int) -> int:
        v = C.c_int32(0)
        self._call("picard_gpu_get_option", option, C.byref(v))
        return int(v.value)

    def synchronize(self) -> None:
        self._call("picard_gpu_synchronize")

    # ------------------------------------------------------------ transfers
    @property
    def num_local(self) -> int:
        n = C.c_int32(0)
        self._call("picard_gpu_get_num_local", C.byref(n))
        return n.value

    def set_particles(self, rp: np.ndarray, ip: np.ndarray) -> None:
        rp = np.ascontiguousarray(rp, dtype=np.float64)
        ip = np.ascontiguousarray(ip, dtype=np.int32)
        assert rp.ndim == 2 and rp.shape[1] == 8 and ip.shape == (rp.shape[0],)
        self._call("picard_gpu_set_particles", rp.ctypes.data_as(C.POINTER(C.c_double)),
                   ip.ctypes.data_as(C.POINTER(C.c_int32)), rp.shape[0])

    def particles(self):
        n = self.num_local
        rp = np.zeros((max(n, 1), 8), np.float64)
        ip = np.zeros(max(n, 1), np.int32)
        got = C.c_int32(0)
        self._call("picard_gpu_get_particles", rp.ctypes.data_as(C.POINTER(C.c_double)),
                   ip.ctypes.data_as(C.POINTER(C.c_int32)), rp.shape[0], C.byref(got))
        return rp[:got.value], ip[:got.value]

    def _shape(self, which: int):
        p = self.p
        box = (p.nz + 2, p.ny + 2, p.nx + 2)
        if which in (capi.FIELD_U, capi.FIELD_C):
            return box
        if which == capi.FIELD_E:
            return box + (3,)
        if which == capi.FIELD_N:
            return box + (p.species,)
        if which == capi.FIELD_F:
            return box + (3, p.species)
        if which == capi.FIELD_D:
            return (2 * p.nz + 1, 2 * p.ny + 1, 2 * p.nx + 1)
        raise ValueError(which)

    def field(self, which: int) -> np.ndarray:
        out = np.zeros(self._shape(which), np.float64)
        self._call("picard_gpu_get_field", which, out.ctypes.data_as(C.POINTER(C.c_double)))
        return out

    def set_field(self, which: int, arr: np.ndarray) -> None:
        a = np.ascontiguousarray(arr, dtype=np.float64)
        assert a.shape == self._shape(which)
        self._call("picard_gpu_set_field", which, a.ctypes.data_as(C.POINTER(C.c_double)))

    # ------------------------------------------- the reference's subroutines
    def calc_distance(self):                       # CalcDistance.f90:1
        self._call("picard_gpu_calc_distance")

    def particles_initialize(self):                # ParticlesInitialize.f90:2
        self._call("picard_gpu_particles_initialize")

    def bc_inflow(self, iteration: int):           # BCinflow.f90:2
        self._call("picard_gpu_bc_inflow", iteration)

    def advance_position(self, dt: float | None = None):   # AdvancePosition.f90:4
        self._call("picard_gpu_advance_position", self.p.dt if dt is None else dt)

    def particles_produce(self, iteration: int):   # ParticlesProduce.f90:1
        self._call("picard_gpu_particles_produce", iteration)

    def bc_outflow(self):                          # BCoutflow.f90:5
        self._call("picard_gpu_bc_outflow")

    def particles_transfer(self):                  # ParticlesTransfer.f90:2
        self._call("picard_gpu_particles_transfer")

    def sort_particles(self):                      # no reference counterpart
        self._call("picard_gpu_sort_particles")

    def particles_gridify(self):                   # ParticlesGridify.f90:1
        self._call("picard_gpu_particles_gridify")

    def particles_gridify_all(self):               # ParticlesGridifyAll.f90:1
        self._call("picard_gpu_particles_gridify_all")

    def bc_potentials(self):                       # BCpotentials.f90:1
        self._call("picard_gpu_bc_potentials")

    def calc_epotential(self, maxerr: float | None = None, maxit: int | None = None) -> int:   # CalcEpotential.f90:4
        sw = C.c_int32(0)
        self._call("picard_gpu_calc_epotential", self.p.maxerr if maxerr is None else maxerr,
                   self.p.maxit if maxit is None else maxit, C.byref(sw),
                   allow=(capi.OK, capi.ERR_NOT_CONVERGED))
        self.last_sweeps = sw.value
        return sw.value

    def calc_efield(self):                         # CalcEfield.f90:3
        self._call("picard_gpu_calc_efield")

    def bc_fields(self):                           # BCfields.f90:3
        self._call("picard_gpu_bc_fields")

    def advance_velocity(self, dt: float | None = None):   # AdvanceVelocity.f90:6
        self._call("picard_gpu_advance_velocity", self.p.dt if dt is None else dt)

    def advance_velocity_exp(self, deltat: float, dt: float | None = None):   # AdvanceVelocity.f90:128
        self._call("picard_gpu_advance_velocity_exp", deltat, self.p.dt if dt is None else dt)

    def advance_velocity_imp(self, deltat: float, dt: float | None = None):   # AdvanceVelocity.f90:239
        self._call("picard_gpu_advance_velocity_imp", deltat, self.p.dt if dt is None else dt)

    def energy(self) -> np.ndarray:                # picard.f90:651-665 -> (uP, uE, uB)
        out = np.zeros(3, np.float64)
        n = C.c_int32(0)
        self._call("picard_gpu_energy", out.ctypes.data_as(C.POINTER(C.c_double)), C.byref(n))
        return out

    # ----------------------------------------------------------- statistics
    def stats(self) -> dict:
        st = capi.PicardStats()
        self._call("picard_gpu_get_stats", C.byref(st))
        return st.as_dict()

    def reset_stats(self) -> None:
        self._call("picard_gpu_reset_stats")

    @property
    def stream_handle(self) -> int:
        h = C.c_void_p()
        self._call("picard_gpu_get_stream", C.byref(h))
        return int(h.value or 0)

    # ------------------------------------------------------------ main loop
    def run(self, iter_start: int, iter_end: int, log_interval: int = 0, log=None) -> int:
        """picard.f90:554-674; returns the total Jacobi sweeps."""
        total = C.c_int64(0)
        cb = LOG_NONE if log is None else capi.LOG_FN(lambda it, t, n, up, ue, ub, _u: log(it, t, n, up, ue, ub))
        self._call("picard_gpu_run", iter_start, iter_end, log_interval, cb, None, C.byref(total),
                   allow=(capi.OK, capi.ERR_NOT_CONVERGED))
        return total.value

    def run_io(self, iter_start: int, iter_end: int, root: str, write_fields: bool = True,
               write_particles: bool = True, fields_interval: float | None = None,
               particles_interval: float | None = None, fields_iteration: int = 0, particles_iteration: int = 0,
               log_interval: int = 0, log=None) -> tuple[int, int, int]:
        """picard.f90:554-674 with the write-step branch (602-627) and the dumps
        of Write.f90 under ``root`` (the reference's ``save``).  Intervals are
        seconds (reference defaults 100 dt for fields, 1000 dt for particles).
        Returns (sweeps, next fields file number, next particles file number)."""
        io = capi.PicardIO()
        io.write_fields = 1 if write_fields else 0
        io.write_particles = 1 if write_particles else 0
        io.fields_interval = float(100.0 * self.p.dt if fields_interval is None else fields_interval)
        io.particles_interval = float(1000.0 * self.p.dt if particles_interval is None else particles_interval)
        io.fields_iteration = int(fields_iteration)
        io.particles_iteration = int(particles_iteration)
        io.root = root.encode()
        total = C.c_int64(0)
        cb = LOG_NONE if log is None else capi.LOG_FN(lambda it, t, n, up, ue, ub, _u: log(it, t, n, up, ue, ub))
        self._call("picard_gpu_run_io", iter_start, iter_end, log_interval, cb, None, C.byref(io), C.byref(total),
                   allow=(capi.OK, capi.ERR_NOT_CONVERGED))
        return total.value, io.fields_iteration, io.particles_iteration

    def dump_particles(self, root: str, write_iteration: int) -> int:   # Write.f90:1-31
        it = C.c_int32(write_iteration)
        self._call("picard_gpu_dump_particles", root.encode(), C.byref(it))
        return it.value

    def dump_fields(self, root: str, write_iteration: int) -> int:      # Write.f90:34-523
        it = C.c_int32(write_iteration)
        self._call("picard_gpu_dump_fields", root.encode(), C.byref(it))
        return it.value

    def run_fused(self, iter_start: int, iter_end: int) -> int:
        total = C.c_int64(0)
        self._call("picard_gpu_run_fused", iter_start, iter_end, C.byref(total),
                   allow=(capi.OK, capi.ERR_NOT_CONVERGED))
        return total.value


LOG_NONE = capi.LOG_FN()


def batch_run_fused(sims: "list[Simulation]", iter_start: int, iter_end: int) -> list[int]:
    """Advance independent runs together (picard_batch_run_fused): every run's
    particle phases issued before any is waited for, all runs' Jacobi sweeps
    in one launch per sweep.  Returns each run's Jacobi sweeps."""
    n = len(sims)
    arr = (C.c_void_p * n)(*[s._h.value for s in sims])
    sweeps = (C.c_int64 * n)()
    capi.check(capi.lib().picard_batch_run_fused(arr, n, iter_start, iter_end, sweeps), "picard_batch_run_fused",
               (capi.OK, capi.ERR_NOT_CONVERGED))
    return [int(v) for v in sweeps]


def batch_step(sims: "list[Simulation]", iterations: "list[int]") -> list[int]:
    """One main-loop iteration of each run together (picard_batch_step); run r
    takes iteration ``iterations[r]`` (1-based), so runs at different points of
    their loops share the step.  Returns each run's Jacobi sweeps."""
    n = len(sims)
    arr = (C.c_void_p * n)(*[s._h.value for s in sims])
    its = (C.c_int32 * n)(*[int(i) for i in iterations])
    sweeps = (C.c_int64 * n)()
    capi.check(capi.lib().picard_batch_step(arr, n, its, sweeps), "picard_batch_step",
               (capi.OK, capi.ERR_NOT_CONVERGED))
    return [int(v) for v in sweeps]
