"""ctypes bindings of the FP64 CPU oracle (liboracle.so built from picard_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() to
compare against, and by bench.py's CPU-baseline leg.  The product never imports it.
PARITY UNPINNED: the reference (Fortran 90 + MPI) cannot be built here and
ships no golden vectors; the restatement is pinned by physics known-answer
tests and the published Philox4x32-10 vectors instead.

Arrays use the reference layouts (column-major, species/components fastest):
real_particles (8, n) -> numpy (n, 8) C-order; U/C (Nx+2, Ny+2, Nz+2) -> numpy
(Nz+2, Ny+2, Nx+2); E (3, ...) -> (Nz+2, Ny+2, Nx+2, 3); N (S, ...) ->
(Nz+2, Ny+2, Nx+2, S).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from picard_b200.params import PicardParams

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None


def build() -> str:
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        P = C.POINTER(PicardParams)
        dp = C.POINTER(C.c_double)
        ip = C.POINTER(C.c_int32)
        L.orc_philox4x32_10.argtypes = [C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]
        L.orc_site_uniform.argtypes = [C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32]
        L.orc_site_uniform.restype = C.c_double
        L.orc_set_threads.argtypes = [C.c_int]
        L.orc_max_threads.restype = C.c_int
        L.orc_derive_params.argtypes = [P]
        L.orc_calc_distance.argtypes = [P, dp]
        L.orc_particles_initialize.argtypes = [P, dp, ip, ip]
        L.orc_particles_initialize.restype = C.c_int
        L.orc_bc_inflow.argtypes = [P, C.c_int, dp, ip, ip]
        L.orc_bc_inflow.restype = C.c_int
        L.orc_advance_position.argtypes = [dp, C.c_double, C.c_int32]
        L.orc_particles_produce.argtypes = [P, C.c_int, dp, ip, ip]
        L.orc_particles_produce.restype = C.c_int
        L.orc_bc_outflow.argtypes = [P, dp, ip, ip]
        L.orc_particles_transfer.argtypes = [P, dp, C.c_int32]
        L.orc_cell_indices.argtypes = [P, dp, C.c_int32, ip]
        L.orc_particles_gridify.argtypes = [P, dp, ip, C.c_int32, dp, dp]
        L.orc_particles_gridify_all.argtypes = [P, dp, ip, C.c_int32, dp, dp, dp]
        L.orc_bc_potentials.argtypes = [P, dp, dp, dp]
        L.orc_bc_potentials_sampled.argtypes = [P, dp, dp, dp, C.c_int]
        L.orc_calc_epotential.argtypes = [P, dp, dp, C.c_double, C.c_int, C.POINTER(C.c_int), dp]
        L.orc_calc_epotential.restype = C.c_int
        L.orc_calc_efield.argtypes = [P, dp, dp]
        L.orc_bc_fields.argtypes = [P, dp]
        L.orc_advance_velocity.argtypes = [P, dp, ip, C.c_int32, dp, C.c_double, C.c_double, C.c_int]
        L.orc_energy.argtypes = [P, dp, ip, C.c_int32, dp, dp]
        L.orc_step.argtypes = [P, C.c_int, dp, ip, ip, dp, dp, dp, dp, dp]
        L.orc_step.restype = C.c_int
        _lib = L
    return _lib


def _d(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _i(a: np.ndarray):
    assert a.dtype == np.int32 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_int32))


def philox4x32_10(ctr, key):
    c = (C.c_uint32 * 4)(*ctr)
    k = (C.c_uint32 * 2)(*key)
    o = (C.c_uint32 * 4)()
    lib().orc_philox4x32_10(c, k, o)
    return [int(x) for x in o]


def site_uniform(seed, a, b, it, tag, n):
    return lib().orc_site_uniform(seed, a, b, it, tag, n)


def set_threads(n: int) -> None:
    lib().orc_set_threads(n)


def max_threads() -> int:
    return lib().orc_max_threads()


def derive(p: PicardParams) -> PicardParams:
    q = p.copy()
    lib().orc_derive_params(C.byref(q))
    return q


class OracleState:
    """Reference-layout state arrays of one run plus the per-routine calls of
    the main loop (picard.f90:554-631)."""

    def __init__(self, p: PicardParams):
        self.p = p
        nxp, nyp, nzp = p.nx + 2, p.ny + 2, p.nz + 2
        S = p.species
        self.rp = np.zeros((p.max_per_proc, 8), np.float64)
        self.ip = np.zeros(p.max_per_proc, np.int32)
        self.num = C.c_int32(0)
        self.D = np.zeros((2 * p.nz + 1, 2 * p.ny + 1, 2 * p.nx + 1), np.float64)
        self.U = np.zeros((nzp, nyp, nxp), np.float64)
        self.E = np.zeros((nzp, nyp, nxp, 3), np.float64)
        self.N = np.zeros((nzp, nyp, nxp, S), np.float64)
        self.F = np.zeros((nzp, nyp, nxp, 3, S), np.float64)
        self.C = np.zeros((nzp, nyp, nxp), np.float64)
        self.last_sweeps = 0

    @property
    def num_local(self) -> int:
        return self.num.value

    def set_particles(self, rp: np.ndarray, ip: np.ndarray) -> None:
        n = rp.shape[0]
        self.rp[:n] = rp
        self.ip[:n] = ip
        self.num.value = n

    def particles(self):
        n = self.num.value
        return self.rp[:n].copy(), self.ip[:n].copy()

    def calc_distance(self):
        lib().orc_calc_distance(C.byref(self.p), _d(self.D))

    def initialize(self):
        rc = lib().orc_particles_initialize(C.byref(self.p), _d(self.rp), _i(self.ip), C.byref(self.num))
        if rc:
            raise RuntimeError("oracle: capacity exceeded")

    def bc_inflow(self, iteration: int):
        rc = lib().orc_bc_inflow(C.byref(self.p), iteration, _d(self.rp), _i(self.ip), C.byref(self.num))
        if rc:
            raise RuntimeError("oracle: capacity exceeded")

    def advance_position(self, dt: float | None = None):
        lib().orc_advance_position(_d(self.rp), self.p.dt if dt is None else dt, self.num.value)

    def produce(self, iteration: int):
        rc = lib().orc_particles_produce(C.byref(self.p), iteration, _d(self.rp), _i(self.ip), C.byref(self.num))
        if rc:
            raise RuntimeError("oracle: capacity exceeded")

    def bc_outflow(self):
        lib().orc_bc_outflow(C.byref(self.p), _d(self.rp), _i(self.ip), C.byref(self.num))

    def transfer(self):
        lib().orc_particles_transfer(C.byref(self.p), _d(self.rp), self.num.value)

    def cell_indices(self) -> np.ndarray:
        n = self.num.value
        out = np.zeros((n, 3), np.int32)
        lib().orc_cell_indices(C.byref(self.p), _d(self.rp), n, _i(out))
        return out

    def gridify(self):
        lib().orc_particles_gridify(C.byref(self.p), _d(self.rp), _i(self.ip), self.num.value, _d(self.N), _d(self.C))

    def gridify_all(self):
        lib().orc_particles_gridify_all(C.byref(self.p), _d(self.rp), _i(self.ip), self.num.value, _d(self.F),
                                        _d(self.N), _d(self.C))

    def bc_potentials(self):
        lib().orc_bc_potentials(C.byref(self.p), _d(self.U), _d(self.C), _d(self.D))

    def bc_potentials_sampled(self, stride: int):
        lib().orc_bc_potentials_sampled(C.byref(self.p), _d(self.U), _d(self.C), _d(self.D), stride)

    def calc_epotential(self, maxerr: float | None = None, maxit: int | None = None):
        conv = C.c_int(0)
        res = np.zeros(2, np.float64)
        s = lib().orc_calc_epotential(C.byref(self.p), _d(self.U), _d(self.C),
                                      self.p.maxerr if maxerr is None else maxerr,
                                      self.p.maxit if maxit is None else maxit, C.byref(conv), _d(res))
        self.last_sweeps = s
        return s, bool(conv.value), res

    def calc_efield(self):
        lib().orc_calc_efield(C.byref(self.p), _d(self.E), _d(self.U))

    def bc_fields(self):
        lib().orc_bc_fields(C.byref(self.p), _d(self.E))

    def advance_velocity(self, mode: int = 0, deltat: float = 0.0, dt: float | None = None):
        lib().orc_advance_velocity(C.byref(self.p), _d(self.rp), _i(self.ip), self.num.value, _d(self.E),
                                   self.p.dt if dt is None else dt, deltat, mode)

    def energy(self):
        out = np.zeros(3, np.float64)
        lib().orc_energy(C.byref(self.p), _d(self.rp), _i(self.ip), self.num.value, _d(self.E), _d(out))
        return out

    def step(self, iteration: int) -> int:
        s = lib().orc_step(C.byref(self.p), iteration, _d(self.rp), _i(self.ip), C.byref(self.num), _d(self.D),
                           _d(self.U), _d(self.E), _d(self.N), _d(self.C))
        if s < 0:
            raise RuntimeError("oracle: capacity exceeded")
        self.last_sweeps = s
        return s


# ------------------------------------------------------------------ dumps

def format_e(value: float, w: int = 10, d: int = 4) -> str:
    """Fortran Ew.d editing with scale factor 0 (Fortran 2008 10.7.2.3.3), as
    Write.f90 uses it: 0.d1..dd E+ee with the mantissa correctly rounded, the
    optional leading zero dropped when the sign needs its column, the E
    dropped for three-digit exponents, gfortran's NaN / Infinity words right
    justified, and w asterisks when the field is too narrow."""
    import math

    if math.isnan(value):
        s = "NaN"
    elif math.isinf(value):
        s = "Infinity" if value > 0 else "-Infinity"
    else:
        neg = math.copysign(1.0, value) < 0 and value != 0.0
        if value == 0.0:
            digits, exp = "0" * d, 0
        else:
            m = f"{abs(value):.{d - 1}e}"          # correctly rounded d digits
            mant, e = m.split("e")
            digits = mant.replace(".", "")
            exp = int(e) + 1                       # 0.d1d2.. x 10^exp
        ex = f"E{'-' if exp < 0 else '+'}{abs(exp):02d}" if abs(exp) <= 99 else f"{'-' if exp < 0 else '+'}{abs(exp):03d}"
        body = "." + digits + ex
        s = ("-" if neg else "") + ("0" + body if len(body) + (1 if neg else 0) < w else body)
    return s.rjust(w) if len(s) <= w else "*" * w


def dump_particles(rp: np.ndarray, ip: np.ndarray, root: str, iteration: int) -> int:
    """Write.f90:2-31: real_particles(1:7, 1:num_local) with column 7 = the
    species number, 7E10.4 (one particle per line), to
    root/particles/particles_IIIII_00000; returns the next file number."""
    d = os.path.join(root, "particles")
    os.makedirs(d, exist_ok=True)
    with open(os.path.join(d, f"particles_{iteration:05d}_00000"), "w") as f:
        for row, s in zip(rp, ip):
            f.write("".join(format_e(float(v)) for v in row[:6]) + format_e(float(s)) + "\n")
    return iteration + 1


def dump_fields(st: "OracleState", root: str, iteration: int) -> int:
    """Write.f90:34-523: UE, Ex, Ey, Ez, then N#, X#, Y#, Z# for species
    1..species, one E10.4 value per line in x-fastest order (ghost nodes
    included), to root/fields/NAME_IIIII_00000; returns the next file
    number."""
    d = os.path.join(root, "fields")
    os.makedirs(d, exist_ok=True)
    arrays = [("UE", st.U), ("Ex", st.E[..., 0]), ("Ey", st.E[..., 1]), ("Ez", st.E[..., 2])]
    S = st.p.species
    arrays += [(f"N{s + 1}", st.N[..., s]) for s in range(S)]
    for c, comp in (("X", 0), ("Y", 1), ("Z", 2)):
        arrays += [(f"{c}{s + 1}", st.F[..., comp, s]) for s in range(S)]
    for name, a in arrays:
        with open(os.path.join(d, f"{name}_{iteration:05d}_00000"), "w") as f:
            f.write("".join(format_e(float(v)) + "\n" for v in a.ravel()))
    return iteration + 1
