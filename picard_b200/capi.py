"""ctypes binding of libpicard_gpu.so (include/picard_gpu.h).

The library is built in-tree (picard_b200/lib/libpicard_gpu.so, see build.py).
There is no CPU fallback: if the library is missing or the machine has no CUDA
device, the calls raise.
"""
from __future__ import annotations

import ctypes as C
import os

from .params import PicardParams

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libpicard_gpu.so")

OK = 0
ERR_BAD_ARG = 1
ERR_CAPACITY = 2
ERR_NOT_CONVERGED = 3
ERR_TIMEOUT = 4
ERR_CUDA = 5
ERR_STATE = 6
STATUS_NAMES = {0: "OK", 1: "BAD_ARG", 2: "CAPACITY", 3: "NOT_CONVERGED", 4: "TIMEOUT", 5: "CUDA", 6: "STATE"}

LAYOUT_F64 = 0
LAYOUT_CELL32 = 1
SOLVER_F64 = 0
SOLVER_F32_REFINE = 1
SOLVER_SPECTRAL = 2

FIELD_U, FIELD_E, FIELD_N, FIELD_C, FIELD_F, FIELD_D = range(6)
OPT_BCPOT_TENSOR = 0
OPT_SWEEP_CTAS = 1
OPT_SWEEP_PDL = 2
OPT_SWEEP_STAGES = 3
OPT_SWEEP_RESIDENT = 4
OPT_SWEEP_PAIRS = 5
OPT_SWEEP_FUSED = 6
OPT_WAIT_TEST = 7
OPT_SWEEP_R_GLOBAL = 8
OPT_SORT_EVERY = 9

class PicardStats(C.Structure):
    _fields_ = [
        ("kernel_launches", C.c_int64),
        ("solves", C.c_int64),
        ("sweeps", C.c_int64),
        ("sweep_launches", C.c_int64),
        ("sweep_ms", C.c_double),
        ("anchor_launches", C.c_int64),
        ("anchor_ms", C.c_double),
        ("last_residual", C.c_double),
        ("last_bnorm", C.c_double),
        ("steps", C.c_int64),
        ("particle_steps", C.c_int64),
        ("h2d_bytes", C.c_int64),
        ("d2h_bytes", C.c_int64),
        ("phase_ms", C.c_double * 5),
        ("last_sweeps", C.c_int64),
        ("spectral_transforms", C.c_int64),
        ("spectral_transform_ms", C.c_double),
    ]

    PHASES = ("particles", "deposit", "bc_potentials", "jacobi", "field_push")

    def as_dict(self) -> dict:
        d = {k: getattr(self, k) for k, _ in self._fields_ if k != "phase_ms"}
        d["phase_ms"] = {n: self.phase_ms[i] for i, n in enumerate(self.PHASES)}
        return d


class PicardRequest(C.Structure):
    """include/picard_server.h picard_request."""
    _fields_ = [
        ("id", C.c_int64),
        ("params", PicardParams),
        ("layout", C.c_int32),
        ("solver", C.c_int32),
        ("steps", C.c_int32),
        ("arrival_ms", C.c_double),
    ]


class PicardResult(C.Structure):
    """include/picard_server.h picard_result."""
    _fields_ = [
        ("id", C.c_int64),
        ("status", C.c_int32),
        ("num_local", C.c_int32),
        ("arrival_ms", C.c_double),
        ("start_ms", C.c_double),
        ("finish_ms", C.c_double),
        ("sweeps", C.c_int64),
        ("particle_steps", C.c_int64),
        ("energy", C.c_double * 3),
        ("u_sum", C.c_double),
        ("u_abs_sum", C.c_double),
        ("warnings", C.c_uint32),
        ("shard", C.c_int32),
    ]

    def as_dict(self) -> dict:
        d = {k: getattr(self, k) for k, _ in self._fields_ if k != "energy"}
        d["energy"] = tuple(self.energy)
        return d


class PicardPlasma(C.Structure):
    """include/picard_io.h picard_plasma."""
    _fields_ = [
        ("wp", C.c_double * 3), ("wc", C.c_double * 3), ("va", C.c_double), ("vc", C.c_double * 3),
        ("Ld", C.c_double * 3), ("rL", C.c_double * 3), ("rPU", C.c_double * 3), ("Li", C.c_double * 3),
        ("sd", C.c_double), ("rM", C.c_double * 3), ("cfl", C.c_double), ("freq", C.c_double),
        ("dt_c", C.c_double), ("dt_opt_part", C.c_double), ("dt_opt_wave", C.c_double), ("dt_opt", C.c_double),
        ("dt_rec", C.c_double), ("vth", C.c_double * 8), ("warnings", C.c_uint32),
    ]

    def as_dict(self) -> dict:
        out = {}
        for k, _ in self._fields_:
            v = getattr(self, k)
            out[k] = tuple(v) if hasattr(v, "__len__") else v
        return out


class PicardIO(C.Structure):
    """include/picard_io.h picard_io."""
    _fields_ = [
        ("write_fields", C.c_int32),
        ("write_particles", C.c_int32),
        ("fields_interval", C.c_double),
        ("particles_interval", C.c_double),
        ("fields_iteration", C.c_int32),
        ("particles_iteration", C.c_int32),
        ("root", C.c_char * 512),
    ]


WARN_COUNT = 17

LOG_FN = C.CFUNCTYPE(None, C.c_int32, C.c_double, C.c_int32, C.c_double, C.c_double, C.c_double, C.c_void_p)


class PicardError(RuntimeError):
    def __init__(self, code: int, where: str, message: str):
        super().__init__(f"{where}: {STATUS_NAMES.get(code, code)}: {message}")
        self.code = code


_lib = None


def lib():
    """Load libpicard_gpu.so; raise if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise FileNotFoundError(f"{LIB_PATH} is missing: build it with `python -m picard_b200.build`")
    L = C.CDLL(LIB_PATH)
    P = C.POINTER(PicardParams)
    ctx = C.c_void_p
    dp = C.POINTER(C.c_double)
    ip = C.POINTER(C.c_int32)
    sig = {
        "picard_params_default": [P],
        "picard_params_derive": [P],
        "picard_gpu_create": [P, C.c_int32, C.c_int32, C.POINTER(C.c_void_p)],
        "picard_gpu_destroy": [ctx],
        "picard_gpu_synchronize": [ctx],
        "picard_gpu_footprint": [P, C.c_int32, C.c_int32, C.POINTER(C.c_uint64)],
        "picard_gpu_pool_keep": [C.c_int32, C.c_uint64],
        "picard_gpu_set_particles": [ctx, dp, ip, C.c_int32],
        "picard_gpu_get_particles": [ctx, dp, ip, C.c_int32, ip],
        "picard_gpu_get_num_local": [ctx, ip],
        "picard_gpu_get_field": [ctx, C.c_int32, dp],
        "picard_gpu_set_field": [ctx, C.c_int32, dp],
        "picard_gpu_calc_distance": [ctx],
        "picard_gpu_particles_initialize": [ctx],
        "picard_gpu_bc_inflow": [ctx, C.c_int32],
        "picard_gpu_advance_position": [ctx, C.c_double],
        "picard_gpu_particles_produce": [ctx, C.c_int32],
        "picard_gpu_bc_outflow": [ctx],
        "picard_gpu_particles_transfer": [ctx],
        "picard_gpu_sort_particles": [ctx],
        "picard_gpu_particles_gridify": [ctx],
        "picard_gpu_particles_gridify_all": [ctx],
        "picard_gpu_bc_potentials": [ctx],
        "picard_gpu_calc_epotential": [ctx, C.c_double, C.c_int32, ip],
        "picard_gpu_calc_efield": [ctx],
        "picard_gpu_bc_fields": [ctx],
        "picard_gpu_advance_velocity": [ctx, C.c_double],
        "picard_gpu_advance_velocity_exp": [ctx, C.c_double, C.c_double],
        "picard_gpu_advance_velocity_imp": [ctx, C.c_double, C.c_double],
        "picard_gpu_energy": [ctx, dp, ip],
        "picard_gpu_run": [ctx, C.c_int32, C.c_int32, C.c_int32, LOG_FN, C.c_void_p, C.POINTER(C.c_int64)],
        "picard_gpu_run_fused": [ctx, C.c_int32, C.c_int32, C.POINTER(C.c_int64)],
        "picard_gpu_get_stats": [ctx, C.POINTER(PicardStats)],
        "picard_gpu_reset_stats": [ctx],
        "picard_gpu_get_stream": [ctx, C.POINTER(C.c_void_p)],
        "picard_gpu_set_option": [ctx, C.c_int32, C.c_int32],
        "picard_gpu_get_option": [ctx, C.c_int32, ip],
        "picard_batch_run_fused": [C.POINTER(C.c_void_p), C.c_int32, C.c_int32, C.c_int32, C.POINTER(C.c_int64)],
        "picard_batch_step": [C.POINTER(C.c_void_p), C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_int64)],
        "picard_server_create": [C.c_uint64, C.c_int32, C.POINTER(C.c_void_p)],
        "picard_server_create_batched": [C.c_uint64, C.c_int32, C.c_int32, C.POINTER(C.c_void_p)],
        "picard_server_create_multi": [C.POINTER(C.c_int32), C.c_int32, C.c_uint64, C.c_int32, C.c_int32, C.c_int32,
                                       C.POINTER(C.c_void_p)],
        "picard_server_submit": [C.c_void_p, C.POINTER(PicardRequest)],
        "picard_server_now_ms": [C.c_void_p, dp],
        "picard_server_poll": [C.c_void_p, C.POINTER(PicardResult), C.c_int32, ip, C.c_int32],
        "picard_server_load": [C.c_void_p, ip, ip, C.POINTER(C.c_uint64)],
        "picard_server_destroy": [C.c_void_p],
        "picard_gpu_particles_gridify_noalloc": [P, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32,
                                                 C.c_void_p, C.c_void_p, C.c_void_p],
        "picard_format_e": [C.c_double, C.c_int32, C.c_int32, C.c_char_p],
        "picard_gpu_dump_particles": [ctx, C.c_char_p, ip],
        "picard_gpu_dump_fields": [ctx, C.c_char_p, ip],
        "picard_params_plasma": [P, C.POINTER(PicardPlasma)],
        "picard_write_parameters": [P, C.c_char_p, C.POINTER(C.c_uint32)],
        "picard_gpu_run_io": [ctx, C.c_int32, C.c_int32, C.c_int32, LOG_FN, C.c_void_p, C.POINTER(PicardIO),
                              C.POINTER(C.c_int64)],
    }
    for name, args in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = C.c_int
    L.picard_gpu_last_error.argtypes = []
    L.picard_gpu_last_error.restype = C.c_char_p
    L.picard_warning_text.argtypes = [C.c_int32]
    L.picard_warning_text.restype = C.c_char_p
    _lib = L
    return L


def last_error() -> str:
    return lib().picard_gpu_last_error().decode(errors="replace")


def check(rc: int, where: str, allow=(OK,)) -> int:
    if rc not in allow:
        raise PicardError(rc, where, last_error())
    return rc


def params_default() -> PicardParams:
    p = PicardParams()
    check(lib().picard_params_default(C.byref(p)), "picard_params_default")
    return p


def params_derive(p: PicardParams) -> PicardParams:
    q = p.copy()
    check(lib().picard_params_derive(C.byref(q)), "picard_params_derive")
    return q


def footprint(p: PicardParams, layout: int, solver: int) -> int:
    b = C.c_uint64(0)
    check(lib().picard_gpu_footprint(C.byref(p), layout, solver, C.byref(b)), "picard_gpu_footprint")
    return int(b.value)


def pool_keep(device: int, nbytes: int) -> None:
    """Keep up to nbytes of freed context memory in the device's pool."""
    check(lib().picard_gpu_pool_keep(device, nbytes), "picard_gpu_pool_keep")


def format_e(value: float, w: int = 10, d: int = 4) -> str:
    """Fortran Ew.d of value (picard_format_e)."""
    buf = C.create_string_buffer(w + 1)
    check(lib().picard_format_e(float(value), w, d, buf), "picard_format_e")
    return buf.value.decode()


def plasma(p) -> dict:
    """WriteWarnings.f90's plasma quantities and warning mask of derived params."""
    out = PicardPlasma()
    check(lib().picard_params_plasma(C.byref(p), C.byref(out)), "picard_params_plasma")
    return out.as_dict()


def warning_texts(mask: int) -> list[str]:
    return [lib().picard_warning_text(k).decode() for k in range(WARN_COUNT) if mask >> k & 1]


def write_parameters(p, root: str) -> int:
    """<root>/parameters.dat and <root>/warnings.dat; returns the warning mask."""
    m = C.c_uint32(0)
    check(lib().picard_write_parameters(C.byref(p), root.encode(), C.byref(m)), "picard_write_parameters")
    return int(m.value)
