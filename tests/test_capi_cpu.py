"""The C-ABI library without a GPU: it loads, exports every entry point that
include/*.h declares, and its host-only routines (parameter defaults
and derivation, footprint) agree with the reference and the oracle."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

from oracle import oracle as O
from picard_b200 import capi
from picard_b200 import params as P

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    inc = os.path.join(ROOT, "include")
    text = "".join(open(os.path.join(inc, h)).read() for h in sorted(os.listdir(inc)) if h.endswith(".h"))
    return sorted(set(re.findall(r"PICARD_API\s+[\w\s\*]+?\b(picard_\w+)\s*\(", text)))


def test_header_declares_the_entry_points():
    names = declared_symbols()
    assert len(names) >= 30
    for must in ("picard_gpu_calc_epotential", "picard_gpu_particles_gridify", "picard_gpu_advance_velocity",
                 "picard_gpu_bc_inflow", "picard_gpu_bc_potentials", "picard_gpu_run"):
        assert must in names


def test_library_exports_every_declared_symbol():
    L = capi.lib()
    for name in declared_symbols():
        assert hasattr(L, name), name


def test_struct_layout_matches_header():
    # the ctypes mirror must have the size the C compiler gives picard_params
    assert C.sizeof(P.PicardParams) % 8 == 0
    assert P.PicardParams.u0.offset == C.sizeof(P.PicardParams) - 8


def test_defaults_are_the_reference_values():
    p = capi.params_default()
    assert (p.nx, p.ny, p.nz, p.species) == (30, 30, 30, 3)
    assert p.maxit == 2 ** 20 and p.maxerr == 2.0 ** -16
    assert p.dt == 4.0e-6 and p.xmin == -600.0 and p.xmax == 600.0
    assert p.ppc[1] == 64 and p.density[1] == 1.07e6
    assert p.v0[0][0] == -430.0e3 and p.B0[1] == pytest.approx(400.0 * 1.78e-9)
    assert p.Qn[2] == pytest.approx(400.0 ** -3 * 1.99e26)


@pytest.mark.parametrize("make", [
    lambda: P.config_plain_32(),
    lambda: P.config_plain_scale(nx=16, ny=8, nz=8),
    lambda: capi.params_default(),
])
def test_derivation_matches_oracle_bit_for_bit(make):
    p = make()
    a = capi.params_derive(p)
    b = O.derive(p)
    assert bytes(a) == bytes(b)


def test_footprint_scales_with_capacity():
    p = capi.params_derive(P.config_plain_32(n=8, ppc=2))
    small = capi.footprint(p, capi.LAYOUT_CELL32, capi.SOLVER_F32_REFINE)
    p2 = p.copy()
    p2.max_per_proc = p.max_per_proc * 2
    big = capi.footprint(p2, capi.LAYOUT_CELL32, capi.SOLVER_F32_REFINE)
    # one particle buffer (BCoutflow removes in place) plus its keep words and
    # block scan: 8 B x (64 + 3) per block of 2048 particles
    assert big - small == pytest.approx((29 + 8 * 67 / 2048) * p.max_per_proc, rel=0.01)
    # where particles dominate, the FP64 layout (49 B/particle) holds more
    # than CELL32 (29 B/particle) even with CELL32's tensor-core scratch
    p3 = p.copy()
    p3.max_per_proc = 10_000_000
    assert capi.footprint(p3, capi.LAYOUT_F64, capi.SOLVER_F64) > capi.footprint(
        p3, capi.LAYOUT_CELL32, capi.SOLVER_F32_REFINE)


def test_bad_arguments_are_rejected_without_a_device():
    p = capi.params_derive(P.config_plain_32(n=8, ppc=2))
    bad = p.copy()
    bad.species = 9
    h = C.c_void_p()
    rc = capi.lib().picard_gpu_create(C.byref(bad), capi.LAYOUT_F64, capi.SOLVER_F64, C.byref(h))
    assert rc == capi.ERR_BAD_ARG and "species" in capi.last_error()
    rc = capi.lib().picard_gpu_create(C.byref(p), 7, capi.SOLVER_F64, C.byref(h))
    assert rc == capi.ERR_BAD_ARG
    underived = P.config_plain_32(n=8, ppc=2)
    rc = capi.lib().picard_gpu_create(C.byref(underived), capi.LAYOUT_F64, capi.SOLVER_F64, C.byref(h))
    assert rc == capi.ERR_BAD_ARG and "derive" in capi.last_error()


_LAYOUT_PROBE = r"""
#include <stddef.h>
#include <stdio.h>
#include "picard_server.h"
#include "picard_io.h"
#define F(T, m) printf(#T "." #m " %zu\n", offsetof(T, m))
int main(void) {
  printf("picard_plasma %zu\n", sizeof(picard_plasma));
  printf("picard_io %zu\n", sizeof(picard_io));
  F(picard_plasma, va); F(picard_plasma, sd); F(picard_plasma, cfl); F(picard_plasma, dt_rec);
  F(picard_plasma, vth); F(picard_plasma, warnings);
  F(picard_io, fields_interval); F(picard_io, fields_iteration); F(picard_io, root);
  printf("picard_params %zu\n", sizeof(picard_params));
  printf("picard_stats %zu\n", sizeof(picard_stats));
  printf("picard_request %zu\n", sizeof(picard_request));
  printf("picard_result %zu\n", sizeof(picard_result));
  F(picard_request, params); F(picard_request, layout); F(picard_request, steps); F(picard_request, arrival_ms);
  F(picard_result, status); F(picard_result, sweeps); F(picard_result, energy); F(picard_result, u_abs_sum); F(picard_result, warnings); F(picard_result, shard);
  F(picard_stats, phase_ms); F(picard_stats, last_sweeps);
  PARAMS_FIELDS
  return 0;
}
"""


def test_ctypes_structs_match_the_c_compiler(tmp_path):
    """Every struct that crosses the C ABI has the size and field offsets gcc
    gives it from the headers."""
    src = tmp_path / "probe.c"
    # every field of picard_params: the Fortran derived type of the
    # integration module mirrors this block field for field
    fields = " ".join(f"F(picard_params, {name});" for name, _ in P.PicardParams._fields_)
    src.write_text(_LAYOUT_PROBE.replace("PARAMS_FIELDS", fields))
    exe = tmp_path / "probe"
    subprocess.run(["gcc", "-std=c99", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = dict(line.split() for line in subprocess.run([str(exe)], capture_output=True, text=True,
                                                        check=True).stdout.splitlines())
    assert int(got["picard_params"]) == C.sizeof(P.PicardParams)
    assert int(got["picard_stats"]) == C.sizeof(capi.PicardStats)
    assert int(got["picard_request"]) == C.sizeof(capi.PicardRequest)
    assert int(got["picard_result"]) == C.sizeof(capi.PicardResult)
    assert int(got["picard_plasma"]) == C.sizeof(capi.PicardPlasma)
    assert int(got["picard_io"]) == C.sizeof(capi.PicardIO)
    for key, val in got.items():
        if "." not in key:
            continue
        sname, field = key.split(".")
        cls = {"picard_request": capi.PicardRequest, "picard_result": capi.PicardResult,
               "picard_stats": capi.PicardStats, "picard_params": P.PicardParams,
               "picard_plasma": capi.PicardPlasma, "picard_io": capi.PicardIO}[sname]
        assert getattr(cls, field).offset == int(val), key


def test_server_rejects_bad_arguments_without_a_device():
    L = capi.lib()
    out = C.c_void_p()
    assert L.picard_server_create(0, 2, C.byref(out)) == capi.ERR_BAD_ARG
    assert L.picard_server_create(1 << 30, 0, C.byref(out)) == capi.ERR_BAD_ARG
    devs = (C.c_int32 * 2)(0, 0)
    assert L.picard_server_create_multi(devs, 0, 1 << 30, 2, 0, 1, C.byref(out)) == capi.ERR_BAD_ARG
    assert L.picard_server_create_multi(devs, 2, 1 << 30, 0, 0, 1, C.byref(out)) == capi.ERR_BAD_ARG
    assert L.picard_server_create_multi(None, 2, 1 << 30, 2, 0, 1, C.byref(out)) == capi.ERR_BAD_ARG
    assert L.picard_server_submit(None, None) == capi.ERR_BAD_ARG
    assert L.picard_server_destroy(None) == capi.OK
