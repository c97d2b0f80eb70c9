"""The C-ABI library without a GPU: it loads, exports every entry point that
include/picard_gpu.h declares, and its host-only routines (parameter defaults
and derivation, footprint) agree with the reference and the oracle."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from oracle import oracle as O
from picard_b200 import capi
from picard_b200 import params as P

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "picard_gpu.h")).read()
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
    assert big - small == pytest.approx(2 * 29 * p.max_per_proc, rel=0.01)
    assert capi.footprint(p, capi.LAYOUT_F64, capi.SOLVER_F64) > small


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
