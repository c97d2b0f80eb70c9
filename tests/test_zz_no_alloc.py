"""The allocation-free deposit, picard_gpu_particles_gridify_noalloc.

Callers that cannot allocate device memory when they need a deposit -- a host
whose device arrays sit in a pool another runtime reserved up front, a server
that has promised all of the HBM to resident runs, a pipeline that cannot take
the device-wide synchronisation of cudaFree -- pass their own particle arrays
and output grids; the entry point's scratch is a fixed array inside the
library.  These tests call it through the C ABI and compare it with the
context-based picard_gpu_particles_gridify on the same particles, twice in a
row with different particles (the shared scratch must not carry the first
call's sums into the second).  This file is collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest

from oracle import oracle as O
from picard_b200 import capi
from picard_b200.simulation import Simulation
from tests.helpers import rel_l2, small_plasma

pytestmark = pytest.mark.gpu


def _noalloc(p, rp, ip):
    import torch

    dev = torch.device("cuda", 0)
    x = torch.tensor(np.ascontiguousarray(rp[:, 0]), dtype=torch.float64, device=dev)
    y = torch.tensor(np.ascontiguousarray(rp[:, 1]), dtype=torch.float64, device=dev)
    z = torch.tensor(np.ascontiguousarray(rp[:, 2]), dtype=torch.float64, device=dev)
    s = torch.tensor(ip, dtype=torch.int32, device=dev)
    nodes = (p.nx + 2) * (p.ny + 2) * (p.nz + 2)
    N = torch.full((nodes * p.species,), float("nan"), dtype=torch.float64, device=dev)
    Cg = torch.full((nodes,), float("nan"), dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    rc = capi.lib().picard_gpu_particles_gridify_noalloc(C.byref(p), x.data_ptr(), y.data_ptr(), z.data_ptr(),
                                                         s.data_ptr(), rp.shape[0], N.data_ptr(), Cg.data_ptr(),
                                                         C.c_void_p(stream))
    capi.check(rc, "picard_gpu_particles_gridify_noalloc")
    torch.cuda.synchronize(dev)
    shape = (p.nz + 2, p.ny + 2, p.nx + 2)
    return N.cpu().numpy().reshape(shape + (p.species,)), Cg.cpu().numpy().reshape(shape)


def _reference_deposit(p, rp, ip):
    g = Simulation(p, derive=False, layout=capi.LAYOUT_F64, solver=capi.SOLVER_F64)
    g.set_particles(rp, ip)
    g.particles_gridify()
    out = g.field(capi.FIELD_N), g.field(capi.FIELD_C)
    g.close()
    return out


@pytest.mark.parametrize("periodic", [None, "x", "y"])
def test_noalloc_deposit_matches_context_deposit_twice(periodic):
    kw = {} if periodic is None else {periodic + "flow": 0}
    p = O.derive(small_plasma(n=12, ppc=4, seed=17, **kw))
    o = O.OracleState(p)
    o.calc_distance()
    o.initialize()
    o.step(1)
    first = o.particles()
    for it in range(2, 5):
        o.step(it)
    second = o.particles()
    assert first[0].shape != second[0].shape or not np.array_equal(first[0], second[0])
    for rp, ip in (first, second):
        N_ref, C_ref = _reference_deposit(p, rp, ip)
        N, Cg = _noalloc(p, rp, ip)
        assert np.isfinite(N).all() and np.isfinite(Cg).all()
        assert rel_l2(N, N_ref) < 1e-10
        scale = max(abs(p.charge[s]) * np.abs(N_ref[..., s]).max() for s in range(p.species))
        assert np.abs(Cg - C_ref).max() < 1e-10 * scale
        # and against the oracle's own ParticlesGridify on the same arrays
        o2 = O.OracleState(p)
        o2.set_particles(rp, ip)
        o2.gridify()
        assert rel_l2(N, o2.N) < 1e-10
        assert np.abs(Cg - o2.C).max() < 1e-10 * scale


def test_noalloc_skips_foreign_species_and_far_out_particles():
    # Particles of species number 0 or species+1, and particles farther than
    # half a cell outside the domain on an axis (a periodic one included, and
    # NaN), leave N and C exactly as the deposit of the others.
    p = O.derive(small_plasma(n=10, ppc=3, seed=23, xflow=0))
    o = O.OracleState(p)
    o.calc_distance()
    o.initialize()
    o.step(1)
    rp, ip = o.particles()
    N0, C0 = _noalloc(p, rp, ip)
    extra_r = np.repeat(rp[:1], 7, axis=0).copy()
    extra_i = np.array([0, p.species + 1, 1, 2, 1, 2, 1], np.int32)
    d = p.dxyz[0]
    extra_r[2, 0] = p.Lx_max + 3.0 * d          # periodic x, three cells out
    extra_r[3, 0] = p.Lx_min - 0.75 * d         # periodic x, below half a cell
    extra_r[4, 1] = p.Ly_max + 1e30             # open y, far out
    extra_r[5, 2] = float("nan")
    extra_r[6, 0] = -1e300                      # periodic x, far beyond any period count
    rp2 = np.concatenate([extra_r[:4], rp, extra_r[4:]])
    ip2 = np.concatenate([extra_i[:4], ip, extra_i[4:]])
    N1, C1 = _noalloc(p, rp2, ip2)
    np.testing.assert_array_equal(N1, N0)
    np.testing.assert_array_equal(C1, C0)


def test_noalloc_rejects_grids_beyond_its_scratch():
    p = O.derive(small_plasma(n=130, ppc=1))
    rc = capi.lib().picard_gpu_particles_gridify_noalloc(C.byref(p), None, None, None, None, 0, None, None, None)
    assert rc == capi.ERR_BAD_ARG
    assert "fixed scratch" in capi.last_error()
