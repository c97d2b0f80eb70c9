"""SOLVER_SPECTRAL: CalcEpotential's Jacobi iterate in closed form
(CalcEpotential.f90:55-96), through the C ABI, against the FP64 oracle's
sweeps and against the FP64 sweep solver on the GPU.

The sweep operator is diagonal in the product of per-axis sine (open) or
Fourier (periodic) bases, so the iterate of any sweep count and the residual
norm of every iterate follow from one transform of the initial residual.
Bars: the same stopping sweep as the FP64 sweeps and the potential within
1e-11 relative L2 of theirs (both are FP64; the sweeps round each of their
updates); in the whole loop the tolerances of the FP64 solver.
"""
import numpy as np
import pytest

from oracle import oracle as O
from picard_b200 import capi
from picard_b200.simulation import Simulation
from tests.helpers import rel_l2, small_haser, small_plasma
from tests.test_gpu_fused import compare_with_oracle, developed

pytestmark = pytest.mark.gpu

SPEC64 = dict(layout=capi.LAYOUT_F64, solver=capi.SOLVER_SPECTRAL)
SPEC32 = dict(layout=capi.LAYOUT_CELL32, solver=capi.SOLVER_SPECTRAL)
F64 = dict(layout=capi.LAYOUT_F64, solver=capi.SOLVER_F64)


def blobs(o, p, seed, count=4, amp=1e-12, width=18.0):
    """Gaussian charge blobs inside the box, zero on the ghost layer."""
    nx, ny, nz = p.nx, p.ny, p.nz
    rng = np.random.default_rng(seed)
    z, y, x = np.meshgrid(np.arange(nz + 2), np.arange(ny + 2), np.arange(nx + 2), indexing="ij")
    C = np.zeros_like(o.C)
    for _ in range(count):
        c = rng.uniform([1, 1, 1], [nx, ny, nz])
        C += rng.normal() * amp * np.exp(-((x - c[0]) ** 2 + (y - c[1]) ** 2 + (z - c[2]) ** 2) / width)
    C[0, :, :] = C[-1, :, :] = C[:, 0, :] = C[:, -1, :] = C[:, :, 0] = C[:, :, -1] = 0.0
    return C


def boxed(nx, ny, nz, seed=31, **kw):
    p = small_plasma(n=8, ppc=1, seed=seed, **kw)
    p.nx, p.ny, p.nz = nx, ny, nz
    p.xmin, p.xmax = -500.0 * nx, 500.0 * nx
    p.ymin, p.ymax = -500.0 * ny, 500.0 * ny
    p.zmin, p.zmax = -500.0 * nz, 500.0 * nz
    p.max_per_proc = 1024
    return O.derive(p)


@pytest.mark.parametrize("kw", [SPEC64, SPEC32])
def test_spectral_matches_oracle_on_a_plasma(kw):
    # BCpotentials' face values and a developed plasma's charge (12^3, open
    # axes): the oracle's FP64 sweeps from the same U and C.
    p = O.derive(small_plasma(n=12, ppc=4, seed=5))
    o = developed(p, steps=1)
    o.gridify()
    o.bc_potentials()
    g = Simulation(p, derive=False, **kw)
    g.set_field(capi.FIELD_C, o.C)
    g.set_field(capi.FIELD_U, o.U)
    sweeps_o, conv, _ = o.calc_epotential()
    sweeps_g = g.calc_epotential()
    err = rel_l2(g.field(capi.FIELD_U), o.U)
    print(f"spectral vs oracle: {sweeps_g} vs {sweeps_o} sweeps, U rel L2 {err:.2e}")
    assert conv and sweeps_o > 50
    assert sweeps_g == sweeps_o
    assert err < 1e-11
    st = g.stats()
    assert st["spectral_transforms"] == 2 and st["sweep_launches"] == 0
    g.close()


@pytest.mark.parametrize("dims", [(72, 40, 36), (33, 20, 18), (1, 17, 5)])
def test_spectral_matches_oracle_on_blobs(dims):
    # uneven boxes (every tile edge case of the 64 x 64 product tiles) with a
    # boundary potential on the faces: the oracle's FP64 sweeps
    nx, ny, nz = dims
    p = boxed(nx, ny, nz)
    o = O.OracleState(p)
    o.C[...] = blobs(o, p, seed=5)
    o.calc_distance()
    o.bc_potentials()
    U0 = o.U.copy()
    g = Simulation(p, derive=False, **SPEC64)
    g.set_field(capi.FIELD_C, o.C)
    g.set_field(capi.FIELD_U, U0)
    sweeps_o, conv, _ = o.calc_epotential()
    sweeps_g = g.calc_epotential()
    err = rel_l2(g.field(capi.FIELD_U), o.U)
    print(f"{dims}: spectral {sweeps_g} vs oracle {sweeps_o} sweeps, U rel L2 {err:.2e}")
    assert conv
    assert sweeps_g == sweeps_o
    assert err < 1e-11
    g.close()


@pytest.mark.parametrize("flows", [(1, 0, 0), (0, 1, 1), (1, 1, 0)])
def test_spectral_matches_fp64_sweeps_with_periodic_axes(flows):
    # periodic axes: the FP64 sweep solver on the GPU (which wraps with
    # current values, like the Fourier basis) from the same U and C
    xf, yf, zf = flows
    p = boxed(24, 20, 18, xflow=xf, yflow=yf, zflow=zf)
    o = O.OracleState(p)
    o.C[...] = blobs(o, p, seed=9, width=30.0)
    o.calc_distance()
    o.bc_potentials()
    sims = [Simulation(p, derive=False, **kw) for kw in (SPEC64, F64)]
    for s in sims:
        s.set_field(capi.FIELD_C, o.C)
        s.set_field(capi.FIELD_U, o.U)
    sw = [s.calc_epotential() for s in sims]
    err = rel_l2(sims[0].field(capi.FIELD_U), sims[1].field(capi.FIELD_U))
    print(f"flows {flows}: spectral {sw[0]} vs FP64 sweeps {sw[1]}, U rel L2 {err:.2e}")
    assert sw[0] == sw[1] and sw[0] > 10
    assert err < 1e-11
    for s in sims:
        s.close()


def test_spectral_cap_reports_not_converged():
    # without a hit before maxit the reference runs all 2*maxit+1 sweeps and
    # keeps that iterate
    p = boxed(10, 9, 8)
    o = O.OracleState(p)
    C = np.zeros_like(o.C)
    C[2:-2, 2:-2, 2:-2] = 1e-15
    o.C[...] = C
    g = Simulation(p, derive=False, **SPEC64)
    g.set_field(capi.FIELD_C, C)
    g.set_field(capi.FIELD_U, np.zeros_like(o.U))
    s_o, conv, _ = o.calc_epotential(maxerr=1e-12, maxit=3)
    with pytest.raises(capi.PicardError) as e:
        g._call("picard_gpu_calc_epotential", 1e-12, 3, None)
    assert e.value.code == capi.ERR_NOT_CONVERGED
    assert not conv and s_o == 7
    assert rel_l2(g.field(capi.FIELD_U), o.U) < 1e-12
    g.close()


def test_spectral_per_subroutine_step_matches_oracle():
    # one iteration of picard_gpu_run (the reference's call sequence) in the
    # F64 layout: positions bit-exact, the same sweeps, U and E within 1e-10
    p = O.derive(small_plasma(n=8, ppc=4, seed=1))
    o = developed(p, steps=1)
    g = Simulation(p, derive=False, **SPEC64)
    g.calc_distance()
    g.set_particles(*o.particles())
    sweeps_o = o.step(2)
    sweeps_g = g.run(1, 2)
    assert sweeps_g == sweeps_o
    assert g.num_local == o.num_local
    rg, ig = g.particles()
    ro, io = o.particles()
    np.testing.assert_array_equal(ig, io)
    np.testing.assert_array_equal(rg[:, :3], ro[:, :3])
    np.testing.assert_allclose(rg[:, 3:6], ro[:, 3:6], rtol=1e-9, atol=1e-6)
    assert rel_l2(g.field(capi.FIELD_U), o.U) < 1e-10
    assert rel_l2(g.field(capi.FIELD_E), o.E) < 1e-10
    g.close()


@pytest.mark.parametrize("steps", [1, 3])
def test_fused_cell32_spectral_matches_oracle(steps):
    # the fused loop in the CELL32 layout with the closed-form solve, from
    # identical particle arrays (as the F32_REFINE fused tests)
    p = O.derive(small_plasma(n=10, ppc=4, seed=13))
    o = developed(p)
    g = Simulation(p, derive=False, **SPEC32)
    g.calc_distance()
    g.set_particles(*o.particles())
    sw_o = [o.step(it) for it in range(21, 21 + steps)]
    sw_g = g.run_fused(20, 20 + steps)
    errs = compare_with_oracle(p, g, o, steps, f"fused CELL32 spectral, {steps} step(s)")
    assert abs(sw_g - sum(sw_o)) <= steps
    assert errs["U"] < 5e-7
    g.close()


def test_fused_cell32_spectral_haser_matches_oracle():
    # the at-scale workload's shape shrunk (64 x 32 x 32, Haser source at
    # dt-scaled production) after 8 FP64-layout steps
    p = O.derive(small_haser(nx=64, ny=32, nz=32, ppc=2, seed=3))
    o = O.OracleState(p)
    o.calc_distance()
    o.initialize()
    for it in range(1, 9):
        o.step(it)
    g = Simulation(p, derive=False, **SPEC32)
    g.calc_distance()
    g.set_particles(*o.particles())
    o.step(9)
    g.run_fused(8, 9)
    compare_with_oracle(p, g, o, 1, "fused CELL32 spectral, Haser 64x32x32")
    g.close()
