"""Failure detection on the device without a fault: a bounded wait that runs
out returns PICARD_ERR_TIMEOUT, and the context stays usable.

PICARD_OPT_WAIT_TEST makes the grid barrier of the register-resident Jacobi
kernel wait for one arrival more than its grid makes, with a short poll limit
(2^14 polls), so every CTA gives up and returns -- no trap, no fault, no
unbounded wait.  The same context then solves normally and equals a fresh
context bit for bit.
"""
import numpy as np
import pytest

from oracle import oracle as O
from picard_b200 import capi
from picard_b200.simulation import Simulation
from tests.helpers import rel_l2, small_plasma

pytestmark = pytest.mark.gpu

C32 = dict(layout=capi.LAYOUT_CELL32, solver=capi.SOLVER_F32_REFINE)


def blob_problem(nx=40, ny=24, nz=16):
    p = small_plasma(n=8, ppc=1, seed=41)
    p.nx, p.ny, p.nz = nx, ny, nz
    p.xmin, p.xmax = -500.0 * nx, 500.0 * nx
    p.ymin, p.ymax = -500.0 * ny, 500.0 * ny
    p.zmin, p.zmax = -500.0 * nz, 500.0 * nz
    p.max_per_proc = 1024
    q = O.derive(p)
    z, y, x = np.meshgrid(np.arange(nz + 2), np.arange(ny + 2), np.arange(nx + 2), indexing="ij")
    C = 1e-12 * np.exp(-((x - nx / 2) ** 2 + (y - ny / 3) ** 2 + (z - nz / 2) ** 2) / 20.0)
    C[0, :, :] = C[-1, :, :] = C[:, 0, :] = C[:, -1, :] = C[:, :, 0] = C[:, :, -1] = 0.0
    return q, C


def solve(g, C):
    g.set_field(capi.FIELD_C, C)
    g.set_field(capi.FIELD_U, np.zeros_like(C))
    return g.calc_epotential(), g.field(capi.FIELD_U)


def test_wait_that_runs_out_reports_timeout_and_context_recovers():
    p, C = blob_problem()
    g = Simulation(p, derive=False, **C32)
    g.set_option(capi.OPT_SWEEP_RESIDENT, 1)
    assert g.get_option(capi.OPT_SWEEP_RESIDENT) == 1
    g.set_option(capi.OPT_WAIT_TEST, 1)
    assert g.get_option(capi.OPT_WAIT_TEST) == 1
    g.set_field(capi.FIELD_C, C)
    g.set_field(capi.FIELD_U, np.zeros_like(C))
    with pytest.raises(capi.PicardError) as e:
        g._call("picard_gpu_calc_epotential", p.maxerr, p.maxit, None)
    assert e.value.code == capi.ERR_TIMEOUT
    # the same context, test off: a normal solve, equal to a fresh context's
    g.set_option(capi.OPT_WAIT_TEST, 0)
    sweeps, U = solve(g, C)
    h = Simulation(p, derive=False, **C32)
    h.set_option(capi.OPT_SWEEP_RESIDENT, 1)
    sweeps_h, U_h = solve(h, C)
    assert sweeps == sweeps_h > 10
    np.testing.assert_array_equal(U, U_h)
    o = O.OracleState(p)
    o.C[...] = C
    s_o, conv, _ = o.calc_epotential()
    assert conv and abs(s_o - sweeps) <= 1
    assert rel_l2(U, o.U) < 1e-6
    g.close()
    h.close()
