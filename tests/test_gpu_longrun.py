"""Long runs against the oracle: the 32^3 solar-wind workload (32x32x32 cells,
16 ions + 16 electrons per cell, inflow at x-min, Philox seed 0) for its full
100 steps through picard_gpu_run, compared with the oracle's FP64 loop on the
energy log the reference prints every 10 steps (picard.f90:649-672) and on the
moments of the final density N.

Bars (measured on a B200: FP64 layout counts identical, energies within 5e-14 /
2.4e-12, moments within 2e-15; CELL32 one particle of 1,048,400, kinetic 5.6e-8,
field 5.9e-5, moments 1e-11 .. 1.3e-6):
  FP64 layout + FP64 Jacobi  counts equal; kinetic and magnetic energy 1e-11,
                             field energy 1e-9; moments 1e-12 (first moments
                             1e-11 cells);
  CELL32 + FP32 refine       counts 1e-5; kinetic energy 1e-6, field energy
                             1e-3; density moments: total 1e-9, centre 1e-4
                             cells, spread 1e-5.
The FP32 positions and the FP32 Jacobi of the CELL32 path make the run drift
from the FP64 one chaotically but slowly; the moments are what a long run must
keep."""
import numpy as np
import pytest

from oracle import oracle as O
from picard_b200 import capi
from picard_b200 import params as P
from picard_b200.simulation import Simulation

pytestmark = pytest.mark.gpu

STEPS = 100


def _moments(N):
    """Per species: total, centre (node index units) and spread along x, y, z."""
    nz, ny, nx, S = N.shape
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    out = []
    for s in range(S):
        w = N[..., s]
        m0 = float(w.sum())
        m1 = [float((w * c).sum() / m0) for c in (i, j, k)]
        m2 = [float((w * (c - m) ** 2).sum() / m0) for c, m in zip((i, j, k), m1)]
        out.append((m0, m1, m2))
    return out


@pytest.fixture(scope="module")
def oracle_run():
    p = O.derive(P.config_plain_32())
    o = O.OracleState(p)
    o.calc_distance()
    o.initialize()
    log = []
    for it in range(1, STEPS + 1):
        o.step(it)
        if it % 10 == 0:
            log.append((it, o.num_local) + tuple(np.asarray(o.energy()) / p.u0))
    return p, log, _moments(o.N)


@pytest.mark.parametrize("name,kw,tol", [
    ("f64", dict(layout=capi.LAYOUT_F64, solver=capi.SOLVER_F64),
     dict(n=0.0, uP=1e-11, uE=1e-9, uB=1e-11, m0=1e-12, m1=1e-11, m2=1e-12)),
    ("cell32", dict(layout=capi.LAYOUT_CELL32, solver=capi.SOLVER_F32_REFINE),
     dict(n=1e-5, uP=1e-6, uE=1e-3, uB=1e-11, m0=1e-9, m1=1e-4, m2=1e-5)),
])
def test_long_run_energy_log_and_density_moments(oracle_run, name, kw, tol):
    p, elog, mo = oracle_run
    g = Simulation(p, derive=False, **kw)
    g.calc_distance()
    g.particles_initialize()
    glog = []
    g.run(0, STEPS, log_interval=10, log=lambda it, t, n, up, ue, ub: glog.append((it, n, up, ue, ub)))
    mg = _moments(g.field(capi.FIELD_N))
    g.close()
    assert [r[0] for r in glog] == [r[0] for r in elog]
    for a, b in zip(glog, elog):
        it = a[0]
        assert abs(a[1] - b[1]) <= tol["n"] * b[1], (name, it, "particles")
        assert abs(a[2] - b[2]) <= tol["uP"] * abs(b[2]), (name, it, "kinetic")
        assert abs(a[3] - b[3]) <= tol["uE"] * abs(b[3]), (name, it, "field")
        assert abs(a[4] - b[4]) <= tol["uB"] * abs(b[4]), (name, it, "magnetic")
    for s, (a, b) in enumerate(zip(mg, mo)):
        assert abs(a[0] - b[0]) <= tol["m0"] * b[0], (name, s, "total")
        for ax in range(3):
            assert abs(a[1][ax] - b[1][ax]) <= tol["m1"], (name, s, ax, "centre")
            assert abs(a[2][ax] - b[2][ax]) <= tol["m2"] * b[2][ax], (name, s, ax, "spread")


def test_long_fused_run_with_sort_keeps_the_moments(oracle_run):
    # The benchmarked path over the same 100 steps: picard_gpu_run_fused in
    # CELL32 with the FP32-refine Jacobi, the particles put back in cell order
    # every 10 steps.  The particle count, the energies after the last step and
    # the density moments meet the CELL32 bars above.
    p, elog, mo = oracle_run
    tol = dict(n=1e-5, uP=1e-6, uE=1e-3, uB=1e-11, m0=1e-9, m1=1e-4, m2=1e-5)
    g = Simulation(p, derive=False, layout=capi.LAYOUT_CELL32, solver=capi.SOLVER_F32_REFINE)
    g.set_option(capi.OPT_SORT_EVERY, 10)
    g.calc_distance()
    g.particles_initialize()
    g.run_fused(0, STEPS)
    n = g.num_local
    up, ue, ub = (float(v) / p.u0 for v in g.energy())
    mg = _moments(g.field(capi.FIELD_N))
    g.close()
    it, n_o, up_o, ue_o, ub_o = elog[-1]
    assert it == STEPS
    print(f"fused + sort, step {it}: particles {n} vs {n_o}, kinetic {up / up_o - 1:.1e}, "
          f"field {ue / ue_o - 1:.1e}, magnetic {ub / ub_o - 1:.1e}")
    assert abs(n - n_o) <= tol["n"] * n_o
    assert abs(up - up_o) <= tol["uP"] * abs(up_o)
    assert abs(ue - ue_o) <= tol["uE"] * abs(ue_o)
    assert abs(ub - ub_o) <= tol["uB"] * abs(ub_o)
    for s, (a, b) in enumerate(zip(mg, mo)):
        assert abs(a[0] - b[0]) <= tol["m0"] * b[0], (s, "total")
        for ax in range(3):
            assert abs(a[1][ax] - b[1][ax]) <= tol["m1"], (s, ax, "centre")
            assert abs(a[2][ax] - b[2][ax]) <= tol["m2"] * b[2][ax], (s, ax, "spread")
