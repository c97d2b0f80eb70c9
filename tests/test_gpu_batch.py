"""Batched runs (picard_batch_run_fused) on the device.

Bar: every run of a batch ends bit for bit where the same run advanced alone
with picard_gpu_run_fused ends -- potential, density, particle count and
Jacobi sweeps (the batched sweep launch computes each node and each tile
partial exactly as the single-run kernels) -- with a mix of grid sizes, both
tile depths (nz < 64 and nz >= 64) and one run with a periodic axis, which
solves on its own inside the batch.  The particles too: inflow survivors are
appended in candidate order and BCoutflow fills holes in a fixed order, so
the particle arrays and the energies summed over them match bit for bit."""
import numpy as np
import pytest

from picard_b200 import capi
from picard_b200 import params as P
from picard_b200.simulation import Simulation, batch_run_fused, batch_step

pytestmark = pytest.mark.gpu


def _runs():
    out = []
    for k, (n, ny, nz, ppc) in enumerate([(24, 24, 24, 3), (40, 24, 72, 2), (16, 16, 16, 4), (33, 20, 18, 2)]):
        p = P.config_plain_32(seed=40 + k, n=8, ppc=ppc)
        p.nx, p.ny, p.nz = n, ny, nz
        p.xmin, p.xmax = -500.0 * n, 500.0 * n
        p.ymin, p.ymax = -500.0 * ny, 500.0 * ny
        p.zmin, p.zmax = -500.0 * nz, 500.0 * nz
        if k == 3:
            p.zflow = 0  # periodic z: not batchable, solved on its own
        p = P._size_capacity(p, 10, ppc)
        out.append(capi.params_derive(p))
    return out


def _start(p, solver=capi.SOLVER_F32_REFINE):
    g = Simulation(p, derive=False, layout=capi.LAYOUT_CELL32, solver=solver)
    g.calc_distance()
    g.particles_initialize()
    return g


@pytest.mark.parametrize("w32,unified", [("0", "1"), ("1", "1"), ("1", "2"), ("0", "0"), ("1", "0")])
def test_batch_equals_each_run_alone(w32, unified, monkeypatch):
    monkeypatch.setenv("PICARD_BATCH_W32", w32)  # 32-wide tiles for the 24^3 and 16^3 runs when "1"
    # one launch per tick and tile depth ("1"), per tick ("2") or per tile class ("0")
    monkeypatch.setenv("PICARD_BATCH_UNIFIED", unified)
    steps = 4
    params = _runs()
    alone = []
    for p in params:
        g = _start(p)
        sw = g.run_fused(0, steps)
        alone.append((sw, g.num_local, g.field(capi.FIELD_U), g.field(capi.FIELD_N), g.energy(), g.particles()))
        g.close()
    sims = [_start(p) for p in params]
    sweeps = batch_run_fused(sims, 0, steps)
    for k, g in enumerate(sims):
        sw, n, U, N, e, (rp, ip) = alone[k]
        assert sweeps[k] == sw, k
        assert g.num_local == n, k
        np.testing.assert_array_equal(g.field(capi.FIELD_U), U, err_msg=f"run {k}")
        np.testing.assert_array_equal(g.field(capi.FIELD_N), N, err_msg=f"run {k}")
        np.testing.assert_array_equal(g.energy(), e, err_msg=f"run {k}")
        rg, ig = g.particles()
        np.testing.assert_array_equal(ig, ip, err_msg=f"run {k}")
        np.testing.assert_array_equal(rg, rp, err_msg=f"run {k}")
    for g in sims:
        g.close()


def test_batch_rejects_duplicates():
    p = _runs()[0]
    g = _start(p)
    with pytest.raises(capi.PicardError) as e:
        batch_run_fused([g, g], 0, 1)
    assert e.value.code == capi.ERR_BAD_ARG
    g.close()


def test_staggered_steps_equal_each_run_alone():
    """picard_batch_step: runs at different iterations of their loops share a
    step (continuous batching) and still end bit for bit where they end alone."""
    steps = 4
    params = _runs()[:3]
    offsets = [0, 2, 1]  # iterations each run took alone before joining
    alone = []
    for p in params:
        g = _start(p)
        g.run_fused(0, steps)
        alone.append((g.num_local, g.field(capi.FIELD_U), g.field(capi.FIELD_N)))
        g.close()
    sims = [_start(p) for p in params]
    done = list(offsets)
    for g, k in zip(sims, offsets):
        if k:
            g.run_fused(0, k)
    while any(d < steps for d in done):
        live = [i for i in range(len(sims)) if done[i] < steps]
        batch_step([sims[i] for i in live], [done[i] + 1 for i in live])
        for i in live:
            done[i] += 1
    for k, g in enumerate(sims):
        n, U, N = alone[k]
        assert g.num_local == n, k
        np.testing.assert_array_equal(g.field(capi.FIELD_U), U, err_msg=f"run {k}")
        np.testing.assert_array_equal(g.field(capi.FIELD_N), N, err_msg=f"run {k}")
    for g in sims:
        g.close()


def test_batch_with_closed_form_solves_equals_each_run_alone():
    """Runs with SOLVER_SPECTRAL in a batch (their Parseval evaluations
    collected for all of them together), mixed with FP32-sweep runs ticked
    together: every run bit for bit where it ends alone."""
    steps = 3
    params = _runs()
    solvers = [capi.SOLVER_SPECTRAL, capi.SOLVER_F32_REFINE, capi.SOLVER_SPECTRAL, capi.SOLVER_SPECTRAL]
    alone = []
    for p, sv in zip(params, solvers):
        g = _start(p, sv)
        sw = g.run_fused(0, steps)
        alone.append((sw, g.num_local, g.field(capi.FIELD_U), g.field(capi.FIELD_N), g.particles()))
        g.close()
    sims = [_start(p, sv) for p, sv in zip(params, solvers)]
    sweeps = batch_run_fused(sims, 0, steps)
    for k, g in enumerate(sims):
        sw, n, U, N, (rp, ip) = alone[k]
        assert sweeps[k] == sw, k
        assert g.num_local == n, k
        np.testing.assert_array_equal(g.field(capi.FIELD_U), U, err_msg=f"run {k}")
        np.testing.assert_array_equal(g.field(capi.FIELD_N), N, err_msg=f"run {k}")
        rg, ig = g.particles()
        np.testing.assert_array_equal(rg, rp, err_msg=f"run {k}")
    for g in sims:
        g.close()


def test_pool_keep_then_contexts_come_and_go():
    """picard_gpu_pool_keep: freed context memory stays in the device's pool;
    contexts created and released afterwards run as before."""
    capi.pool_keep(0, 1 << 30)
    p = _runs()[2]
    out = []
    for _ in range(2):
        g = _start(p, capi.SOLVER_SPECTRAL)
        g.run_fused(0, 2)
        out.append(g.field(capi.FIELD_U))
        g.close()
    np.testing.assert_array_equal(out[0], out[1])
    with pytest.raises(capi.PicardError) as e:
        capi.pool_keep(1 << 20, 0)  # no such device
    assert e.value.code == capi.ERR_BAD_ARG
