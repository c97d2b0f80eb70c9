"""The serving loop (include/picard_server.h) on the device.

Bars: a run's result is the same alone and in a mix of concurrent runs -- the
final potential's checksums, the particle count, the particle-steps and the
Jacobi sweep count bit for bit (deposits are fixed point and every reduction
on the field path has a fixed order), and the energies bit for bit too (their
FP64 sums run over the particles in storage order, which is deterministic:
inflow survivors land in candidate order, BCoutflow fills holes in a fixed
order).  Admission never lets the admitted runs' footprints exceed the
budget.
"""
import numpy as np
import pytest

from picard_b200 import capi
from picard_b200 import params as P
from picard_b200.server import Server
from picard_b200.simulation import Simulation

pytestmark = pytest.mark.gpu

GB = 1 << 30


def _serving_requests(seed, count, steps):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        n = int(rng.integers(16, 33))
        p = P.config_plain_scale(seed=seed * 100 + i, nx=n, ny=n, nz=n, ppc_ion=int(rng.integers(2, 6)))
        p.Qn[2] = float(10.0 ** rng.uniform(25.0, 28.0))
        p = P._size_capacity(p, steps, 6)
        out.append(capi.params_derive(p))
    return out


def _same(a, b):
    for k in ("status", "num_local", "particle_steps", "sweeps", "u_sum", "u_abs_sum"):
        assert a[k] == b[k], k
    np.testing.assert_array_equal(a["energy"], b["energy"])


def test_result_is_the_same_alone_and_in_the_mix():
    steps = 6
    reqs = _serving_requests(11, 5, steps)
    target = 2
    with Server(8 * GB, 1) as s:
        s.submit(target, reqs[target], steps)
        alone = s.poll(wait_all=True)
    assert len(alone) == 1 and alone[0]["status"] == capi.OK
    with Server(8 * GB, 4) as s:
        for i, p in enumerate(reqs):
            s.submit(i, p, steps)
        mix = {r["id"]: r for r in s.poll(wait_all=True)}
    assert sorted(mix) == list(range(len(reqs)))
    assert all(r["status"] == capi.OK for r in mix.values())
    # the runs did overlap on the device
    spans = sorted((r["start_ms"], r["finish_ms"]) for r in mix.values())
    assert any(spans[k + 1][0] < spans[k][1] for k in range(len(spans) - 1))
    _same(alone[0], mix[target])


def test_served_run_equals_the_direct_fused_loop():
    steps = 4
    p = _serving_requests(12, 1, steps)[0]
    g = Simulation(p, derive=False, layout=capi.LAYOUT_CELL32, solver=capi.SOLVER_F32_REFINE)
    g.calc_distance()
    g.particles_initialize()
    g.run_fused(0, steps)
    e = g.energy()
    n = g.num_local
    U = g.field(capi.FIELD_U)
    with Server(4 * GB, 2) as s:
        s.submit(0, p, steps)
        r = s.poll(wait_all=True)[0]
    assert r["status"] == capi.OK
    assert r["warnings"] == capi.plasma(p)["warnings"]  # WriteWarnings.f90 on the request
    assert r["num_local"] == n
    assert r["u_sum"] == pytest.approx(float(U.sum()), rel=1e-12, abs=0)
    np.testing.assert_array_equal(r["energy"], e)


def test_admission_keeps_within_the_budget():
    steps = 3
    reqs = _serving_requests(13, 4, steps)
    fps = [capi.footprint(p, capi.LAYOUT_CELL32, capi.SOLVER_F32_REFINE) for p in reqs]
    budget = int(max(fps) * 1.5)
    with Server(budget, 4) as s:
        for i, p in enumerate(reqs):
            s.submit(i, p, steps)
        res = s.poll(wait_all=True)
    assert all(r["status"] == capi.OK for r in res)
    # at every admission instant the admitted runs' footprints fit the budget
    for r in res:
        t = r["start_ms"]
        held = sum(fps[q["id"]] for q in res if q["start_ms"] <= t < q["finish_ms"])
        assert held <= budget
    # a run larger than the whole budget is refused at submission
    with Server(max(fps) // 2, 2) as s:
        big = int(np.argmax(fps))
        with pytest.raises(capi.PicardError) as e:
            s.submit(0, reqs[big], steps)
        assert e.value.code == capi.ERR_CAPACITY


def test_batched_server_result_is_the_same_alone_and_in_the_mix():
    """Continuous batching: runs join and leave the cohort between steps (the
    step counts differ), and each result equals the run served alone and the
    run served by the stream-mode server."""
    reqs = _serving_requests(14, 5, 8)
    steps = [3, 5, 2, 4, 6]
    target = 3
    with Server(8 * GB, 1, batched=True) as s:
        s.submit(target, reqs[target], steps[target])
        alone = s.poll(wait_all=True)
    assert len(alone) == 1 and alone[0]["status"] == capi.OK
    with Server(8 * GB, 1) as s:
        s.submit(target, reqs[target], steps[target])
        streamed = s.poll(wait_all=True)[0]
    with Server(8 * GB, 3, batched=True, preparers=2) as s:
        for i, p in enumerate(reqs):
            s.submit(i, p, steps[i])
        mix = {r["id"]: r for r in s.poll(wait_all=True)}
    assert sorted(mix) == list(range(len(reqs)))
    assert all(r["status"] == capi.OK for r in mix.values())
    spans = sorted((r["start_ms"], r["finish_ms"]) for r in mix.values())
    assert any(spans[k + 1][0] < spans[k][1] for k in range(len(spans) - 1))
    _same(alone[0], mix[target])
    _same(streamed, mix[target])


@pytest.mark.parametrize("batched", [False, True])
def test_multi_device_placement_spreads_runs_and_keeps_results(batched):
    """picard_server_create_multi with the device list [0, 0]: two shards on
    one GPU (the only one a test box has).  Runs go to both shards, and each
    result equals the same run served by a single-device server."""
    reqs = _serving_requests(15, 4, 3)
    with Server(8 * GB, 2) as s:
        for i, p in enumerate(reqs):
            s.submit(i, p, 3)
        single = {r["id"]: r for r in s.poll(wait_all=True)}
    with Server(8 * GB, 2, batched=batched, preparers=1, devices=[0, 0]) as s:
        for i, p in enumerate(reqs):
            s.submit(i, p, 3)
        multi = {r["id"]: r for r in s.poll(wait_all=True)}
        assert s.load()[:2] == (0, 0)
    assert sorted(multi) == list(range(len(reqs)))
    assert {r["shard"] for r in multi.values()} == {0, 1}
    for i in range(len(reqs)):
        _same(single[i], multi[i])
