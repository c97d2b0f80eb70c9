"""The counting sort by cell (picard_gpu_sort_particles).

On one rank ParticlesTransfer.f90:488-519 only wraps coordinates; the sort
sits in its slot and puts the particles back in the order ParticlesInitialize
creates them (cell by cell, x fastest), which cell crossings, BCoutflow's hole
filling and appended particles wear down.  Bars: the sort equals numpy's
stable argsort of the cell keys bit for bit, on shuffled, clustered and
already sorted arrays in both layouts; a freshly initialised plasma is already
in that order; the deposit gives the same N bits before and after; and the
fused loop with a sort every other step holds exactly the same particles (as
a set), the same sweep counts and the same N, U and E bits as without.
"""
import numpy as np
import pytest

from oracle import oracle as O
from picard_b200 import capi
from picard_b200.simulation import Simulation
from tests.helpers import small_haser, small_plasma, sort_particles

pytestmark = pytest.mark.gpu

LAYOUTS = {"cell32": dict(layout=capi.LAYOUT_CELL32, solver=capi.SOLVER_F32_REFINE),
           "f64": dict(layout=capi.LAYOUT_F64, solver=capi.SOLVER_F64)}


def random_particles(p, n, rng, cells=None):
    """n particles uniform over the domain (or over its first cells^3 cells),
    velocities of ~100 km/s, species 1..S, in random order."""
    lo = np.array([p.Lx_min, p.Ly_min, p.Lz_min])
    hi = np.array([p.Lx_max, p.Ly_max, p.Lz_max])
    if cells is not None:
        hi = lo + cells * np.array(list(p.dxyz))
    rp = np.zeros((n, 8))
    rp[:, :3] = lo + (hi - lo) * rng.random((n, 3))
    rp[:, 3:6] = rng.normal(0.0, 1.0e5, (n, 3))
    ip = rng.integers(1, p.species + 1, n).astype(np.int32)
    return rp, ip


def cell_keys(p, rp):
    """((k+1)(Ny+4) + j+1)(Nx+4) + i+1 with (i, j, k) = floor((x - L_min)/d + 1),
    the node-centred cell holding the particle, clamped to [-1, N+2]."""
    lo = np.array([p.Lx_min, p.Ly_min, p.Lz_min])
    t = (rp[:, :3] - lo) / np.array(list(p.dxyz)) + 1.0
    frac = t - np.floor(t)
    # no particle within 1e-9 cells of a cell face, so the host's cell is the
    # device's whatever the rounding of either conversion
    assert np.all(np.minimum(frac, 1.0 - frac) > 1e-9)
    c = np.floor(t).astype(np.int64)
    c = np.clip(c, -1, np.array([p.nx, p.ny, p.nz]) + 2)
    return ((c[:, 2] + 1) * (p.ny + 4) + (c[:, 1] + 1)) * (p.nx + 4) + (c[:, 0] + 1)


def make(layout, nx=16, ny=12, nz=10, n=20000, seed=1, cells=None, **flows):
    p = small_plasma(n=8, ppc=4, seed=seed)
    p.nx, p.ny, p.nz = nx, ny, nz
    half = [500.0 * nx, 500.0 * ny, 500.0 * nz]
    p.xmin, p.xmax, p.ymin, p.ymax, p.zmin, p.zmax = -half[0], half[0], -half[1], half[1], -half[2], half[2]
    p.max_per_proc = 2 * n + 1024
    for k, v in flows.items():
        setattr(p, k, v)
    p = O.derive(p)
    g = Simulation(p, derive=False, **LAYOUTS[layout])
    rp, ip = random_particles(p, n, np.random.default_rng(seed), cells)
    g.set_particles(rp, ip)
    return p, g


@pytest.mark.parametrize("layout", list(LAYOUTS))
@pytest.mark.parametrize("case", ["shuffled", "clustered", "large_grid"])
def test_sort_equals_stable_argsort(layout, case):
    # shuffled: one run per particle on a 16x12x10 grid (2 radix passes);
    # clustered: 20,000 particles in 3^3 cells, ~700 per key (stability);
    # large_grid: 64x32x32, 3 radix passes over ~120,000 runs.
    if case == "shuffled":
        p, g = make(layout, n=20000, seed=2)
    elif case == "clustered":
        p, g = make(layout, n=20000, seed=3, cells=3)
    else:
        p, g = make(layout, nx=64, ny=32, nz=32, n=120000, seed=4)
    rp, ip = g.particles()
    order = np.argsort(cell_keys(p, rp), kind="stable")
    g.sort_particles()
    assert g.num_local == len(ip)
    rs, is_ = g.particles()
    np.testing.assert_array_equal(is_, ip[order])
    np.testing.assert_array_equal(rs, rp[order])
    # an already sorted array stays as it is
    g.sort_particles()
    r2, i2 = g.particles()
    np.testing.assert_array_equal(i2, is_)
    np.testing.assert_array_equal(r2, rs)
    g.close()


@pytest.mark.parametrize("layout", list(LAYOUTS))
def test_initialised_plasma_is_in_cell_order(layout):
    # ParticlesInitialize creates the particles cell by cell, x fastest: the
    # sort finds no run out of order and moves nothing.
    p = O.derive(small_haser(nx=16, ny=12, nz=10, ppc=4, seed=8))
    g = Simulation(p, derive=False, **LAYOUTS[layout])
    g.particles_initialize()
    rp, ip = g.particles()
    assert np.all(np.diff(cell_keys(p, rp)) >= 0)
    g.sort_particles()
    r2, i2 = g.particles()
    np.testing.assert_array_equal(i2, ip)
    np.testing.assert_array_equal(r2, rp)
    g.close()


@pytest.mark.parametrize("flows", [dict(), dict(yflow=0), dict(xflow=0, zflow=0)])
def test_deposit_after_sort_is_bit_identical(flows):
    # The same particles deposited before and after the sort (the tiled
    # kernel, in random order and in cell order): N and C bit for bit.
    p, g = make("cell32", n=60000, seed=5, **flows)
    g.particles_gridify()
    n0, c0 = g.field(capi.FIELD_N), g.field(capi.FIELD_C)
    g.sort_particles()
    g.particles_gridify()
    np.testing.assert_array_equal(g.field(capi.FIELD_N), n0)
    np.testing.assert_array_equal(g.field(capi.FIELD_C), c0)
    assert np.abs(n0).sum() > 0
    g.close()


def test_sorted_deposit_matches_oracle():
    # The deposit of sorted particles against the FP64 oracle's
    # ParticlesGridify of the same particles (the bar of the CELL32 deposit:
    # 1e-10 relative L2).
    p, g = make("cell32", n=40000, seed=6, yflow=0)
    g.sort_particles()
    g.particles_gridify()
    o = O.OracleState(p)
    o.set_particles(*g.particles())
    o.gridify()
    n_g = g.field(capi.FIELD_N)
    den = np.linalg.norm(o.N.ravel())
    assert np.linalg.norm((n_g - o.N).ravel()) / den < 1e-10
    g.close()


@pytest.mark.parametrize("layout", list(LAYOUTS))
def test_fused_loop_with_sort_holds_the_same_state(layout):
    # Six fused steps with the Haser source, sorting every other step, against
    # the same six steps unsorted: the same particle set, sweeps and fields,
    # bit for bit (the sort is a permutation and nothing downstream depends on
    # the order).
    p = O.derive(small_haser(nx=16, ny=12, nz=10, ppc=4, seed=9))
    runs = [Simulation(p, derive=False, **LAYOUTS[layout]) for _ in range(2)]
    for s in runs:
        s.calc_distance()
        s.particles_initialize()
    plain, sorted_ = runs
    sorted_.set_option(capi.OPT_SORT_EVERY, 2)
    assert sorted_.get_option(capi.OPT_SORT_EVERY) == 2
    sa = plain.run_fused(0, 6)
    sb = sorted_.run_fused(0, 6)
    assert sa == sb
    assert plain.num_local == sorted_.num_local
    ra, ia = sort_particles(*plain.particles())
    rb, ib = sort_particles(*sorted_.particles())
    np.testing.assert_array_equal(ia, ib)
    np.testing.assert_array_equal(ra, rb)
    for f in (capi.FIELD_N, capi.FIELD_U, capi.FIELD_E):
        np.testing.assert_array_equal(plain.field(f), sorted_.field(f))
    for s in runs:
        s.close()


def test_sort_option_is_checked():
    p, g = make("cell32", n=1000, seed=7)
    with pytest.raises(capi.PicardError):
        g.set_option(capi.OPT_SORT_EVERY, -1)
    assert g.get_option(capi.OPT_SORT_EVERY) == 0
    g.close()
