"""The counting sort by CIC stencil (picard_gpu_sort_particles) and the
warp-aggregated tiled deposit that takes sorted particles.

On one rank ParticlesTransfer.f90:488-519 only wraps coordinates; the sort
sits in its slot.  Bars: the sort equals numpy's stable argsort of the stencil
keys (base node x fastest, then y and z, species within a node) bit for bit,
on shuffled, clustered and already sorted arrays in both layouts; the
deposit gives the same N bits whatever the kernel and the order; and the
fused loop with a sort every other step holds exactly the same particles
(as a set), the same sweep counts and the same N, U and E bits as without.
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


def stencil_keys(p, rp, ip):
    """((k+1)(Ny+3) + j+1)(Nx+3) + i+1) S + s: the 0-based CIC base node
    (ParticlesGridify.f90:65-67) clamped to [-1, N+1], species 0-based."""
    lo = np.array([p.Lx_min, p.Ly_min, p.Lz_min])
    t = (rp[:, :3] - lo) / np.array(list(p.dxyz)) + 0.5
    frac = t - np.floor(t)
    # no particle within 1e-9 cells of a node plane, so the host's base node
    # is the device's whatever the rounding of either conversion
    assert np.all(np.minimum(frac, 1.0 - frac) > 1e-9)
    b = np.floor(t).astype(np.int64)
    hi = np.array([p.nx, p.ny, p.nz]) + 1
    b = np.clip(b, -1, hi)
    node = ((b[:, 2] + 1) * (p.ny + 3) + (b[:, 1] + 1)) * (p.nx + 3) + (b[:, 0] + 1)
    return node * p.species + (ip.astype(np.int64) - 1)


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
    # clustered: 20,000 particles in 3^3 cells, ~300 per key (stability);
    # large_grid: 64x32x32, 3 radix passes over ~120,000 runs.
    if case == "shuffled":
        p, g = make(layout, n=20000, seed=2)
    elif case == "clustered":
        p, g = make(layout, n=20000, seed=3, cells=3)
    else:
        p, g = make(layout, nx=64, ny=32, nz=32, n=120000, seed=4)
    rp, ip = g.particles()
    order = np.argsort(stencil_keys(p, rp, ip), kind="stable")
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


@pytest.mark.parametrize("flows", [dict(), dict(yflow=0), dict(xflow=0, zflow=0)])
def test_stencil_deposit_equals_tiled_deposit(flows):
    # The same particles deposited by the tiled kernel (OPT_DEPOSIT 1) and its
    # warp-aggregated form (2), unsorted and sorted: N and C bit for bit.
    p, g = make("cell32", n=60000, seed=5, **flows)
    out = []
    for sort in (False, True):
        if sort:
            g.sort_particles()
        for kernel in (1, 2):
            g.set_option(capi.OPT_DEPOSIT, kernel)
            g.particles_gridify()
            out.append((g.field(capi.FIELD_N), g.field(capi.FIELD_C)))
    for n_, c_ in out[1:]:
        np.testing.assert_array_equal(n_, out[0][0])
        np.testing.assert_array_equal(c_, out[0][1])
    assert np.abs(out[0][0]).sum() > 0
    g.close()


def test_stencil_deposit_matches_oracle():
    # The warp-aggregated kernel on sorted particles against the FP64 oracle's
    # ParticlesGridify of the same particles (the bar of the other CELL32
    # deposits: 1e-10 relative L2).
    p, g = make("cell32", n=40000, seed=6, yflow=0)
    g.sort_particles()
    g.set_option(capi.OPT_DEPOSIT, 2)
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
    with pytest.raises(capi.PicardError):
        g.set_option(capi.OPT_DEPOSIT, 3)
    assert g.get_option(capi.OPT_DEPOSIT) == 0
    g.close()
