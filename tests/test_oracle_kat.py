"""Known-answer tests pinning the FP64 oracle (CPU only).

The reference ships no tests or golden vectors, so the oracle is pinned by
(1) the published Philox4x32-10 test vectors, (2) the parameter derivation of
picard.f90:333-467 evaluated by hand for the 32^3 workload, and (3) physics
identities each routine must satisfy.
"""
import math

import numpy as np
import pytest

from oracle import oracle as O
from picard_b200 import params as P
from tests.helpers import cell_indices, small_haser, small_plasma


# Random123 kat_vectors for philox4x32_10 (Salmon et al., SC'11)
PHILOX_KAT = [
    ([0, 0, 0, 0], [0, 0], [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]),
    ([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2, [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]),
    ([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], [0xA4093822, 0x299F31D0],
     [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]),
]


@pytest.mark.parametrize("ctr,key,want", PHILOX_KAT)
def test_philox_published_vectors(ctr, key, want):
    assert O.philox4x32_10(ctr, key) == want


def test_site_uniforms_in_unit_interval_and_distinct():
    u = np.array([O.site_uniform(5, 1, 2, 3, 2, n) for n in range(64)])
    assert np.all(u >= 0.0) and np.all(u < 1.0)
    assert len(set(u.tolist())) == 64
    # different tags give different streams
    assert O.site_uniform(5, 1, 2, 3, 1, 0) != O.site_uniform(5, 1, 2, 3, 2, 0)


def test_derive_plain_32_by_hand():
    p = O.derive(P.config_plain_32())
    # one ion species with one electron per ion (picard.f90:384-392)
    assert list(p.ipp)[:3] == [0, 16, 0]
    assert list(p.epp)[:2] == [0, 1] and p.hpp[1] == 0
    assert list(p.ppc)[:2] == [16, 16]
    dV = 1000.0 ** 3
    assert p.dV == pytest.approx(dV, rel=1e-15)
    assert p.n2p[0] == pytest.approx(dV * 5e6 / 16, rel=1e-15)
    assert p.n2p[1] == pytest.approx(dV * 5e6 / 16, rel=1e-15)
    assert p.density[0] == pytest.approx(5e6, rel=1e-15)
    # dt = 0.05 / w_pe, w_pe = sqrt(n e^2 / (eps0 m_e)) with m_e = m_p / 100
    wpe = math.sqrt(5e6 * P.EC ** 2 / (P.EPS0 * P.MP / 100))
    assert p.dt == pytest.approx(0.05 / wpe, rel=1e-14)
    assert p.dt == pytest.approx(1.698e-6, rel=1e-3)
    # mass-weighted bulk velocity = the common drift; E0 = -ve x B0
    assert list(p.ve)[:3] == pytest.approx([4e5, 0.0, 0.0])
    assert list(p.E0)[:3] == pytest.approx([0.0, 4e5 * 5e-9, 0.0])
    # Boris factors (picard.f90:452-466)
    t = 0.5 * p.dt * 5e-9 * (-P.EC / (P.MP / 100))
    assert p.tB[0][2] == pytest.approx(t, rel=1e-14)
    assert p.sB[0][2] == pytest.approx(2 * t / (1 + t * t), rel=1e-14)


def test_derive_haser_species_three_inactive_upstream():
    p = O.derive(P.config_plain_scale(nx=8, ny=4, nz=4, ppc_ion=32))
    assert p.ppc[2] == 0 and p.density[2] == 0.0       # produced only by the Haser source
    assert p.epp[2] == 1                                  # one electron per produced ion
    assert p.n2p[2] == p.n2p[0]                           # picard.f90:399


def test_initial_plasma_is_neutral_and_jacobi_exits_before_sweep_one():
    p = O.derive(small_plasma(n=6, ppc=3))
    s = O.OracleState(p)
    s.calc_distance()
    s.initialize()
    assert s.num_local == 6 ** 3 * 3 * 2
    s.gridify()
    assert np.abs(s.C).max() == 0.0   # co-located electrons (ParticlesInitialize.f90:85)
    s.bc_potentials()
    sweeps, conv, _ = s.calc_epotential()
    assert sweeps == 0 and conv


def test_cic_weights_conserve_particle_number():
    p = O.derive(small_plasma(n=6, ppc=3, seed=11))
    s = O.OracleState(p)
    s.initialize()
    # move everybody so that the stencils straddle the open faces
    s.advance_position(dt=p.dt * 2000)
    s.bc_outflow()
    s.transfer()
    s.gridify()
    rp, ip = s.particles()
    for sp in (1, 2):
        count = int((ip == sp).sum())
        assert s.N[..., sp - 1].sum() == pytest.approx(count * p.n2p[sp - 1], rel=1e-12)
    # open faces: the ghost layers are folded away (ParticlesGridify.f90:149-171)
    assert np.abs(s.N[0]).max() == 0 and np.abs(s.N[-1]).max() == 0
    assert np.abs(s.N[:, 0]).max() == 0 and np.abs(s.N[:, :, -1]).max() == 0


def test_periodic_fold_mirrors_ghosts():
    p = small_plasma(n=6, ppc=2, seed=5)
    p.yflow = 0
    p = O.derive(p)
    s = O.OracleState(p)
    s.initialize()
    s.advance_position(dt=p.dt * 3000)
    s.bc_outflow()
    s.transfer()
    s.gridify()
    # node 1 == node Ny+1 and node 2 == node Ny+2 on the periodic axis
    assert np.array_equal(s.N[:, 0], s.N[:, p.ny])
    assert np.array_equal(s.N[:, p.ny + 1], s.N[:, 1])


def test_outflow_and_transfer_sets():
    p = small_plasma(n=5, ppc=2, seed=9)
    p.zflow = 0
    p = O.derive(p)
    s = O.OracleState(p)
    s.initialize()
    s.advance_position(dt=p.dt * 4000)
    rp, ip = s.particles()
    x = rp[:, :3]
    keep = ((x[:, 0] >= p.xmin) & (x[:, 0] <= p.xmax) & (x[:, 1] >= p.ymin) & (x[:, 1] <= p.ymax))
    s.bc_outflow()
    assert s.num_local == int(keep.sum())
    s.transfer()
    rq, _ = s.particles()
    assert np.all(rq[:, 2] >= p.zmin) and np.all(rq[:, 2] <= p.zmax)


def test_linear_potential_gives_constant_field():
    p = O.derive(small_plasma(n=6, ppc=1))
    s = O.OracleState(p)
    z, y, x = np.meshgrid(*[np.arange(n + 2) for n in (p.nz, p.ny, p.nx)], indexing="ij")
    g = np.array([3.0, -2.0, 0.5])
    s.U[...] = g[0] * x * p.dxyz[0] + g[1] * y * p.dxyz[1] + g[2] * z * p.dxyz[2]
    s.calc_efield()
    s.bc_fields()
    inner = s.E[1:-1, 1:-1, 1:-1]
    for c in range(3):
        np.testing.assert_allclose(inner[..., c], -g[c], rtol=1e-12)
    assert np.abs(s.E[0]).max() == 0 and np.abs(s.E[:, :, -1]).max() == 0


def test_point_charge_boundary_potential_is_coulomb():
    p = O.derive(small_plasma(n=6, ppc=1))
    s = O.OracleState(p)
    s.calc_distance()
    q = 1e-9
    ci = (3, 2, 4)  # 1-based cell (i, j, k) -> node index (i, j, k) in the padded box
    s.C[ci[2], ci[1], ci[0]] = q
    s.bc_potentials()
    # x0 face node (1, j, k) at x = Lx_min - dx/2
    for (j, k) in [(1, 1), (3, 5), (6, 6)]:
        dx = (ci[0] - 0) * p.dxyz[0]
        dy = (ci[1] - j) * p.dxyz[1]
        dz = (ci[2] - k) * p.dxyz[2]
        r = math.sqrt(dx * dx + dy * dy + dz * dz)
        assert s.U[k, j, 0] == pytest.approx(q / (4 * math.pi * P.EPS0 * r), rel=1e-13)
    # face edges and corners stay zero (BCpotentials.f90:71-76)
    assert s.U[0, 0, 0] == 0.0 and s.U[-1, 0, 0] == 0.0


def _one_particle_state(p, v, e_field):
    s = O.OracleState(p)
    rp = np.zeros((1, 8))
    rp[0, :3] = [0.3 * p.dxyz[0], -0.2 * p.dxyz[1], 0.1 * p.dxyz[2]]
    rp[0, 3:6] = v
    s.set_particles(rp, np.array([2], np.int32))
    s.E[...] = e_field
    return s


def test_boris_pure_rotation_keeps_speed_in_drift_frame():
    p = O.derive(small_plasma(n=4, ppc=1))
    v = np.array([4.3e5, 2.1e4, -1.7e4])
    s = _one_particle_state(p, v, 0.0)
    for _ in range(50):
        s.advance_velocity()
    w = s.particles()[0][0, 3:6] - np.array(list(p.ve)[:3])
    assert np.linalg.norm(w) == pytest.approx(np.linalg.norm(v - np.array(list(p.ve)[:3])), rel=1e-13)


def test_boris_exb_drift_is_stationary():
    p = O.derive(small_plasma(n=4, ppc=1))
    B = np.array(list(p.B0)[:3])
    E1 = np.array([1e-4, -2e-4, 0.0])        # perpendicular to B = B z
    vd = np.cross(E1, B) / B.dot(B)
    v = np.array(list(p.ve)[:3]) + vd
    s = _one_particle_state(p, v, E1)
    s.advance_velocity()
    np.testing.assert_allclose(s.particles()[0][0, 3:6], v, rtol=1e-12, atol=1e-9)


def test_exp_imp_half_steps_compose_and_keep_speed_without_field():
    p = O.derive(small_plasma(n=4, ppc=1))
    v = np.array([3.1e5, -4.0e4, 2.5e4])
    s = _one_particle_state(p, v, 0.0)
    s.advance_velocity(mode=2, deltat=0.5 * p.dt)   # Imp
    s.advance_velocity(mode=1, deltat=0.5 * p.dt)   # Exp
    w = s.particles()[0][0, 3:6] - np.array(list(p.ve)[:3])
    assert np.linalg.norm(w) == pytest.approx(np.linalg.norm(v - np.array(list(p.ve)[:3])), rel=1e-13)


def test_jacobi_converges_to_discrete_solution():
    p = O.derive(small_plasma(n=10, ppc=1))
    s = O.OracleState(p)
    nz, ny, nx = s.U.shape
    rng = np.random.default_rng(1)
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    ustar = np.sin(np.pi * x / (nx - 1)) * np.sin(np.pi * y / (ny - 1)) * np.sin(np.pi * z / (nz - 1))
    ustar += 0.01 * rng.standard_normal(ustar.shape)
    d = p.dxyz
    lap = np.zeros_like(ustar)
    lap[1:-1, 1:-1, 1:-1] = ((ustar[1:-1, 1:-1, 2:] + ustar[1:-1, 1:-1, :-2] - 2 * ustar[1:-1, 1:-1, 1:-1]) / d[0] ** 2
                             + (ustar[1:-1, 2:, 1:-1] + ustar[1:-1, :-2, 1:-1] - 2 * ustar[1:-1, 1:-1, 1:-1]) / d[1] ** 2
                             + (ustar[2:, 1:-1, 1:-1] + ustar[:-2, 1:-1, 1:-1] - 2 * ustar[1:-1, 1:-1, 1:-1]) / d[2] ** 2)
    s.C[...] = -lap * p.dV * P.EPS0           # b = -C/(dV eps0) = lap
    s.U[...] = ustar
    s.U[1:-1, 1:-1, 1:-1] = 0.0
    sweeps, conv, res = s.calc_epotential(maxerr=1e-10)
    assert conv and sweeps > 10
    assert res[0] <= 1e-10 * res[1]
    inner = (slice(1, -1),) * 3
    assert np.abs(s.U[inner] - ustar[inner]).max() < 1e-6 * np.abs(ustar).max()


def test_jacobi_cap_runs_two_maxit_plus_one():
    p = O.derive(small_plasma(n=6, ppc=1))
    s = O.OracleState(p)
    s.C[2:-2, 2:-2, 2:-2] = 1e-15
    sweeps, conv, _ = s.calc_epotential(maxerr=1e-12, maxit=3)
    assert not conv and sweeps == 7


def test_inflow_fills_guard_shell_once():
    p = O.derive(small_plasma(n=4, ppc=2, seed=1))
    s = O.OracleState(p)
    s.bc_inflow(iteration=1)
    rp, ip = s.particles()
    per_cell = 2 * 2      # 2 ions + 2 electrons
    shell = 6 ** 3 - 4 ** 3 - 12 * 1 - 8    # six faces + edges covered once; BCinflow skips some edges
    # x faces: 2*(Ny+2)(Nz+2); +y: Nx(Nz+1); -y: Nx(Nz+1); +z: Nx(Ny+1); -z: Nx(Ny+1)
    cells = 2 * 6 * 6 + 4 * 5 * 2 + 4 * 5 * 2
    assert s.num_local == cells * per_cell
    ijk = cell_indices(p, rp)
    x = rp[:, :3]
    lo = np.array([p.xmin, p.ymin, p.zmin]) - np.array(list(p.dxyz))
    hi = np.array([p.xmax, p.ymax, p.zmax]) + np.array(list(p.dxyz))
    assert np.all(x >= lo) and np.all(x < hi)
    inside = np.all((x >= [p.xmin, p.ymin, p.zmin]) & (x <= [p.xmax, p.ymax, p.zmax]), axis=1)
    assert not inside.any()
    assert ijk.min() >= 1


def test_produce_counts_follow_haser_rate():
    p = O.derive(small_haser(nx=8, ny=8, nz=8, ppc=1, q=3e24, dt_scaled=0))
    s = O.OracleState(p)
    s.produce(iteration=1)
    rp, ip = s.particles()
    assert s.num_local > 0
    ions = ip == 3
    assert (ip == 1).sum() == ions.sum()           # one electron per ion (epp(3) = 1)
    # produced ions move radially outward at vn (ui = 0 for Ek = 0)
    x = rp[ions, :3]
    v = rp[ions, 3:6]
    np.testing.assert_allclose(np.linalg.norm(v, axis=1), p.vn[2], rtol=1e-12)
    assert np.all(np.einsum("ij,ij->i", x, v) > 0)
