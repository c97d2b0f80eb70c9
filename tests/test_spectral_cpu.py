"""The closed form behind SOLVER_SPECTRAL, restated in numpy and checked
against the oracle's FP64 Jacobi sweeps (CalcEpotential.f90:55-96) on the
CPU: the iterate of sweep d is U_0 - af Q^T[(1 - g^d)/(1 - g) Q r_0] and its
residual norm is a Parseval sum, with Q the product of the per-axis sine
(open) or Fourier (periodic) bases.  The numpy code is a check of the method,
not the product (picard_b200/csrc/spectral.cu)."""
import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import rel_l2, small_plasma

EPS0 = 8.854187817e-12


def axis_basis(n, periodic):
    i = np.arange(n)
    if not periodic:
        m = np.arange(1, n + 1)
        return np.sqrt(2.0 / (n + 1)) * np.sin(np.pi * np.outer(m, i + 1) / (n + 1)), 2 * np.cos(np.pi * m / (n + 1))
    rows, sig = [np.full(n, 1 / np.sqrt(n))], [2.0]
    for f in range(1, (n + 1) // 2):
        for fn in (np.cos, np.sin):
            rows.append(np.sqrt(2.0 / n) * fn(2 * np.pi * f * i / n))
            sig.append(2 * np.cos(2 * np.pi * f / n))
    if n % 2 == 0:
        rows.append((-1.0) ** i / np.sqrt(n))
        sig.append(-2.0)
    return np.array(rows), np.array(sig)


def coefficients(p):
    dx, dy, dz = p.dxyz[0], p.dxyz[1], p.dxyz[2]
    S = (dx * dy) ** 2 + (dx * dz) ** 2 + (dy * dz) ** 2
    return 0.5 / S * (dy * dz) ** 2, 0.5 / S * (dx * dz) ** 2, 0.5 / S * (dx * dy) ** 2, 0.5 / S * (dx * dy * dz) ** 2


def laplacian(p, U, periodic):
    V = U.copy()
    # periodic axes: the ghosts hold the wrapped interior (numpy axes z, y, x)
    for ax, per in zip((2, 1, 0), periodic):
        if per:
            sl = [slice(None)] * 3
            src = [slice(None)] * 3
            sl[ax], src[ax] = 0, -2
            V[tuple(sl)] = V[tuple(src)]
            sl[ax], src[ax] = -1, 1
            V[tuple(sl)] = V[tuple(src)]
    dx, dy, dz = p.dxyz[0], p.dxyz[1], p.dxyz[2]
    c = V[1:-1, 1:-1, 1:-1]
    return ((V[1:-1, 1:-1, 2:] + V[1:-1, 1:-1, :-2] - 2 * c) / dx ** 2 + (V[1:-1, 2:, 1:-1] + V[1:-1, :-2, 1:-1] - 2 * c) / dy ** 2
            + (V[2:, 1:-1, 1:-1] + V[:-2, 1:-1, 1:-1] - 2 * c) / dz ** 2)


def spectral_solve(p, U0, Cg, maxerr, maxit, periodic=(False, False, False)):
    ax, ay, az, af = coefficients(p)
    b = -Cg / (p.dxyz[0] * p.dxyz[1] * p.dxyz[2] * EPS0)
    bint = b[1:-1, 1:-1, 1:-1]
    r0 = bint - laplacian(p, U0, periodic)
    (Qx, sx), (Qy, sy), (Qz, sz) = (axis_basis(n, per) for n, per in zip((p.nx, p.ny, p.nz), periodic))
    rh = np.einsum("ai,kji->kja", Qx, r0)
    rh = np.einsum("bj,kja->kba", Qy, rh)
    rh = np.einsum("ck,kba->cba", Qz, rh)
    omg = ax * (2 - sx)[None, None, :] + ay * (2 - sy)[None, :, None] + az * (2 - sz)[:, None, None]
    g = 1 - omg
    w = rh ** 2
    tol = maxerr * np.sqrt((bint ** 2).sum())
    d = 0
    for d in range(1, maxit):  # the check at the top of sweep d + 1 <= maxit
        if np.sqrt((w * np.abs(g) ** (2 * d)).sum()) <= tol:
            break
    else:
        d = 2 * maxit + 1
    gd = np.sign(g) ** d * np.abs(g) ** d
    uh = -af * (1 - gd) / omg * rh
    u = np.einsum("ck,cba->kba", Qz, uh)
    u = np.einsum("bj,kba->kja", Qy, u)
    u = np.einsum("ai,kja->kji", Qx, u)
    out = U0.copy()
    out[1:-1, 1:-1, 1:-1] += u
    return d, out


def jacobi_loop(p, U0, Cg, sweeps, periodic):
    """FP64 sweeps with the wrap taken from current values."""
    ax, ay, az, af = coefficients(p)
    b = -Cg / (p.dxyz[0] * p.dxyz[1] * p.dxyz[2] * EPS0)
    U = U0.copy()
    for _ in range(sweeps):
        U[1:-1, 1:-1, 1:-1] -= af * (b[1:-1, 1:-1, 1:-1] - laplacian(p, U, periodic))
    return U


@pytest.mark.parametrize("dims", [(24, 20, 16), (9, 13, 7)])
def test_closed_form_equals_oracle_sweeps(dims):
    p = small_plasma(n=8, ppc=4, seed=3)
    p.nx, p.ny, p.nz = dims
    p.xmin, p.xmax = -500.0 * dims[0], 500.0 * dims[0]
    p.ymin, p.ymax = -500.0 * dims[1], 500.0 * dims[1]
    p.zmin, p.zmax = -500.0 * dims[2], 500.0 * dims[2]
    p = O.derive(p)
    o = O.OracleState(p)
    o.calc_distance()
    o.initialize()
    for it in range(1, 4):
        o.step(it)
    o.bc_inflow(4)
    o.advance_position()
    o.bc_outflow()
    o.transfer()
    o.gridify()
    o.bc_potentials()
    U0, Cg = o.U.copy(), o.C.copy()
    s, conv, _ = o.calc_epotential()
    d, U = spectral_solve(p, U0, Cg, p.maxerr, p.maxit)
    assert conv and s > 20
    assert d == s
    assert rel_l2(U, o.U) < 1e-12


def test_closed_form_not_converged_takes_every_sweep():
    p = O.derive(small_plasma(n=6, ppc=1))
    o = O.OracleState(p)
    C = np.zeros_like(o.C)
    C[2:-2, 2:-2, 2:-2] = 1e-15
    o.C[...] = C
    s, conv, _ = o.calc_epotential(maxerr=1e-12, maxit=3)
    d, U = spectral_solve(p, np.zeros_like(o.U), C, 1e-12, 3)
    assert not conv and s == d == 7
    assert rel_l2(U, o.U) < 1e-12


@pytest.mark.parametrize("periodic", [(False, True, True), (True, False, False)])
def test_closed_form_with_periodic_axes_equals_wrapped_sweeps(periodic):
    p = small_plasma(n=8, ppc=1, seed=2)
    p.nx, p.ny, p.nz = 12, 10, 8
    p = O.derive(p)
    rng = np.random.default_rng(4)
    Cg = np.zeros((p.nz + 2, p.ny + 2, p.nx + 2))
    Cg[1:-1, 1:-1, 1:-1] = rng.normal(size=(p.nz, p.ny, p.nx)) * 1e-12
    U0 = np.zeros_like(Cg)
    U0[:, :, 0] = rng.normal(size=U0[:, :, 0].shape) * 1e-3  # an open face's boundary potential
    d, U = spectral_solve(p, U0, Cg, 1e-6, 1 << 20, periodic)
    ref = jacobi_loop(p, U0, Cg, d, periodic)
    assert d > 10
    assert rel_l2(U, ref) < 1e-12


def folded(n):
    """Qe, QoR of the folded sine basis: even modes from x[i] + x[n-1-i] (and
    the middle of an odd n), odd modes from x[i] - x[n-1-i] held at n-1-i."""
    Q, _ = axis_basis(n, False)
    h = n // 2
    hs = n - h
    Qe = Q[0::2, :hs]
    QoR = Q[1::2, :h][:, ::-1]
    return Q, Qe, QoR, h, hs


@pytest.mark.parametrize("n", [1, 2, 3, 8, 9, 128, 257])
def test_folded_sine_basis_equals_the_dense_one(n):
    # the in-place butterfly, the two half products and the inverse butterfly
    # reproduce y = Q x and x = Q^T y with modes in the order [even | odd]
    rng = np.random.default_rng(n)
    x = rng.normal(size=n)
    Q, Qe, QoR, h, hs = folded(n)
    f = x.copy()
    for i in range(h):
        a, b = f[i], f[n - 1 - i]
        f[i], f[n - 1 - i] = a + b, a - b
    y = np.concatenate([Qe @ f[:hs], QoR @ f[hs:]])
    dense = Q @ x
    np.testing.assert_allclose(y, np.concatenate([dense[0::2], dense[1::2]]), rtol=0, atol=1e-13 * np.abs(x).sum())
    g = np.concatenate([Qe.T @ y[:hs], QoR.T @ y[hs:]])
    for i in range(h):
        e, o = g[i], g[n - 1 - i]
        g[i], g[n - 1 - i] = e + o, e - o
    np.testing.assert_allclose(g, x, rtol=0, atol=1e-12 * np.abs(x).max())
