"""Run parameters: a ctypes mirror of ``picard_params`` (include/picard_gpu.h).

The fields are the knobs ``program picard`` hard-codes (picard.f90:41-302) for a
single domain, plus the quantities it derives from them (picard.f90:333-467).
Species index ``s`` here is the reference's species ``s + 1`` (0 = electrons,
1 = H+), and two-index arrays keep the reference's memory order
(``v0[s][c]`` is ``v0(c+1, s+1)``).

``config_plain_32``, ``config_plain_scale`` and ``config_batch_run`` build the
workloads the benchmarks and tests use: the 32^3 two-species solar-wind plasma,
the 256x128x128 plasma with a Haser source, and the per-run grids of the
batched sweep.
"""
from __future__ import annotations

import ctypes as C
import math

# physical constants, picard.f90:56-66
TAU = 6.2831853071795864769252867665590
EC = 1.60217646e-19
MP = 1.6726216e-27
ME = 9.1093819e-31
EPS0 = 8.854187817e-12
KB = 1.380650e-23
MU0 = 1.25663706143591729538505735331180e-6

D8 = C.c_double * 8
I8 = C.c_int32 * 8
D84 = (C.c_double * 4) * 8
D4 = C.c_double * 4
D3 = C.c_double * 3


class PicardParams(C.Structure):
    _fields_ = [
        ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
        ("species", C.c_int32),
        ("max_per_proc", C.c_int32),
        ("xflow", C.c_int32), ("yflow", C.c_int32), ("zflow", C.c_int32),
        ("maxit", C.c_int32),
        ("produce_dt_scaled", C.c_int32),
        ("gyration", I8), ("fluid", I8),
        ("ppc", I8),
        ("xmin", C.c_double), ("xmax", C.c_double),
        ("ymin", C.c_double), ("ymax", C.c_double),
        ("zmin", C.c_double), ("zmax", C.c_double),
        ("dt", C.c_double), ("maxerr", C.c_double),
        ("mass", D8), ("charge", D8), ("density", D8), ("kelvin", D8),
        ("v0", D84),
        ("B0", D4),
        ("vn", D8), ("Qn", D8), ("nu_i", D8), ("nu_d", D8), ("Ek", D8),
        ("seed", C.c_uint64),
        ("Lx_min", C.c_double), ("Lx_max", C.c_double),
        ("Ly_min", C.c_double), ("Ly_max", C.c_double),
        ("Lz_min", C.c_double), ("Lz_max", C.c_double),
        ("dxyz", D3), ("dV", C.c_double),
        ("ipp", I8), ("epp", I8), ("hpp", I8),
        ("n2p", D8), ("eta", D8),
        ("ve", D4), ("E0", D4),
        ("tB", D84), ("sB", D84),
        ("u0", C.c_double),
    ]

    def copy(self) -> "PicardParams":
        out = PicardParams()
        C.memmove(C.byref(out), C.byref(self), C.sizeof(PicardParams))
        return out

    @property
    def nodes(self) -> int:
        return (self.nx + 2) * (self.ny + 2) * (self.nz + 2)

    @property
    def cells(self) -> int:
        return self.nx * self.ny * self.nz


def _base(nx: int, ny: int, nz: int, species: int) -> PicardParams:
    p = PicardParams()
    p.nx, p.ny, p.nz = nx, ny, nz
    p.species = species
    p.xflow = p.yflow = p.zflow = 1
    p.maxit = 2 ** 20
    p.produce_dt_scaled = 0
    for s in range(8):
        p.gyration[s] = 1
        p.fluid[s] = 0
        p.charge[s] = EC
        p.mass[s] = MP
    # picard.f90:192-199 default masses for species 3..5
    p.mass[2] = MP * 18.0
    p.mass[3] = MP * 4.0
    p.mass[4] = MP * 44.0
    return p


def plasma_dt(density: float, electron_mass: float, fraction: float = 0.05) -> float:
    """``fraction`` of the inverse electron plasma frequency sqrt(n e^2/(eps0 m_e))."""
    wpe = math.sqrt(density * EC * EC / (EPS0 * electron_mass))
    return fraction / wpe


def config_plain_32(seed: int = 0, n: int = 32, ppc: int = 16, capacity: int | None = None) -> PicardParams:
    """The 32^3 plain-method workload: cells of 1 km, H+ (1 amu) and electrons
    with mass ratio 100, 16 macro-particles per cell per species, 400 km/s
    drift along +x, kT = 10 eV, n = 5 cm^-3, B = 5 nT along z, dt = 0.05/w_pe,
    Jacobi tolerance 1e-6.  ``n`` and ``ppc`` shrink it for fast tests."""
    p = _base(n, n, n, 2)
    half = 1000.0 * n / 2
    p.xmin, p.xmax = -half, half
    p.ymin, p.ymax = -half, half
    p.zmin, p.zmax = -half, half
    p.mass[0] = MP / 100.0
    p.mass[1] = MP
    p.density[1] = 5.0e6
    p.ppc[1] = ppc
    kelvin = 10.0 * 1.1605e4
    p.kelvin[0] = kelvin
    p.kelvin[1] = kelvin
    for s in range(8):
        p.v0[s][0], p.v0[s][1], p.v0[s][2] = 4.0e5, 0.0, 0.0
    p.B0[0], p.B0[1], p.B0[2] = 0.0, 0.0, 5.0e-9
    p.dt = plasma_dt(5.0e6, p.mass[0])
    p.maxerr = 1.0e-6
    p.seed = seed
    cells = n * n * n
    p.max_per_proc = capacity if capacity is not None else int(cells * ppc * 2 * 1.25 + 64 * 6 * (n + 2) ** 2 * ppc)
    return p


def config_plain_scale(seed: int = 0, nx: int = 256, ny: int = 128, nz: int = 128, ppc_ion: int = 32,
                       capacity: int | None = None) -> PicardParams:
    """The at-scale plain workload: 256x128x128 cells of 1 km, 32 H+ + 32
    electrons per cell (64 ppc total, 268,435,456 particles), the same
    solar-wind plasma, plus a Haser source at the domain centre for an 18 amu
    ion: Q = 1e27 s^-1, neutral outflow 1 km/s, ionisation and destruction
    rates 1e-6 s^-1, excess energy 0.  The production rate is multiplied by dt
    (produce_dt_scaled = 1): ParticlesProduce.f90:70 as written treats the rate
    as a count per step, which at these parameters would create ~4e8
    macro-particles per step."""
    p = _base(nx, ny, nz, 3)
    p.xmin, p.xmax = -500.0 * nx, 500.0 * nx
    p.ymin, p.ymax = -500.0 * ny, 500.0 * ny
    p.zmin, p.zmax = -500.0 * nz, 500.0 * nz
    p.mass[0] = MP / 100.0
    p.mass[1] = MP
    p.mass[2] = MP * 18.0
    p.density[1] = 5.0e6
    p.ppc[1] = ppc_ion
    kelvin = 10.0 * 1.1605e4
    p.kelvin[0] = kelvin
    p.kelvin[1] = kelvin
    p.kelvin[2] = kelvin
    for s in range(8):
        p.v0[s][0], p.v0[s][1], p.v0[s][2] = 4.0e5, 0.0, 0.0
    p.B0[0], p.B0[1], p.B0[2] = 0.0, 0.0, 5.0e-9
    p.vn[2] = 1.0e3
    p.Qn[2] = 1.0e27
    p.nu_i[2] = 1.0e-6
    p.nu_d[2] = 1.0e-6
    p.Ek[2] = 0.0
    p.produce_dt_scaled = 1
    p.dt = plasma_dt(5.0e6, p.mass[0])
    p.maxerr = 1.0e-6
    p.seed = seed
    cells = nx * ny * nz
    face = 2 * ((ny + 2) * (nz + 2) + (nx + 2) * (nz + 2) + (nx + 2) * (ny + 2))
    p.max_per_proc = capacity if capacity is not None else int(cells * ppc_ion * 2 * 1.05 + face * ppc_ion * 2 + 1_000_000)
    return p


def expected_produced(p: PicardParams, steps: int) -> float:
    """Expected number of particles ParticlesProduce adds in ``steps``
    iterations (ions plus their co-produced electrons and protons), from the
    Haser density at each cell (ParticlesProduce.f90:40-70); ``p`` must be
    derived.  Used to size max_per_proc for runs with a neutral source."""
    import numpy as np

    dx, dy, dz = p.dxyz[0], p.dxyz[1], p.dxyz[2]
    dV = dx * dy * dz
    x0 = p.Lx_min + dx * np.arange(p.nx)
    y0 = p.Ly_min + dy * np.arange(p.ny)
    z0 = p.Lz_min + dz * np.arange(p.nz)
    X, Y, Z = np.meshgrid(x0, y0, z0, indexing="ij")
    r1 = np.sqrt((X + 0.5 * dx) ** 2 + (Y + 0.5 * dy) ** 2 + (Z + 0.5 * dz) ** 2)
    near = (4.0 * r1) ** 3 < dV
    if near.any():
        s = np.zeros(int(near.sum()))
        for fx in (0.25, 0.75):
            for fy in (0.25, 0.75):
                for fz in (0.25, 0.75):
                    s += np.sqrt((X[near] + fx * dx) ** 2 + (Y[near] + fy * dy) ** 2 + (Z[near] + fz * dz) ** 2)
        r1[near] = s / 8.0
    total = 0.0
    for s in range(p.species):
        if p.vn[s] <= 0.0 or p.n2p[s] <= 0.0:
            continue
        nden = p.Qn[s] / (2.0 * TAU * r1 * r1 * p.vn[s]) * np.exp(-p.nu_d[s] * r1 / p.vn[s])
        rate = p.nu_i[s] * nden * dV / p.n2p[s]
        if p.produce_dt_scaled:
            rate = rate * p.dt
        total += float(rate.sum()) * (1 + p.epp[s] + p.hpp[s])
    return total * steps


def _size_capacity(p: PicardParams, steps: int, ppc_ion: int) -> PicardParams:
    """max_per_proc for a run of ``steps`` iterations: the initial plasma with
    5% spare, a face of inflow, and the expected Haser production with 20%
    spare."""
    from .capi import params_derive

    q = params_derive(p)
    cells = p.nx * p.ny * p.nz
    face = 2 * ((p.ny + 2) * (p.nz + 2) + (p.nx + 2) * (p.nz + 2) + (p.nx + 2) * (p.ny + 2))
    p.max_per_proc = int(cells * ppc_ion * 2 * 1.05 + face * ppc_ion * 2 + 1.2 * expected_produced(q, steps) + 65536)
    return p


def config_batch_run(rng, seed: int) -> tuple[PicardParams, int]:
    """One run of the batched parameter sweep: a cubic grid of edge drawn from
    16..96 cells (1 km cells), 8..32 macro-particles per cell in total (half
    H+, half electrons), drift drawn from 300..800 km/s along +x, |B| drawn from
    1..10 nT in an isotropic random direction, the 32^3 workload's plasma
    otherwise, no neutral source, 100 steps.  ``rng`` is a numpy Generator."""
    n = int(rng.integers(16, 97))
    ppc_ion = max(1, int(rng.integers(8, 33)) // 2)
    p = config_plain_32(seed=seed, n=n, ppc=ppc_ion)
    v = float(rng.uniform(300e3, 800e3))
    for s in range(8):
        p.v0[s][0] = v
    bmag = float(rng.uniform(1e-9, 10e-9))
    u = rng.normal(size=3)
    u = u / math.sqrt(float((u * u).sum()))
    p.B0[0], p.B0[1], p.B0[2] = (bmag * float(c) for c in u)
    steps = 100
    return _size_capacity(p, steps, ppc_ion), steps


def config_serving_run(rng, seed: int) -> tuple[PicardParams, int]:
    """One request of the serving stream: the at-scale plasma with a Haser
    source on a cubic grid of edge drawn from 24..128 cells, 8..64
    macro-particles per cell in total, Q log-uniform in [1e25, 1e28] s^-1,
    200 steps."""
    n = int(rng.integers(24, 129))
    ppc_ion = max(1, int(rng.integers(8, 65)) // 2)
    p = config_plain_scale(seed=seed, nx=n, ny=n, nz=n, ppc_ion=ppc_ion)
    p.Qn[2] = float(10.0 ** rng.uniform(25.0, 28.0))
    steps = 200
    return _size_capacity(p, steps, ppc_ion), steps


def serving_stream(seed: int, count: int, rate_per_s: float = 20.0):
    """``count`` requests with Poisson arrivals at ``rate_per_s``: a list of
    (arrival seconds, params, steps), run seeds seed*1000 + i."""
    import numpy as np

    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(count):
        t += float(rng.exponential(1.0 / rate_per_s))
        p, steps = config_serving_run(rng, seed * 1000 + i)
        out.append((t, p, steps))
    return out


def batch_set(seed: int, count: int = 64):
    """The batched sweep's ``count`` runs: a list of (params, steps)."""
    import numpy as np

    rng = np.random.default_rng(seed)
    return [config_batch_run(rng, seed * 1000 + i) for i in range(count)]
