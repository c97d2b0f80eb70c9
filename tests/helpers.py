"""Shared helpers of the test suite: small workloads and comparisons."""
from __future__ import annotations

import numpy as np

from picard_b200 import params as P


def small_plasma(n: int = 8, ppc: int = 4, seed: int = 7, **kw) -> P.PicardParams:
    """The 32^3 solar-wind workload shrunk to n^3 cells and ppc ions per cell."""
    p = P.config_plain_32(seed=seed, n=n, ppc=ppc)
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def small_haser(nx=16, ny=8, nz=8, ppc=4, seed=3, dt_scaled=1, q=1e27) -> P.PicardParams:
    """The Haser-source workload shrunk; q large enough that ions are produced."""
    p = P.config_plain_scale(seed=seed, nx=nx, ny=ny, nz=nz, ppc_ion=ppc)
    p.Qn[2] = q
    p.produce_dt_scaled = dt_scaled
    return p


def rel_l2(a: np.ndarray, b: np.ndarray) -> float:
    den = np.linalg.norm(b.ravel())
    num = np.linalg.norm((a - b).ravel())
    return float(num / den) if den > 0 else float(num)


def sort_particles(rp: np.ndarray, ip: np.ndarray):
    """Canonical order (species, x, y, z, vx, vy, vz) so that sets compare."""
    keys = (rp[:, 5], rp[:, 4], rp[:, 3], rp[:, 2], rp[:, 1], rp[:, 0], ip)
    o = np.lexsort(keys)
    return rp[o], ip[o]


def cell_indices(p: P.PicardParams, rp: np.ndarray) -> np.ndarray:
    """index_local of AdvanceVelocity.f90:49-51 (1-based, truncation)."""
    lo = np.array([p.Lx_min, p.Ly_min, p.Lz_min])
    d = np.array(list(p.dxyz))
    return 1 + ((rp[:, :3] - lo) / d + 0.5).astype(np.int64)



def unmatched_particles(ra: np.ndarray, ia: np.ndarray, rb: np.ndarray, ib: np.ndarray, pos_atol: float,
                        vel_atol: float) -> int:
    """Particles of either set without a partner in the other.  Partners have
    the same species, are each other's nearest neighbour in (position /
    pos_atol, velocity / vel_atol) space, and lie within ``pos_atol`` of each
    other on every position axis and within ``vel_atol`` on every velocity
    axis."""
    from scipy.spatial import cKDTree

    miss = 0
    for s in np.union1d(np.unique(ia), np.unique(ib)):
        a = ra[ia == s, :6] / np.array([pos_atol] * 3 + [vel_atol] * 3)
        b = rb[ib == s, :6] / np.array([pos_atol] * 3 + [vel_atol] * 3)
        if len(a) == 0 or len(b) == 0:
            miss += len(a) + len(b)
            continue
        _, ab = cKDTree(b).query(a)
        _, ba = cKDTree(a).query(b)
        mutual = ba[ab] == np.arange(len(a))
        close = np.all(np.abs(a - b[ab]) <= 1.0, axis=1)
        matched = int(np.count_nonzero(mutual & close))
        miss += (len(a) - matched) + (len(b) - matched)
    return miss
