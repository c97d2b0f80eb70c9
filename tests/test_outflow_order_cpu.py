"""The parallel removal rule of the in-place BCoutflow kernels, on the CPU.

The kernels (picard_b200/csrc/outflow.cuh) fill every hole p below the
survivor count n' with the particle reached from p by q -> q + S(q), S(q) the
survivors above q, jumping in one step over the stretch where S stays
constant (to the first point q + kS past the next survivor, k found by
galloping and bisection on the survivor counts).  This file models that rule
with numpy (the same keep words, block offsets and probes) and checks it
against the oracle's literal
BCoutflow loop (BCoutflow.f90:24-83: walk from the end, move the current last
particle into each hole) on random and structured keep patterns.  Each
particle carries its original index in vz, so the order is compared exactly.
"""
import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import small_plasma

TILE = 2048  # particles per kernel block


def chase_model(keep: np.ndarray) -> np.ndarray:
    """Original index in each surviving slot, as the fill kernel computes it."""
    n = len(keep)
    nb = max(1, -(-n // TILE))
    k = np.zeros(nb * TILE, bool)
    k[:n] = keep
    words = k.reshape(-1, 32)
    bits = (words * (1 << np.arange(32, dtype=np.uint64))).sum(axis=1).astype(np.uint64)
    counts = words.sum(axis=1)
    per_block = counts.reshape(nb, TILE // 32)
    word_before = (np.cumsum(per_block, axis=1) - per_block).ravel()  # survivors before the word in its block
    block_counts = per_block.sum(axis=1)
    block_offsets = np.cumsum(block_counts) - block_counts
    np_ = int(block_counts.sum())

    def kept_through(q: int) -> int:
        w = int(bits[q >> 5])
        upto = w & ((1 << ((q & 31) + 1)) - 1)
        return int(block_offsets[q // TILE]) + int(word_before[q >> 5]) + bin(upto).count("1")

    out = np.arange(np_)
    for p in range(np_):
        if keep[p]:
            continue
        s = p
        for _ in range(n):
            kept = kept_through(s)
            above = np_ - kept
            assert above >= 1
            kmax = (n - 1 - s) // above
            assert kmax >= 1
            k = 1
            if kept_through(s + above) == kept:
                lo, hi = 1, 2
                while True:
                    h = min(hi, kmax)
                    if kept_through(s + h * above) > kept:
                        hi = h
                        break
                    assert h < kmax
                    lo, hi = h, 2 * hi
                while hi - lo > 1:
                    mid = lo + (hi - lo) // 2
                    if kept_through(s + mid * above) > kept:
                        hi = mid
                    else:
                        lo = mid
                k = hi
            s += k * above
            if keep[s]:
                break
        else:
            raise AssertionError("chain did not reach a survivor")
        out[p] = s
    return out


def oracle_order(keep: np.ndarray) -> np.ndarray:
    n = len(keep)
    p0 = small_plasma(n=4, ppc=1, seed=1)
    p0.max_per_proc = max(p0.max_per_proc, n + 1)
    p = O.derive(p0)
    assert p.xflow
    rp = np.zeros((n, 8))
    rp[:, 0] = 0.5 * (p.xmin + p.xmax)
    rp[:, 1] = 0.5 * (p.ymin + p.ymax)
    rp[:, 2] = 0.5 * (p.zmin + p.zmax)
    rp[~keep, 0] = p.xmax + 0.5 * p.dxyz[0]
    rp[:, 5] = np.arange(n)  # identity in vz
    o = O.OracleState(p)
    o.set_particles(rp, np.ones(n, np.int32))
    o.bc_outflow()
    r, _ = o.particles()
    return r[:, 5].astype(np.int64)


def patterns():
    rng = np.random.default_rng(5)
    out = []
    for n in (0, 1, 2, 31, 32, 33, 2047, 2048, 2049, 5000):
        out.append(np.ones(n, bool))
        out.append(np.zeros(n, bool))
        if n:
            last = np.zeros(n, bool)
            last[-1] = True
            out.append(last)
            alt = np.ones(n, bool)
            alt[::2] = False
            out.append(alt)
        for frac in (0.03, 0.5, 0.97):
            out.append(rng.random(n) > frac)
    # a removed run at the top above a few survivors, and the reverse
    k = np.ones(6000, bool)
    k[4000:5990] = False
    out.append(k)
    k = np.zeros(6000, bool)
    k[::997] = True
    out.append(k)
    # a long removed stretch spanning empty blocks before the only survivor
    k = np.zeros(3 * TILE + 17, bool)
    k[-1] = True
    out.append(k)
    k = np.ones(5 * TILE, bool)
    k[TILE // 2: 4 * TILE] = False
    out.append(k)
    # the per-subroutine loop's shape: a bulk with a few per cent outflowing,
    # then appended inflow candidates face by face, some faces removed almost
    # entirely (long removed stretches far above the holes of the bulk)
    bulk = rng.random(20000) > 0.03
    faces = [rng.random(1500) > f for f in (0.1, 0.995, 0.5, 1.0, 0.98, 0.3)]
    out.append(np.concatenate([bulk] + faces))
    return out


@pytest.mark.parametrize("k", range(len(patterns())))
def test_chase_rule_equals_the_reference_loop(k):
    keep = patterns()[k]
    want = oracle_order(keep)
    got = chase_model(keep)
    np.testing.assert_array_equal(got, want)
