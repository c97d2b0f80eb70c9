"""The run decomposition behind the counting sort by stencil (sort.cu),
restated in numpy and checked against a stable argsort on the CPU.

The device sort splits the particle array into runs of equal keys, sorts the
runs by key with a stable 8-bit LSD radix sort over run ids, and sends each
particle to its run's destination (an exclusive scan of the run lengths in
sorted order) plus its place in the run.  This restatement follows the same
steps, pass by pass, so the rule is checked on inputs the GPU tests do not
reach: empty and single-key arrays, one particle per run, ties across many
2,048-particle tiles, and keys that need four radix passes.
"""
import numpy as np
import pytest


def stable_sort_by_runs(keys: np.ndarray, key_bits: int) -> np.ndarray:
    """Destination of every element (a permutation), built as sort.cu does."""
    n = len(keys)
    if n == 0:
        return np.zeros(0, np.int64)
    head = np.ones(n, bool)
    head[1:] = keys[1:] != keys[:-1]
    run_start = np.flatnonzero(head)
    run_key = keys[run_start]
    run_start = np.append(run_start, n)
    ids = np.arange(len(run_key))
    k = run_key.copy()
    passes = max(1, (key_bits + 7) // 8)
    for ps in range(passes):
        digit = (k >> (8 * ps)) & 255
        # per digit, counts in order: a stable counting pass
        order = np.argsort(digit, kind="stable")
        k, ids = k[order], ids[order]
    length = run_start[ids + 1] - run_start[ids]
    off = np.concatenate(([0], np.cumsum(length)[:-1]))
    run_dst = np.empty(len(ids), np.int64)
    run_dst[ids] = off
    run_of = np.cumsum(head) - 1
    return run_dst[run_of] + (np.arange(n) - run_start[run_of])


@pytest.mark.parametrize("case", ["random", "sorted", "one_key", "tiles", "wide", "empty", "single"])
def test_runs_sort_equals_stable_argsort(case):
    rng = np.random.default_rng(11)
    if case == "random":
        keys, bits = rng.integers(0, 5000, 20000), 13
    elif case == "sorted":
        keys, bits = np.sort(rng.integers(0, 5000, 20000)), 13
    elif case == "one_key":
        keys, bits = np.full(7000, 42), 13
    elif case == "tiles":
        # long runs crossing 2,048-element tiles, interleaved keys
        keys, bits = np.repeat(rng.integers(0, 40, 300), rng.integers(1, 200, 300)), 6
    elif case == "wide":
        keys, bits = rng.integers(0, 2**31, 50000), 31
    elif case == "empty":
        keys, bits = np.zeros(0, np.int64), 8
    else:
        keys, bits = np.array([9]), 8
    keys = keys.astype(np.int64)
    dst = stable_sort_by_runs(keys, bits)
    out = np.empty_like(keys)
    out[dst] = keys
    assert np.array_equal(np.sort(dst), np.arange(len(keys)))
    assert np.array_equal(out, keys[np.argsort(keys, kind="stable")])
    # stability: the element that lands at each position is the one a stable
    # argsort puts there
    src = np.empty(len(keys), np.int64)
    src[dst] = np.arange(len(keys))
    assert np.array_equal(src, np.argsort(keys, kind="stable"))
