"""Seeded synthetic inputs for the benchmark configurations (host-side).

The reference's generator (src/generate_dataset.cpp) seeds from
std::random_device, so its datasets cannot be reproduced; these generators are
deterministic given a seed and run in the library's C++ host code
(si_gen_uniform) or numpy.
"""
from __future__ import annotations

import ctypes

import numpy as np

from ._lib import check, lib


def uniform(seed: int, n: int, hi: int, lo: int = 0, threads: int = 0) -> np.ndarray:
    """n distinct uint32 drawn uniformly without replacement from [lo, hi), ascending."""
    out = np.empty(n, dtype=np.uint32)
    st = lib.si_gen_uniform(seed, n, lo, hi, out.ctypes.data_as(ctypes.c_void_p), threads)
    check(st, "si_gen_uniform")
    return out


def sisi_plain(seed_a: int = 1, seed_b: int = 2, n: int = 1 << 20, universe: int = 1 << 24):
    """|A| = |B| = 2^20 from [0, 2^24), seeds 1 and 2 (the plain single-pair case)."""
    return uniform(seed_a, n, universe), uniform(seed_b, n, universe)


def sisi_large(seed_a: int = 3, seed_b: int = 4, n: int = 1 << 28, universe: int = 1 << 31):
    """|A| = |B| = 2^28 from [0, 2^31) (the large single-pair case)."""
    return uniform(seed_a, n, universe), uniform(seed_b, n, universe)


def sisi_skewed(seed: int = 5, n_small: int = 1 << 16, n_large: int = 1 << 26,
                universe: int = 1 << 30, planted_frac: float = 0.2):
    """|A| = 2^16, |B| = 2^26 from [0, 2^30), with round(0.2*|A|) elements of A
    planted into B.  B's other elements are uniform over the universe minus the
    planted values (rank mapping), so |B| is exact."""
    a = uniform(seed, n_small, universe)
    n_plant = int(round(planted_frac * n_small))
    pick = uniform(seed + 1000003, n_plant, n_small)          # indices into a
    planted = a[pick.astype(np.int64)]
    w = uniform(seed + 2000003, n_large - n_plant, universe - n_plant).astype(np.int64)
    # map w in [0, U - P) to the w-th value of [0, U) that is not planted
    q = planted.astype(np.int64) - np.arange(n_plant, dtype=np.int64)
    rest = w + np.searchsorted(q, w, side="right")
    b = np.empty(n_large, dtype=np.uint32)
    pos_p = np.searchsorted(rest, planted.astype(np.int64)) + np.arange(n_plant)
    mask = np.ones(n_large, dtype=bool)
    mask[pos_p] = False
    b[pos_p] = planted
    b[mask] = rest.astype(np.uint32)
    return a, b


def bernoulli(seed: int, k: int, n_values: int, p: float, threads: int = 0):
    """k sets over [0, n_values), each value a member with probability p.
    Returns (elements uint32, offsets int64[k + 1]) in CSR form."""
    offsets = np.empty(k + 1, dtype=np.uint64)
    st = lib.si_gen_bernoulli(seed, k, n_values, p, offsets.ctypes.data_as(ctypes.c_void_p), None, threads)
    check(st, "si_gen_bernoulli")
    elements = np.empty(int(offsets[-1]), dtype=np.uint32)
    st = lib.si_gen_bernoulli(seed, k, n_values, p, offsets.ctypes.data_as(ctypes.c_void_p),
                              elements.ctypes.data_as(ctypes.c_void_p), threads)
    check(st, "si_gen_bernoulli")
    return elements, offsets.astype(np.int64)


def misi_dense(seed: int = 6, k: int = 16384, n_values: int = 65536, p: float = 0.05):
    """The dense all-pairs collection: 16384 sets over 65536 values,
    Bernoulli(0.05) membership."""
    return bernoulli(seed, k, n_values, p)


def powerlaw(seed: int, k: int, n_min: int, n_max: int, size_exp: float, universe: int, value_exp: float,
             threads: int = 0):
    """k sets, sizes ~ n^-size_exp on [n_min, n_max], distinct values of
    [1, universe] with Zipf(value_exp) popularity.  Set a depends only on
    (seed, a), so the first j sets of a collection are the collection of j
    sets.  Returns (elements uint32, offsets int64[k + 1])."""
    offsets = np.empty(k + 1, dtype=np.uint64)
    args = (seed, k, n_min, n_max, size_exp, universe, value_exp)
    st = lib.si_gen_powerlaw(*args, offsets.ctypes.data_as(ctypes.c_void_p), None, threads)
    check(st, "si_gen_powerlaw")
    elements = np.empty(int(offsets[-1]), dtype=np.uint32)
    st = lib.si_gen_powerlaw(*args, offsets.ctypes.data_as(ctypes.c_void_p),
                             elements.ctypes.data_as(ctypes.c_void_p), threads)
    check(st, "si_gen_powerlaw")
    return elements, offsets.astype(np.int64)


def misi_powerlaw(seed: int = 7, k: int = 8192):
    """The power-law all-pairs collection: 8192 sets, sizes ~ n^-1.1 on
    [16, 65536], values of [1, 2^20] with Zipf(0.8) popularity."""
    return powerlaw(seed, k, 16, 65536, 1.1, 1 << 20, 0.8)


def loguniform(seed: int, k: int, n_min: int, n_max: int, universe: int, threads: int = 0):
    """k sets, sizes log-uniform on [n_min, n_max], distinct uniform values of
    [0, universe).  Returns (elements uint32, offsets int64[k + 1])."""
    offsets = np.empty(k + 1, dtype=np.uint64)
    st = lib.si_gen_loguniform(seed, k, n_min, n_max, universe, offsets.ctypes.data_as(ctypes.c_void_p), None,
                               threads)
    check(st, "si_gen_loguniform")
    elements = np.empty(int(offsets[-1]), dtype=np.uint32)
    st = lib.si_gen_loguniform(seed, k, n_min, n_max, universe, offsets.ctypes.data_as(ctypes.c_void_p),
                               elements.ctypes.data_as(ctypes.c_void_p), threads)
    check(st, "si_gen_loguniform")
    return elements, offsets.astype(np.int64)


def random_pairs(seed: int, k: int, npairs: int) -> np.ndarray:
    """npairs pairs (i, j), i != j, drawn uniformly from [0, k): uint32[npairs, 2]."""
    rng = np.random.default_rng(seed)
    i = rng.integers(0, k, npairs, dtype=np.int64)
    j = (i + rng.integers(1, k, npairs, dtype=np.int64)) % k
    return np.stack([i, j], 1).astype(np.uint32)


def batch_pool(seed: int = 8, k: int = 100000, npairs: int = 1000000):
    """The batched-pairs workload: a pool of 100000 sets, sizes log-uniform on
    [32, 2^18], values of [0, 2^26); 1M pairs drawn uniformly from the pool."""
    el, off = loguniform(seed, k, 32, 1 << 18, 1 << 26)
    return el, off, random_pairs(seed + 1, k, npairs)
