"""Batched uneven pairs on the GPU: one persistent launch counts a list of
pairs of a collection; every count equal to the oracle's, for each of the six
technique codes (merge, search, hash with windows of 1024 and 512 elements,
window bitmaps of 16384 and 32768 values), the per-bucket table from the
autotuner, and replays of the batch captured in a CUDA graph."""
import numpy as np
import pytest

import oracle
from set_intersection_b200 import dataset as fmt

pytestmark = pytest.mark.gpu

TECHS = ["ip", "obs", "hi", "bitmap", "auto"]
CODES = range(6)


def dev(x, dtype=None):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x)).cuda()


def collection(elements, offsets, universe):
    from set_intersection_b200 import api
    return api.Collection(dev(np.ascontiguousarray(elements, np.uint32).view(np.int32)),
                          dev(np.asarray(offsets, np.int64)), universe)


def count(col, pairs, tech, table=None, ws=None):
    from set_intersection_b200 import api
    return api.batch_count(col, dev(pairs.astype(np.uint32).view(np.int32)), tech, table,
                           workspace=ws).cpu().numpy().view(np.uint32)


@pytest.mark.parametrize("tech", TECHS)
@pytest.mark.parametrize("k,n_min,n_max,universe,npairs,seed", [
    (2, 1, 10, 100, 5, 1), (50, 1, 3000, 1 << 14, 2000, 2), (300, 32, 20000, 1 << 20, 20000, 3),
    (1000, 32, 1 << 16, 1 << 26, 30000, 4), (200, 256, 1 << 15, 1 << 16, 10000, 11),
])
def test_random_pools(cuda, tech, k, n_min, n_max, universe, npairs, seed):
    from set_intersection_b200 import generate
    el, off = generate.loguniform(seed, k, n_min, n_max, universe)
    pairs = generate.random_pairs(seed + 1, k, npairs)
    want = oracle.pairs(el, off, k, pairs)
    np.testing.assert_array_equal(count(collection(el, off, universe - 1), pairs, tech), want)


@pytest.mark.parametrize("tech", TECHS + [f"code{c}" for c in CODES])
def test_edge_pairs(cuda, tech):
    """Empty sets, a set with itself, subsets, disjoint value ranges, extreme
    size ratios, the values 0 and 0xffffffff, windows that end on equal values;
    the five techniques by name, and each of the six codes through a table."""
    top = np.uint32(0xffffffff)
    rng = np.random.default_rng(5)
    big = np.sort(rng.choice(1 << 24, size=200000, replace=False)).astype(np.uint32)
    sets = [np.zeros(0, np.uint32), big, big[::3].copy(), big[:17].copy(), (big + 1).astype(np.uint32),
            np.array([0, top], np.uint32), np.concatenate([big[::5], [top]]).astype(np.uint32),
            np.arange(1 << 25, (1 << 25) + 5000, dtype=np.uint32), big[255:257].copy(), big[::256].copy(),
            np.arange(0, 600, dtype=np.uint32), np.arange(256, 1024, dtype=np.uint32),
            np.array([top], np.uint32), np.array([top - 1, top], np.uint32),
            np.arange((1 << 32) - 40000, 1 << 32, dtype=np.uint64).astype(np.uint32),
            np.arange((1 << 32) - 40000, 1 << 32, 3, dtype=np.uint64).astype(np.uint32),
            np.sort(rng.choice(1 << 16, size=30000, replace=False)).astype(np.uint32),
            np.sort(rng.choice(1 << 16, size=3000, replace=False)).astype(np.uint32)]
    ds = fmt.from_sets(sets)
    k = ds.cardinality
    pairs = np.array([(a, b) for a in range(k) for b in range(k)], np.uint32)
    want = oracle.pairs(ds.elements, ds.offsets, k, pairs)
    table = bytes([int(tech[4:])]) * 1024 if tech.startswith("code") else None
    got = count(collection(ds.elements, ds.offsets, ds.universe), pairs, "auto" if table else tech, table)
    np.testing.assert_array_equal(got, want)


def mixed_pool(seed):
    """Sparse sets over [0, 2^26) and dense ones over [0, 2^16) in one
    collection, so that every density class has pairs."""
    from set_intersection_b200 import generate
    el1, off1 = generate.loguniform(seed, 600, 32, 1 << 16, 1 << 26)
    el2, off2 = generate.loguniform(seed + 1, 400, 64, 1 << 15, 1 << 16)
    el = np.concatenate([el1, el2])
    off = np.concatenate([off1, off2[1:] + off1[-1]])
    return el, off, off.size - 1


@pytest.mark.parametrize("code", CODES)
def test_every_code_on_mixed_pool(cuda, code):
    """A table holding one code for every bucket runs that technique on every
    pair (through the queue keys)."""
    from set_intersection_b200 import generate
    el, off, k = mixed_pool(12)
    pairs = generate.random_pairs(13, k, 20000)
    want = oracle.pairs(el, off, k, pairs)
    np.testing.assert_array_equal(count(collection(el, off, (1 << 26) - 1), pairs, "auto", bytes([code]) * 1024),
                                  want)


def test_codes_past_the_last_count_as_merge(cuda):
    from set_intersection_b200 import generate
    el, off, k = mixed_pool(14)
    pairs = generate.random_pairs(15, k, 3000)
    np.testing.assert_array_equal(count(collection(el, off, (1 << 26) - 1), pairs, "auto", bytes([200]) * 1024),
                                  oracle.pairs(el, off, k, pairs))


def test_autotuned_table_and_graph_replays(cuda):
    import torch
    from set_intersection_b200 import api, generate
    k = 2000
    el, off = generate.loguniform(9, k, 32, 1 << 17, 1 << 26)
    pairs = generate.random_pairs(10, k, 50000)
    want = oracle.pairs(el, off, k, pairs)
    col = collection(el, off, (1 << 26) - 1)
    dpairs = dev(pairs.view(np.int32))
    ws = api.Workspace()
    table = api.batch_tune(col, dpairs, sample=512, workspace=ws)
    assert len(table) == api.BATCH_TABLE_SIZE and set(table) <= set(range(api.BATCH_CODES))
    np.testing.assert_array_equal(count(col, pairs, "auto", table, ws), want)
    counts = torch.zeros(len(pairs), dtype=torch.int32, device="cuda")
    g = api.BatchGraph(col, dpairs, counts, "auto", table)
    for _ in range(2):
        counts.fill_(-1)
        g.launch()
        g.check()
        np.testing.assert_array_equal(counts.cpu().numpy().view(np.uint32), want)
    g.close()


def test_tuner_uses_more_than_merge_and_search(cuda):
    """On a pool with dense and sparse sets the tuned table picks techniques
    other than merge and search for some of the populated buckets, and its
    counts equal the oracle's."""
    from set_intersection_b200 import api, generate
    el, off, k = mixed_pool(16)
    pairs = generate.random_pairs(17, k, 60000)
    col = collection(el, off, (1 << 26) - 1)
    ws = api.Workspace()
    dpairs = dev(pairs.view(np.int32))
    table = api.batch_tune(col, dpairs, sample=1024, workspace=ws)
    sizes = np.diff(off)
    buckets = {api.batch_bucket(int(sizes[a]), int(sizes[b]),
                                int(el[off[a if sizes[a] >= sizes[b] else b]]),
                                int(el[off[(a if sizes[a] >= sizes[b] else b) + 1] - 1])) for a, b in pairs}
    used = {table[b] for b in buckets}
    assert used - {api.BATCH_MERGE, api.BATCH_SEARCH}, used
    np.testing.assert_array_equal(count(col, pairs, "auto", table, ws), oracle.pairs(el, off, k, pairs))


def test_invalid_pair_index_is_reported(cuda):
    from set_intersection_b200._lib import SiError, Status
    el, off = np.arange(10, dtype=np.uint32), np.array([0, 4, 10], np.int64)
    with pytest.raises(SiError) as e:
        count(collection(el, off, 9), np.array([[0, 1], [1, 2]], np.uint32), "auto")
    assert e.value.status == Status.INVALID_INPUT


def test_batched_pool_sample(cuda):
    """A tenth of the batched workload (10000 sets, sizes log-uniform on
    [32, 2^18] over [0, 2^26), 100000 pairs): merge, search, hash, bitmap and
    the tuned table agree on every pair, and 20000 sampled pairs equal the
    oracle's."""
    from set_intersection_b200 import api, generate
    el, off, pairs = generate.batch_pool(k=10000, npairs=100000)
    col = collection(el, off, (1 << 26) - 1)
    ws = api.Workspace()
    merge = count(col, pairs, "ip", ws=ws)
    for tech in ("obs", "hi", "bitmap"):
        np.testing.assert_array_equal(count(col, pairs, tech, ws=ws), merge)
    table = api.batch_tune(col, dev(pairs.view(np.int32)), workspace=ws)
    np.testing.assert_array_equal(count(col, pairs, "auto", table, ws), merge)
    idx = np.random.default_rng(2).choice(len(pairs), 20000, replace=False)
    np.testing.assert_array_equal(merge[idx], oracle.pairs(el, off, off.size - 1, pairs[idx]))


@pytest.mark.slow
def test_batched_config_full_pool(cuda):
    """The full batched configuration (100000 sets, sizes log-uniform on
    [32, 2^18] over [0, 2^26), 1M pairs): the tuned batch replayed from its
    CUDA graph gives every one of the 1M counts the oracle gives."""
    import os
    import torch
    from set_intersection_b200 import api, generate
    el, off, pairs = generate.batch_pool()
    col = collection(el, off, (1 << 26) - 1)
    ws = api.Workspace()
    dpairs = dev(pairs.astype(np.uint32).view(np.int32))
    table = api.batch_tune(col, dpairs, workspace=ws)
    counts = torch.empty(len(pairs), dtype=torch.int32, device=cuda)
    graph = api.BatchGraph(col, dpairs, counts, "auto", table)
    try:
        graph.launch()
        graph.check()
        got = counts.cpu().numpy().view(np.uint32)
    finally:
        graph.close()
    want = oracle.pairs(el, off, off.size - 1, pairs, threads=os.cpu_count() or 1)
    np.testing.assert_array_equal(got, want)
