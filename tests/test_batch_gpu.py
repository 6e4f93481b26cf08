"""Batched uneven pairs on the GPU: one persistent launch counts a list of
pairs of a collection; every count equal to the oracle's, for the merge and
search techniques, the per-bucket table from the autotuner, and replays of the
batch captured in a CUDA graph."""
import numpy as np
import pytest

import oracle
from set_intersection_b200 import dataset as fmt

pytestmark = pytest.mark.gpu

TECHS = ["ip", "obs", "auto"]


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
    (1000, 32, 1 << 16, 1 << 26, 30000, 4),
])
def test_random_pools(cuda, tech, k, n_min, n_max, universe, npairs, seed):
    from set_intersection_b200 import generate
    el, off = generate.loguniform(seed, k, n_min, n_max, universe)
    pairs = generate.random_pairs(seed + 1, k, npairs)
    want = oracle.pairs(el, off, k, pairs)
    np.testing.assert_array_equal(count(collection(el, off, universe - 1), pairs, tech), want)


@pytest.mark.parametrize("tech", TECHS)
def test_edge_pairs(cuda, tech):
    """Empty sets, a set with itself, subsets, disjoint value ranges, extreme
    size ratios, the values 0 and 0xffffffff, windows that end on equal values."""
    top = np.uint32(0xffffffff)
    rng = np.random.default_rng(5)
    big = np.sort(rng.choice(1 << 24, size=200000, replace=False)).astype(np.uint32)
    sets = [np.zeros(0, np.uint32), big, big[::3].copy(), big[:17].copy(), (big + 1).astype(np.uint32),
            np.array([0, top], np.uint32), np.concatenate([big[::5], [top]]).astype(np.uint32),
            np.arange(1 << 25, (1 << 25) + 5000, dtype=np.uint32), big[255:257].copy(), big[::256].copy(),
            np.arange(0, 600, dtype=np.uint32), np.arange(256, 1024, dtype=np.uint32)]
    ds = fmt.from_sets(sets)
    k = ds.cardinality
    pairs = np.array([(a, b) for a in range(k) for b in range(k)], np.uint32)
    want = oracle.pairs(ds.elements, ds.offsets, k, pairs)
    np.testing.assert_array_equal(count(collection(ds.elements, ds.offsets, ds.universe), pairs, tech), want)


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
    assert len(table) == 256 and set(table) <= {0, 1}
    np.testing.assert_array_equal(count(col, pairs, "auto", table, ws), want)
    counts = torch.zeros(len(pairs), dtype=torch.int32, device="cuda")
    g = api.BatchGraph(col, dpairs, counts, "auto", table)
    for _ in range(2):
        counts.fill_(-1)
        g.launch()
        g.check()
        np.testing.assert_array_equal(counts.cpu().numpy().view(np.uint32), want)
    g.close()


def test_invalid_pair_index_is_reported(cuda):
    from set_intersection_b200._lib import SiError, Status
    el, off = np.arange(10, dtype=np.uint32), np.array([0, 4, 10], np.int64)
    with pytest.raises(SiError) as e:
        count(collection(el, off, 9), np.array([[0, 1], [1, 2]], np.uint32), "auto")
    assert e.value.status == Status.INVALID_INPUT


def test_batched_pool_sample(cuda):
    """A tenth of the batched workload (10000 sets, sizes log-uniform on
    [32, 2^18] over [0, 2^26), 100000 pairs): merge, search and the tuned
    table agree on every pair, and 20000 sampled pairs equal the oracle's."""
    from set_intersection_b200 import api, generate
    el, off, pairs = generate.batch_pool(k=10000, npairs=100000)
    col = collection(el, off, (1 << 26) - 1)
    ws = api.Workspace()
    merge = count(col, pairs, "ip", ws=ws)
    np.testing.assert_array_equal(count(col, pairs, "obs", ws=ws), merge)
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
