"""All-pairs counts (MISI) on the GPU, techniques ip / obs / hi / bitmap: every
count equal to the oracle's, for whole collections (triangular order) and for
the reference's tile pairs (triangular self-join tiles, quadratic cross tiles
with the partition as row stride)."""
import numpy as np
import pytest

import oracle
from conftest import golden_path
from set_intersection_b200 import dataset as fmt
from set_intersection_b200 import tiling

pytestmark = pytest.mark.gpu

TECHS = ["ip", "obs", "hi", "bitmap", "auto"]


def collection(elements, offsets, universe):
    import torch
    from set_intersection_b200 import api
    el = torch.from_numpy(np.ascontiguousarray(elements, dtype=np.uint32).view(np.int32)).cuda()
    off = torch.from_numpy(np.ascontiguousarray(offsets, dtype=np.int64)).cuda()
    return api.Collection(el, off, universe)


def run(col, tech, a_range=None, b_range=None, stride=None, ws=None):
    from set_intersection_b200 import api
    return api.misi(col, tech, a_range, b_range, stride, workspace=ws).cpu().numpy().view(np.uint32)


def from_sets(sets, universe=None):
    ds = fmt.from_sets(sets, universe=universe)
    return ds, collection(ds.elements, ds.offsets, ds.universe)


@pytest.mark.parametrize("tech", TECHS)
@pytest.mark.parametrize("name", ["misi_mixed", "misi_onebased"])
def test_golden_datasets(cuda, tech, name):
    """Every pair of the golden datasets equals the reference's result file."""
    ds = fmt.read_dataset(golden_path(f"{name}.bin"))
    got = run(collection(ds.elements, ds.offsets, ds.universe), tech)
    want = fmt.parse_result(golden_path(f"{name}.std.txt"), ds.cardinality)
    np.testing.assert_array_equal(got, want.astype(np.uint32))


@pytest.mark.parametrize("tech", TECHS)
@pytest.mark.parametrize("k,n_max,universe,seed", [
    (2, 100, 1000, 1), (3, 5000, 1 << 16, 2), (40, 3000, 1 << 14, 3), (300, 5000, 1 << 16, 4),
    (257, 40000, 1 << 20, 5), (1000, 2000, 1 << 12, 6),
])
def test_random_powerlaw(cuda, tech, k, n_max, universe, seed):
    from set_intersection_b200 import generate
    el, off = generate.powerlaw(seed, k, 1, n_max, 1.1, universe, 0.8)
    want = oracle.all_pairs(el, off, k, universe, "std")
    np.testing.assert_array_equal(run(collection(el, off, universe), tech), want)


@pytest.mark.parametrize("tech", TECHS)
def test_large_sets_processed_in_chunks(cuda, tech):
    """Sets larger than one shared-memory structure (> 16384 elements, value
    span > 2^20) against each other and against small sets; partners split
    between work items and warp slices."""
    rng = np.random.default_rng(11)
    sets = [np.sort(rng.choice(1 << 26, size=n, replace=False)).astype(np.uint32)
            for n in (100000, 60000, 40000, 20000, 9000, 8193, 8192, 5000, 100, 1)]
    shared = np.sort(rng.choice(1 << 26, size=30000, replace=False)).astype(np.uint32)
    sets += [np.union1d(s, shared).astype(np.uint32) for s in sets[:4]]
    sets.append(np.arange(0, 1 << 26, 7, dtype=np.uint32)[:200000])
    ds, col = from_sets(sets)
    want = oracle.all_pairs(ds.elements, ds.offsets, ds.cardinality, ds.universe, "std")
    np.testing.assert_array_equal(run(col, tech), want)


@pytest.mark.parametrize("tech", TECHS)
def test_edge_sets(cuda, tech):
    """Empty sets, identical sets, subsets, the values 0 and 0xffffffff."""
    top = np.uint32(0xffffffff)
    base = np.arange(0, 3000, 3, dtype=np.uint32)
    sets = [np.zeros(0, np.uint32), base, base.copy(), base[::2].copy(), np.zeros(0, np.uint32),
            np.array([0, top], np.uint32), np.array([top], np.uint32), np.array([0], np.uint32),
            np.concatenate([base, [top]]).astype(np.uint32), np.arange(1, 3000, 3, dtype=np.uint32)]
    ds, col = from_sets(sets)
    want = oracle.all_pairs(ds.elements, ds.offsets, ds.cardinality, ds.universe, "std")
    np.testing.assert_array_equal(run(col, tech), want)
    for k in (0, 1):
        ds, col = from_sets(sets[:k], universe=10)
        assert run(col, tech).size == 0


@pytest.mark.parametrize("tech", TECHS)
@pytest.mark.parametrize("partition", [7, 64, 230])
def test_tile_pairs_match_reference_layout(cuda, tech, partition):
    """The reference's runs (include/util.hpp:40-52): each tile pair's counts,
    triangular (self) or quadratic (cross) with row stride = partition."""
    from set_intersection_b200 import api, generate
    k = 230
    el, off = generate.powerlaw(21, k, 1, 4000, 1.1, 1 << 15, 0.8)
    full = oracle.all_pairs(el, off, k, 1 << 15, "std")
    col = collection(el, off, 1 << 15)
    ws = api.Workspace()
    for A, B in tiling.find_tile_pairs(k, partition):
        got = run(col, tech, (A.start, A.end), (B.start, B.end), partition, ws)
        self_join = A.id == B.id
        for a in range(A.start, A.end):
            bs = range(a + 1, B.end) if self_join else range(B.start, B.end)
            for b in bs:
                idx = (tiling.triangular_index(partition, a - A.start, b - A.start) if self_join
                       else tiling.quadratic_index(partition, a - A.start, b - B.start))
                assert got[idx] == full[tiling.triangular_index(k, a, b)], (A, B, a, b)


@pytest.mark.parametrize("tech", TECHS)
def test_cross_tile_with_uneven_ranges(cuda, tech):
    from set_intersection_b200 import generate
    k = 500
    el, off = generate.powerlaw(31, k, 1, 20000, 1.1, 1 << 18, 0.8)
    full = oracle.all_pairs(el, off, k, 1 << 18, "std")
    col = collection(el, off, 1 << 18)
    for (a0, a1), (b0, b1), stride in [((0, 123), (300, 500), 200), ((450, 500), (0, 77), 77),
                                        ((10, 11), (11, 500), 489)]:
        got = run(col, tech, (a0, a1), (b0, b1), stride)
        for a in range(a0, a1):
            for b in range(b0, b1):
                want = full[tiling.triangular_index(k, min(a, b), max(a, b))]
                assert got[(a - a0) * stride + (b - b0)] == want


@pytest.mark.slow
def test_powerlaw_config_8192_sets(cuda):
    """The full power-law configuration (8192 sets, sizes ~ n^-1.1 on [16, 65536],
    Zipf(0.8) values over [1, 2^20]): the four techniques agree on all 33.5M
    counts, and every count equals the oracle's (its std::set_intersection
    over every pair, OpenMP over all host cores)."""
    import os
    from set_intersection_b200 import api, generate
    el, off = generate.misi_powerlaw()
    k = off.size - 1
    col = collection(el, off, 1 << 20)
    ws = api.Workspace()
    ref = run(col, "bitmap", ws=ws)
    for tech in ("hi", "obs", "ip"):
        assert np.array_equal(run(col, tech, ws=ws), ref), tech
    want = oracle.all_pairs(el, off, k, 1 << 20, "std", threads=os.cpu_count() or 1)
    assert want.size == k * (k - 1) // 2
    np.testing.assert_array_equal(ref, want)