"""Single-pair (SISI) parity on the GPU: every count and every materialised
element bit-exact against the oracle / the reference's golden outputs."""
import numpy as np
import pytest

import oracle
from conftest import golden_path, read_golden_elements
from set_intersection_b200 import dataset as fmt

pytestmark = pytest.mark.gpu

TECHS = ["ip", "bitmap", "hi", "obs", "auto"]


def dev(x):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x, dtype=np.uint32).view(np.int32)).cuda()


def run(a, b, tech="ip", materialize=True, ws=None):
    from set_intersection_b200 import api
    c, out = api.intersect(dev(a), dev(b), tech, materialize, workspace=ws)
    return c, (out.cpu().numpy().view(np.uint32) if out is not None else None)


def check(a, b, tech="ip"):
    want = oracle.set_intersection(a, b)
    c, got = run(a, b, tech)
    assert c == want.size
    np.testing.assert_array_equal(got, want)
    c2, _ = run(a, b, tech, materialize=False)
    assert c2 == want.size


@pytest.mark.parametrize("tech", TECHS)
@pytest.mark.parametrize("name", ["sisi_uniform", "sisi_skewed", "sisi_extremes", "misi_mixed", "misi_onebased"])
def test_golden_pairs(cuda, tech, name):
    ds = fmt.read_dataset(golden_path(f"{name}.bin"))
    want = read_golden_elements(f"{name}.elements.bin")
    c, got = run(ds.set(0), ds.set(1), tech)
    assert c == want.size
    np.testing.assert_array_equal(got, want)
    # either argument order gives the same intersection
    c, got = run(ds.set(1), ds.set(0), tech)
    np.testing.assert_array_equal(got, want)


@pytest.mark.parametrize("tech", TECHS)
def test_all_golden_pairs_of_mixed_dataset(cuda, tech):
    """Every pair of the mixed golden dataset (empty, singleton, identical,
    subset, disjoint, ragged sizes) against the reference's result file."""
    ds = fmt.read_dataset(golden_path("misi_mixed.bin"))
    expected = fmt.parse_result(golden_path("misi_mixed.std.txt"), ds.cardinality)
    sets = ds.sets()
    k = ds.cardinality
    from set_intersection_b200 import tiling
    for a in range(0, k, 3):
        for b in range(a + 1, k, 2):
            c, _ = run(sets[a], sets[b], tech, materialize=False)
            assert c == int(expected[tiling.triangular_index(k, a, b)]), (a, b)


def _u(rng, n, hi):
    return np.sort(rng.choice(hi, size=n, replace=False)).astype(np.uint32)


@pytest.mark.parametrize("tech", TECHS)
@pytest.mark.parametrize("na,nb,hi", [
    (0, 0, 10), (0, 100, 1000), (100, 0, 1000), (1, 1, 2), (3, 5, 8),
    (4095, 4097, 1 << 14), (4096, 4096, 8192), (4097, 12289, 1 << 15),
    (10000, 10, 1 << 20), (10, 10000, 1 << 20), (123457, 98765, 1 << 18),
    (1 << 17, 1 << 17, 1 << 18),
])
def test_random_sizes(cuda, tech, na, nb, hi):
    rng = np.random.default_rng(na * 31 + nb)
    check(_u(rng, na, hi), _u(rng, nb, hi), tech)


@pytest.mark.parametrize("tech", TECHS)
def test_identical_disjoint_subset(cuda, tech):
    x = np.arange(0, 300000, 3, dtype=np.uint32)
    check(x, x.copy(), tech)
    check(x, x + 1, tech)
    check(x, x[::7].copy(), tech)
    check(np.arange(0, 50000, dtype=np.uint32), np.arange(50000, 90000, dtype=np.uint32), tech)


@pytest.mark.parametrize("tech", TECHS)
def test_value_extremes(cuda, tech):
    top = np.arange(0xffffffff - 20000, 0xffffffff + 1, dtype=np.uint64).astype(np.uint32)
    check(top, top[::2].copy(), tech)
    check(top[1::2].copy(), top[::2].copy(), tech)
    check(np.array([0, 0xffffffff], np.uint32), np.array([0xffffffff], np.uint32), tech)
    rng = np.random.default_rng(5)
    a = np.concatenate([[0], _u(rng, 50000, 1 << 32 - 1)[1:-1], [0xffffffff]]).astype(np.uint32)
    a = np.unique(a)
    b = np.unique(np.concatenate([[0, 0xffffffff], a[::5]])).astype(np.uint32)
    check(a, b, tech)


@pytest.mark.parametrize("tech", TECHS)
def test_misaligned_device_pointers(cuda, tech):
    """Sets that start at any 4-byte offset (views into larger buffers)."""
    from set_intersection_b200 import api
    rng = np.random.default_rng(8)
    base_a = _u(rng, 40011, 1 << 17)
    base_b = _u(rng, 40007, 1 << 17)
    da, db = dev(base_a), dev(base_b)
    for oa, ob in ((1, 0), (0, 3), (2, 1), (3, 3)):
        want = oracle.set_intersection(base_a[oa:], base_b[ob:])
        c, out = api.intersect(da[oa:], db[ob:], tech)
        assert c == want.size
        np.testing.assert_array_equal(out.cpu().numpy().view(np.uint32), want)


@pytest.mark.parametrize("tech", TECHS)
def test_workspace_reuse_across_sizes(cuda, tech):
    from set_intersection_b200 import api
    ws = api.Workspace()
    rng = np.random.default_rng(12)
    for n in (50000, 7, 200000, 0, 4096):
        a, b = _u(rng, n, 1 << 19), _u(rng, n, 1 << 19)
        want = oracle.set_intersection(a, b)
        c, got = run(a, b, tech, ws=ws)
        assert c == want.size
        np.testing.assert_array_equal(got, want)


@pytest.mark.parametrize("tech", TECHS)
def test_plain_config_seeds_1_2(cuda, tech):
    """|A| = |B| = 2^20 from [0, 2^24), seeds 1 and 2."""
    from set_intersection_b200 import generate
    a, b = generate.sisi_plain()
    check(a, b, tech)


@pytest.mark.parametrize("tech", TECHS)
def test_skewed_config(cuda, tech):
    """|A| = 2^16, |B| = 2^26 from [0, 2^30), 20 % of A planted into B."""
    from set_intersection_b200 import generate
    a, b = generate.sisi_skewed()
    check(a, b, tech)
    check(b, a, tech)


@pytest.mark.parametrize("tech", TECHS)
def test_hash_collisions_and_strides(cuda, tech):
    """Values that share low bits or hash buckets: strided sets whose tiles are
    dense arithmetic progressions."""
    for stride in (1 << 13, 1 << 16, 4097, 3 << 20):
        a = (np.arange(0, 60000, dtype=np.uint64) * stride % (1 << 32)).astype(np.uint32)
        a = np.unique(a)
        b = np.unique(np.concatenate([a[::3], a[1::5] + 1])).astype(np.uint32)
        check(a, b, tech)


@pytest.mark.parametrize("tech", TECHS)
def test_2_24_against_oracle(cuda, tech):
    from set_intersection_b200 import generate
    a = generate.uniform(21, 1 << 24, 1 << 27)
    b = generate.uniform(22, 1 << 24, 1 << 27)
    check(a, b, tech)


@pytest.mark.slow
@pytest.mark.parametrize("tech", TECHS)
def test_full_size_2_28(cuda, tech):
    """|A| = |B| = 2^28 from [0, 2^31): full-size result equals the oracle's,
    element for element."""
    from set_intersection_b200 import generate
    a, b = generate.sisi_large()
    want = oracle.set_intersection(a, b)
    c, got = run(a, b, tech)
    assert c == want.size
    assert np.array_equal(got, want)


@pytest.mark.parametrize("tech", TECHS)
@pytest.mark.parametrize("gap", [1, 2, 8, 15, 16, 17, 30, 31, 33, 64, 1 << 12, 1 << 20])
def test_value_span_per_tile(cuda, tech, gap):
    """Tiles whose value span is below, at and above the bitmap capacity
    (131072 values for the bitmap engine's tiles of about 8192 elements per
    set: gaps near 16): tiles the bitmaps cannot hold take the search path."""
    rng = np.random.default_rng(gap)
    n = 60000
    hi = min(n * gap * 2, 1 << 32)
    a = _u(rng, n, hi)
    b = np.unique(np.concatenate([_u(rng, n, hi), a[::3]])).astype(np.uint32)
    check(a, b, tech)


@pytest.mark.parametrize("tech", TECHS)
def test_density_changes_within_one_pair(cuda, tech):
    """One call mixes tiles that fit the bitmaps with tiles that do not: a dense
    block, a sparse stretch, a second dense block and a sparse tail up to
    2^32 - 1, with overlap in every region."""
    rng = np.random.default_rng(99)
    parts_a, parts_b = [], []
    for lo, hi, n in ((0, 1 << 18, 100000), (1 << 18, 1 << 28, 40000), (1 << 28, (1 << 28) + (1 << 17), 60000),
                      ((1 << 28) + (1 << 17), 1 << 32, 30000)):
        a = lo + _u(rng, n, hi - lo).astype(np.int64)
        b = lo + _u(rng, n, hi - lo).astype(np.int64)
        b = np.union1d(b, a[::5])
        parts_a.append(a)
        parts_b.append(b)
    a = np.unique(np.concatenate(parts_a)).astype(np.uint32)
    b = np.unique(np.concatenate(parts_b)).astype(np.uint32)
    check(a, b, tech)
    check(b[::2].copy(), a, tech)


def test_validate_sorted(cuda):
    from set_intersection_b200 import api
    assert api.validate_sorted(dev(np.arange(100000, dtype=np.uint32)))
    x = np.arange(100000, dtype=np.uint32)
    x[54321] = x[54320]
    assert not api.validate_sorted(dev(x))
    assert api.validate_sorted(dev(np.zeros(1, np.uint32)))


@pytest.mark.parametrize("pinned", [(False, False), (True, False), (False, True)])
def test_intersect_host_staged_pageable_inputs(cuda, pinned):
    """Pageable inputs larger than several 16 MiB staging buffers (ragged
    tails), alone or beside a pinned one, reused on one context."""
    import torch
    from set_intersection_b200 import api, generate
    a = generate.uniform(31, 9_000_001, 1 << 28)
    b = generate.uniform(32, 7_654_321, 1 << 28)
    want = oracle.set_intersection(a, b)
    ha, hb = torch.from_numpy(a.view(np.int32)), torch.from_numpy(b.view(np.int32))
    if pinned[0]:
        ha = ha.pin_memory()
    if pinned[1]:
        hb = hb.pin_memory()
    ctx = api.HostPair()
    for _ in range(2):
        c, got = api.intersect_host(ha, hb, "auto", ctx=ctx)
        assert c == want.size
        assert np.array_equal(got.numpy().view(np.uint32), want)
    ctx.close()


@pytest.mark.parametrize("chunks", [None, 1, 3, 8])
@pytest.mark.parametrize("tech", ["auto", "ip", "bitmap"])
def test_intersect_host_pipeline(cuda, tech, chunks):
    """The host-buffer call (si_sisi_host), cut into value-range chunks that
    are copied, intersected and copied back in a pipeline: the same count and
    elements as the oracle for balanced, skewed, tiny, empty and identical
    pairs, from pinned and from pageable host memory."""
    import torch
    from set_intersection_b200 import api
    rng = np.random.default_rng(5)
    big = _u(rng, 1 << 21, 1 << 26)
    cases = [(big, _u(rng, 1 << 21, 1 << 26)),                     # balanced, >= 2^22 elements: 8 chunks by default
             (_u(rng, 3000, 1 << 26), big),                        # skewed
             (np.array([5, 9], np.uint32), np.array([1, 5, 7, 9, 11], np.uint32)),  # fewer elements than chunks
             (np.zeros(0, np.uint32), big[:100].copy()),           # one empty
             (big[:500000].copy(), big[:500000].copy())]           # identical
    ctx = api.HostPair()
    for n, (a, b) in enumerate(cases):
        want = oracle.set_intersection(a, b)
        ha = torch.from_numpy(a.view(np.int32))
        hb = torch.from_numpy(b.view(np.int32))
        if n % 2 == 0:  # pinned (the copies overlap) and pageable buffers
            ha, hb = ha.pin_memory(), hb.pin_memory()
        c, got = api.intersect_host(ha, hb, tech, ctx=ctx, chunks=chunks)
        assert c == want.size
        assert np.array_equal(got.numpy().view(np.uint32), want)


@pytest.mark.parametrize("n_small", [1, 7, 100, 18944, 18945, 37888, 37889, 75776, 75777, 400000, 700000,
                                     3000000])
def test_obs_lane_groups_and_chunking(cuda, n_small):
    """obs at sizes either side of each change of lanes per element (8, 4, 2,
    1 on 148 SMs) and of mask words per warp, with planted hits, the values 0
    and 2^32 - 1, and larger sets whose sample stride T is 1, a few and large."""
    rng = np.random.default_rng(n_small)
    for n_large in (5000, 8192 * 3 + 5, 1 << 22):
        n_large = max(n_large, n_small)
        big = _u(rng, n_large, 1 << 31)
        big[0], big[-1] = 0, 0xFFFFFFFF
        big = np.unique(big)
        pool = np.unique(np.concatenate([
            rng.choice(big, size=n_small // 3 + 1, replace=False),
            rng.integers(0, 1 << 32, size=n_small + 16, dtype=np.uint64).astype(np.uint32)]))
        pool = pool[(pool != 0) & (pool != 0xFFFFFFFF)]
        # exactly n_small elements: 0, 2^32 - 1 and n_small - 2 of the pool
        small = np.sort(np.concatenate([np.array([0, 0xFFFFFFFF], dtype=np.uint32)[: min(2, n_small)],
                                        rng.choice(pool, size=max(0, n_small - 2), replace=False)]))
        assert small.size == n_small
        check(small, big, "obs")
        check(big, small, "obs")
