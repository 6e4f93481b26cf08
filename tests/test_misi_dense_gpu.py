"""All-pairs counts of dense collections on the GPU: the tensor-core incidence
product (INT8 and FP8-e4m3) and the plain bitmap AND-popcount kernel, every
count equal to the oracle's (zero error)."""
import numpy as np
import pytest

import oracle
from conftest import golden_path
from set_intersection_b200 import dataset as fmt

pytestmark = pytest.mark.gpu

VARIANTS = [("mm", "int8"), ("mm", "fp8"), ("bitmap_naive", "int8")]


def collection(elements, offsets, universe):
    import torch
    from set_intersection_b200 import api
    el = torch.from_numpy(np.ascontiguousarray(elements, dtype=np.uint32).view(np.int32)).cuda()
    off = torch.from_numpy(np.ascontiguousarray(offsets, dtype=np.int64)).cuda()
    return api.Collection(el, off, universe)


def counts(col, tech, dtype, ws=None):
    from set_intersection_b200 import api
    return api.misi_dense(col, tech, dtype, workspace=ws).cpu().numpy().view(np.uint32)


@pytest.mark.parametrize("tech,dtype", VARIANTS)
@pytest.mark.parametrize("name", ["misi_mixed", "misi_onebased"])
def test_golden_datasets(cuda, tech, dtype, name):
    """Counts of every pair equal the reference's result files (std and
    boost bitset executables)."""
    ds = fmt.read_dataset(golden_path(f"{name}.bin"))
    col = collection(ds.elements, ds.offsets, ds.universe)
    got = counts(col, tech, dtype)
    for ref in ("std", "bitset"):
        want = fmt.parse_result(golden_path(f"{name}.{ref}.txt"), ds.cardinality)
        np.testing.assert_array_equal(got, want.astype(np.uint32))


@pytest.mark.parametrize("tech,dtype", VARIANTS)
@pytest.mark.parametrize("k,n_values,p", [
    (2, 100, 0.5), (3, 1, 1.0), (5, 7, 0.5), (127, 129, 0.3), (128, 128, 0.5), (129, 300, 0.2),
    (255, 1000, 0.1), (256, 4096, 0.05), (257, 5000, 0.1), (300, 4097, 0.3), (513, 200, 0.9),
    (1000, 20000, 0.05), (2100, 3000, 0.02),
])
def test_random_bernoulli(cuda, tech, dtype, k, n_values, p):
    from set_intersection_b200 import generate
    el, off = generate.bernoulli(k * 7 + n_values, k, n_values, p)
    want = oracle.all_pairs(el, off, k, n_values - 1, "bitset")
    got = counts(collection(el, off, n_values - 1), tech, dtype)
    np.testing.assert_array_equal(got, want)


@pytest.mark.parametrize("tech,dtype", VARIANTS)
def test_empty_full_and_tiny(cuda, tech, dtype):
    """Empty sets, sets holding the whole universe, one- and zero-pair cases."""
    rng = np.random.default_rng(3)
    U = 777
    sets = [np.arange(U, dtype=np.uint32), np.zeros(0, np.uint32), np.arange(U, dtype=np.uint32),
            np.array([0], np.uint32), np.array([U - 1], np.uint32)]
    sets += [np.sort(rng.choice(U, size=rng.integers(0, U), replace=False)).astype(np.uint32) for _ in range(200)]
    ds = fmt.from_sets(sets, universe=U - 1)
    want = oracle.all_pairs(ds.elements, ds.offsets, ds.cardinality, ds.universe, "std")
    got = counts(collection(ds.elements, ds.offsets, ds.universe), tech, dtype)
    np.testing.assert_array_equal(got, want)
    for k in (0, 1):
        ds = fmt.from_sets(sets[:k], universe=U - 1)
        assert counts(collection(ds.elements, ds.offsets, U - 1), tech, dtype).size == 0


@pytest.mark.parametrize("tech,dtype", VARIANTS)
def test_value_above_universe_is_reported(cuda, tech, dtype):
    from set_intersection_b200._lib import SiError, Status
    el = np.array([1, 5, 9, 2, 40], np.uint32)
    off = np.array([0, 3, 5], np.int64)
    with pytest.raises(SiError) as e:
        counts(collection(el, off, 30), tech, dtype)
    assert e.value.status == Status.INVALID_INPUT


@pytest.mark.parametrize("tech,dtype", VARIANTS)
def test_workspace_reuse(cuda, tech, dtype):
    from set_intersection_b200 import api, generate
    ws = api.Workspace()
    for seed, (k, n, p) in enumerate([(700, 9000, 0.05), (40, 100, 0.5), (1500, 2000, 0.1)]):
        el, off = generate.bernoulli(100 + seed, k, n, p)
        want = oracle.all_pairs(el, off, k, n - 1, "std")
        np.testing.assert_array_equal(counts(collection(el, off, n - 1), tech, dtype, ws), want)


@pytest.mark.slow
def test_dense_config_16384_sets(cuda):
    """The full dense configuration (16384 sets over 65536 values,
    Bernoulli(0.05)): the INT8 and FP8 tensor-core products and the plain
    popcount kernel agree on all 134M counts, and every count equals the
    oracle's (its bitset probe over every pair, the boost_bitset technique,
    OpenMP over all host cores)."""
    import os
    from set_intersection_b200 import generate
    el, off = generate.misi_dense()
    k = off.size - 1
    col = collection(el, off, 65535)
    c_int8 = counts(col, "mm", "int8")
    c_fp8 = counts(col, "mm", "fp8")
    assert np.array_equal(c_int8, c_fp8)
    c_naive = counts(col, "bitmap_naive", "int8")
    assert np.array_equal(c_int8, c_naive)
    want = oracle.all_pairs(el, off, k, 65535, "bitset", threads=os.cpu_count() or 1)
    assert want.size == k * (k - 1) // 2
    np.testing.assert_array_equal(c_int8, want)