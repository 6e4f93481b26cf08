"""Pins the CPU oracle (oracle/si_oracle.c) against the golden outputs that the
reference's own CPU executables wrote (tests/golden/make_golden.py)."""
import os

import numpy as np
import pytest

import oracle
from conftest import golden_path, read_golden_elements
from set_intersection_b200 import dataset as fmt

DATASETS = ["sisi_uniform", "sisi_skewed", "sisi_extremes", "misi_mixed", "misi_onebased"]


@pytest.mark.parametrize("name", DATASETS)
@pytest.mark.parametrize("tech", ["std", "serial", "bitset"])
def test_all_pairs_matches_reference_output(name, tech):
    ds = fmt.read_dataset(golden_path(f"{name}.bin"))
    ref_file = golden_path(f"{name}.{tech}.txt")
    if not os.path.exists(ref_file):
        pytest.skip("reference executable not applicable to this universe")
    expected = fmt.parse_result(ref_file, ds.cardinality)
    got = oracle.all_pairs(ds.elements, ds.offsets, ds.cardinality, ds.universe, tech, threads=3)
    np.testing.assert_array_equal(got.astype(np.uint64), expected)


@pytest.mark.parametrize("name", DATASETS)
def test_elements_match_reference(name):
    ds = fmt.read_dataset(golden_path(f"{name}.bin"))
    expected = read_golden_elements(f"{name}.elements.bin")
    got = oracle.set_intersection(ds.set(0), ds.set(1))
    np.testing.assert_array_equal(got, expected)


@pytest.mark.parametrize("name", DATASETS)
def test_result_text_is_byte_identical(name):
    """The engine's result writer, fed the oracle's counts, reproduces the
    reference's result file byte for byte."""
    ds = fmt.read_dataset(golden_path(f"{name}.bin"))
    counts = oracle.all_pairs(ds.elements, ds.offsets, ds.cardinality, ds.universe, "std")
    text = "".join(fmt.format_result_lines(ds.cardinality, counts))
    assert text == open(golden_path(f"{name}.std.txt")).read()


def test_threads_do_not_change_counts():
    ds = fmt.read_dataset(golden_path("misi_mixed.bin"))
    one = oracle.all_pairs(ds.elements, ds.offsets, ds.cardinality, ds.universe, "std", threads=1)
    many = oracle.all_pairs(ds.elements, ds.offsets, ds.cardinality, ds.universe, "std", threads=7)
    np.testing.assert_array_equal(one, many)


def test_pairs_matches_all_pairs():
    ds = fmt.read_dataset(golden_path("misi_onebased.bin"))
    k = ds.cardinality
    tri = oracle.all_pairs(ds.elements, ds.offsets, k, ds.universe, "std")
    rng = np.random.default_rng(3)
    a = rng.integers(0, k, 200)
    b = rng.integers(0, k, 200)
    keep = a < b
    pl = np.stack([a[keep], b[keep]], 1)
    got = oracle.pairs(ds.elements, ds.offsets, k, pl)
    want = np.array([tri[oracle.lib().si_oracle_triangular_index(k, int(x), int(y))] for x, y in pl])
    np.testing.assert_array_equal(got, want)


@pytest.mark.parametrize("a,b,want", [
    ([], [], []),
    ([1, 2, 3], [], []),
    ([], [4], []),
    ([0], [0], [0]),
    ([0xffffffff], [0xffffffff], [0xffffffff]),
    ([1, 3, 5], [2, 4, 6], []),
    ([1, 2, 3], [1, 2, 3], [1, 2, 3]),
])
def test_known_answers(a, b, want):
    np.testing.assert_array_equal(oracle.set_intersection(a, b), np.array(want, np.uint32))
    assert oracle.count(a, b, "serial") == len(want)


def test_planted_mistake_is_caught():
    """A planted off-by-one in the oracle's output must be caught by the golden
    comparison (the check is not vacuous)."""
    ds = fmt.read_dataset(golden_path("misi_mixed.bin"))
    expected = fmt.parse_result(golden_path("misi_mixed.std.txt"), ds.cardinality)
    got = oracle.all_pairs(ds.elements, ds.offsets, ds.cardinality, ds.universe, "std").astype(np.uint64)
    got[17] += 1
    assert not np.array_equal(got, expected)


@pytest.mark.parametrize("seed,n,hi,lo", [
    (3, 1 << 16, 1 << 19, 0),          # dense branch (n > U/64)
    (4, 5000, 1 << 14, 100),           # dense, offset range
    (1, 1 << 12, 1 << 24, 0),          # sparse branch
    (7, 1000, (1 << 32), (1 << 32) - (1 << 20)),  # sparse, top of the u32 range
    (9, 0, 10, 0),
])
def test_gen_uniform_equals_engine_generator(seed, n, hi, lo):
    """The oracle's restated generator yields exactly the engine's sets, so the
    reference's executables can be run on the engine's inputs without loading
    the engine's library."""
    from set_intersection_b200 import generate
    want = generate.uniform(seed, n, hi, lo)
    got = oracle.gen_uniform(seed, n, hi, lo)
    np.testing.assert_array_equal(got, want)


def test_write_dataset_matches_format_module(tmp_path):
    sets = [np.array([1, 5, 9], dtype=np.uint32), np.array([], dtype=np.uint32), np.array([0, 2], dtype=np.uint32)]
    p1, p2 = tmp_path / "a.bin", tmp_path / "b.bin"
    oracle.write_dataset(str(p1), sets, 9)
    fmt.write_dataset(str(p2), fmt.from_sets(sets, universe=9))
    assert p1.read_bytes() == p2.read_bytes()
