"""Dataset format, result writer and tiling against the reference's files."""
import os

import numpy as np
import pytest

from conftest import golden_path
from set_intersection_b200 import dataset as fmt
from set_intersection_b200 import tiling


def test_roundtrip_is_byte_identical(tmp_path):
    for name in ("misi_mixed", "sisi_extremes", "misi_onebased"):
        ds = fmt.read_dataset(golden_path(f"{name}.bin"))
        out = tmp_path / f"{name}.bin"
        fmt.write_dataset(out, ds)
        assert out.read_bytes() == open(golden_path(f"{name}.bin"), "rb").read()


def test_reads_reference_txt2bin_output():
    """txt2bin (src/txt2bin.cpp) keeps input order in _asc and sorts by size
    descending in _desc; universe is the max last element."""
    lines = [l.split() for l in open(golden_path("text_sets.txt")) if l.strip()]
    sets = [np.array([int(x) for x in l], np.uint32) for l in lines]
    asc = fmt.read_dataset(golden_path("text_sets_asc.bin"))
    desc = fmt.read_dataset(golden_path("text_sets_desc.bin"))
    assert asc.universe == max(int(s[-1]) for s in sets)
    for got, want in zip(asc.sets(), sets):
        np.testing.assert_array_equal(got, want)
    assert list(desc.sizes) == sorted([s.size for s in sets], reverse=True)


def test_truncated_file_is_an_error(tmp_path):
    raw = open(golden_path("misi_mixed.bin"), "rb").read()
    p = tmp_path / "t.bin"
    p.write_bytes(raw[:-4])
    with pytest.raises(fmt.DatasetError):
        fmt.read_dataset(p)
    p.write_bytes(raw[:10])
    with pytest.raises(fmt.DatasetError):
        fmt.read_dataset(p)


def test_inconsistent_header_is_an_error(tmp_path):
    ds = fmt.read_dataset(golden_path("misi_onebased.bin"))
    bad = fmt.Dataset(ds.cardinality, ds.universe, ds.sizes.copy(), ds.elements)
    bad.sizes[0] += 1
    p = tmp_path / "b.bin"
    fmt.write_dataset(p, bad)
    with pytest.raises(fmt.DatasetError):
        fmt.read_dataset(p)


def test_check_sorted_unique():
    ds = fmt.from_sets([[1, 2, 3], [3, 2], [5, 5], []])
    assert fmt.check_sorted_unique(ds) == [1, 2]


@pytest.mark.parametrize("k,p", [(10, 3), (7, 7), (7, 100), (1, 1), (12, 4)])
def test_tiles_cover_every_pair_once(k, p):
    seen = []
    for A, B in tiling.find_tile_pairs(k, p):
        for i in range(A.start, A.end):
            for j in range(i + 1 if A.id == B.id else B.start, B.end):
                seen.append((i, j))
    assert sorted(seen) == [(i, j) for i in range(k) for j in range(i + 1, k)]
    assert len(set(seen)) == len(seen)


def test_indices_match_reference_definitions():
    n = 9
    idx = [tiling.triangular_index(n, i, j) for i in range(n) for j in range(i + 1, n)]
    assert idx == list(range(tiling.combination(n, 2)))
    assert tiling.quadratic_index(5, 2, 3) == 13


def test_multi_run_line_order(tmp_path):
    """--partition smaller than k writes pairs in tile-pair order
    (include/io.hpp:104-136) with the same counts."""
    k = 5
    counts = np.arange(tiling.combination(k, 2))
    lines = fmt.format_result_lines(k, counts, partition=2)
    assert lines[:2] == ["(1,2): 0\n", "(1,3): 1\n"]
    assert sorted(lines) == sorted(fmt.format_result_lines(k, counts))
    assert lines != fmt.format_result_lines(k, counts)
