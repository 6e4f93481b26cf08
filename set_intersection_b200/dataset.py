"""The reference's binary dataset format and its text result format.

Binary dataset (include/io.hpp:25-54 readDataset, :70-89 writeDataset), all
little-endian, no padding::

    u32 cardinality (k) | u32 universe | u64 totalElements |
    u32 sizes[k] | u32 elements[totalElements]   (set after set, ascending)

Text result (include/io.hpp:91-136 writeResult): one line ``(a,b): count`` per
pair a < b, 1-based.  For one run (k <= partition) the order is row-major over
the upper triangle; for several runs it follows the tile-pair loop.

Readers here read in bulk (the reference reads element by element) and check
the header against the file size, so a truncated or corrupt file is an error
rather than undefined behaviour.
"""
from __future__ import annotations

import dataclasses
import os
import struct

import numpy as np

from . import tiling

_HEADER = struct.Struct("<IIQ")


class DatasetError(ValueError):
    pass


@dataclasses.dataclass
class Dataset:
    cardinality: int
    universe: int
    sizes: np.ndarray      # uint32[k]
    elements: np.ndarray   # uint32[total]

    @property
    def total_elements(self) -> int:
        return int(self.elements.size)

    @property
    def offsets(self) -> np.ndarray:
        """uint64[k+1] CSR offsets (the reference scans sizes into u32 offsets)."""
        off = np.zeros(self.cardinality + 1, dtype=np.uint64)
        np.cumsum(self.sizes, dtype=np.uint64, out=off[1:])
        return off

    def set(self, i: int) -> np.ndarray:
        off = self.offsets
        return self.elements[int(off[i]):int(off[i + 1])]

    def sets(self) -> list[np.ndarray]:
        off = self.offsets
        return [self.elements[int(off[i]):int(off[i + 1])] for i in range(self.cardinality)]


def from_sets(sets, universe: int | None = None) -> Dataset:
    arrs = [np.ascontiguousarray(s, dtype=np.uint32) for s in sets]
    sizes = np.array([a.size for a in arrs], dtype=np.uint32)
    elements = np.concatenate(arrs) if arrs else np.zeros(0, np.uint32)
    if universe is None:
        universe = int(elements.max()) if elements.size else 0
    return Dataset(len(arrs), int(universe), sizes, elements.astype(np.uint32, copy=False))


def read_dataset(path: str | os.PathLike) -> Dataset:
    """include/io.hpp:25-54, as one bulk read with size checks."""
    with open(path, "rb") as f:
        head = f.read(_HEADER.size)
        if len(head) != _HEADER.size:
            raise DatasetError(f"{path}: truncated header")
        k, universe, total = _HEADER.unpack(head)
        sizes = np.fromfile(f, dtype="<u4", count=k)
        if sizes.size != k:
            raise DatasetError(f"{path}: truncated sizes ({sizes.size} of {k})")
        if int(sizes.sum(dtype=np.uint64)) != total:
            raise DatasetError(f"{path}: sizes sum to {int(sizes.sum(dtype=np.uint64))}, header says {total}")
        elements = np.fromfile(f, dtype="<u4", count=total)
        if elements.size != total:
            raise DatasetError(f"{path}: truncated elements ({elements.size} of {total})")
    return Dataset(k, universe, sizes.astype(np.uint32), elements.astype(np.uint32))


def write_dataset(path: str | os.PathLike, ds: Dataset) -> None:
    """include/io.hpp:70-89."""
    with open(path, "wb") as f:
        f.write(_HEADER.pack(ds.cardinality, ds.universe, ds.total_elements))
        ds.sizes.astype("<u4").tofile(f)
        ds.elements.astype("<u4").tofile(f)


def check_sorted_unique(ds: Dataset) -> list[int]:
    """Indices of sets that are not strictly increasing (the reference assumes
    strictly increasing sets and never checks)."""
    bad = []
    for i, s in enumerate(ds.sets()):
        if s.size > 1 and not np.all(s[1:] > s[:-1]):
            bad.append(i)
    return bad


def format_result_lines(k: int, counts, partition: int | None = None) -> list[str]:
    """Lines of the reference's result file for triangular counts.

    counts: sequence indexed by tiling.triangular_index(k, a, b).
    partition: the executable's --partition; None or >= k gives the single-run
    order of include/io.hpp:91-102, otherwise the tile-pair order of :104-136.
    """
    lines = []
    if partition is None or partition >= k:
        for a in range(k):
            for b in range(a + 1, k):
                lines.append(f"({a + 1},{b + 1}): {int(counts[tiling.triangular_index(k, a, b)])}\n")
        return lines
    for A, B in tiling.find_tile_pairs(k, partition):
        self_join = A.id == B.id
        for i in range(A.start, A.end):
            for j in range(i + 1 if self_join else B.start, B.end):
                lines.append(f"({i + 1},{j + 1}): {int(counts[tiling.triangular_index(k, i, j)])}\n")
    return lines


def write_result(path: str | os.PathLike, k: int, counts, partition: int | None = None) -> None:
    with open(path, "w") as f:
        f.writelines(format_result_lines(k, counts, partition))


def parse_result(path: str | os.PathLike, k: int) -> np.ndarray:
    """Reads a result file back into triangular order (uint64)."""
    out = np.zeros(tiling.combination(k, 2), dtype=np.uint64)
    seen = np.zeros(out.size, dtype=bool)
    with open(path) as f:
        for line in f:
            line = line.strip()
            if not line:
                continue
            pair, val = line.split(":")
            a, b = (int(x) for x in pair.strip("()").split(","))
            idx = tiling.triangular_index(k, a - 1, b - 1)
            out[idx] = int(float(val))
            seen[idx] = True
    if not seen.all():
        raise DatasetError(f"{path}: {int((~seen).sum())} pairs missing")
    return out
