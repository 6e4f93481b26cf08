"""All-pairs work decomposition of include/util.hpp, same names and meaning.

tile / splitToTiles / findTilePairs (include/util.hpp:11-52): sets are cut into
tiles of `partition` consecutive sets and every tile pair (i <= j) is one GPU
invocation of the reference; combination / triangular_index / quadratic_index
(:54-74) index the pair counts.
"""
from __future__ import annotations

import dataclasses
import math


@dataclasses.dataclass(frozen=True)
class Tile:
    id: int
    start: int
    end: int

    @property
    def length(self) -> int:
        return self.end - self.start


def split_to_tiles(cardinality: int, partition: int) -> list[Tile]:
    """include/util.hpp:24-38."""
    if partition <= 0:
        raise ValueError("partition must be positive")
    n = math.ceil(cardinality / partition)
    return [Tile(i, i * partition, min(i * partition + partition, cardinality)) for i in range(n)]


def find_tile_pairs(cardinality: int, partition: int) -> list[tuple[Tile, Tile]]:
    """include/util.hpp:40-52: upper-triangular tile pairs, diagonal included."""
    tiles = split_to_tiles(cardinality, partition)
    return [(tiles[i], tiles[j]) for i in range(len(tiles)) for j in range(i, len(tiles))]


def combination(n: int, k: int) -> int:
    """include/util.hpp:54-66."""
    return math.comb(n, k) if 0 <= k <= n else 0


def triangular_index(n: int, i: int, j: int) -> int:
    """include/util.hpp:68-70: offset of pair i < j in the row-major upper triangle."""
    return (n * (n - 1) // 2) - (n - i) * ((n - i) - 1) // 2 + j - i - 1


def quadratic_index(n: int, i: int, j: int) -> int:
    """include/util.hpp:72-74."""
    return i * n + j
