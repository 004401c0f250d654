"""Mini-batch groupings, bit-exact with the reference's seeded scheme.

phaser seeds a PCG64 generator from sha256(json(seed) || json(entropy))
(phaser/utils/misc.py:14-56) and uses it to shuffle the scan index grid
before splitting it into near-equal groups (misc.py:96-115), or to seed
k-means for spatially compact groups (misc.py:118-196).  Groupings are
host-side integer work done once per iteration; the GPU receives the flat
position indices.
"""
from __future__ import annotations

import hashlib
import json
import math
import typing as t

import numpy


def create_rng(seed: t.Any = None, entropy: t.Any = None) -> numpy.random.Generator:
    """PCG64 generator; same seed + entropy -> same stream as phaser/utils/misc.py:36-56."""
    if isinstance(seed, numpy.random.Generator):
        return seed
    if isinstance(seed, numpy.random.BitGenerator):
        return numpy.random.Generator(seed)
    if seed is None:
        return numpy.random.Generator(numpy.random.PCG64(numpy.random.SeedSequence()))
    if isinstance(seed, numpy.random.SeedSequence):
        seed = seed.entropy
    digest = hashlib.sha256()
    digest.update(json.dumps(seed).encode('utf-8'))
    if entropy is not None:
        digest.update(json.dumps(entropy).encode('utf-8'))
    words = numpy.frombuffer(digest.digest(), dtype=numpy.uint32)
    return numpy.random.Generator(numpy.random.PCG64(numpy.random.SeedSequence(words)))


def create_sparse_groupings(shape, max_grouping: int = 8, seed: t.Any = None,
                            i: int = 0) -> t.List[numpy.ndarray]:
    """Random partition of the index grid of `shape` into groups of at most
    `max_grouping` (misc.py:96-115).  Each group is an (ndim, B) int64 array."""
    if isinstance(shape, int):
        shape = (shape,)
    elif not isinstance(shape, (tuple, list)):
        shape = numpy.asarray(shape).shape[:-1]
    grid = numpy.indices(tuple(shape))
    grid = grid.reshape(grid.shape[0], -1).T
    create_rng(seed, f'groupings_{i}' if i != 0 else 'groupings').shuffle(grid)
    n_groups = numpy.ceil(grid.shape[0] / max_grouping).astype(numpy.int64)
    return numpy.array_split(grid.T, n_groups, axis=-1)


def create_compact_groupings(positions: numpy.ndarray, max_grouping: int = 8, seed: t.Any = None,
                             i: int = 0) -> t.List[numpy.ndarray]:
    """Spatially compact groups: k-means++ centroids, then greedy nearest-centroid
    assignment in two phases (groups of size k-1, then k) (misc.py:118-196)."""
    from scipy.spatial import KDTree
    from scipy.cluster.vq import kmeans2

    flat_pos = positions.reshape(-1, 2)
    grid = numpy.indices(positions.shape[:-1])
    grid = grid.reshape(grid.shape[0], -1)
    n = flat_pos.shape[0]
    n_groups = int(numpy.ceil(n / max_grouping))
    if n_groups == 1:
        return [grid]
    size = int(numpy.ceil(n / n_groups))
    rng = create_rng(seed, f'groupings_{i}' if i != 0 else 'groupings')
    centroids, _ = kmeans2(flat_pos, n_groups, minit='++', missing='raise', rng=rng)
    counts = numpy.zeros(n_groups)
    owner = numpy.full(n, -1)
    free = numpy.arange(n)
    tree = KDTree(centroids)
    for cap, target in ((size - 1, (size - 1) * n_groups), (size, n)):
        k = min(4, n_groups)
        while True:
            dist, nbrs = tree.query(flat_pos[free], k)
            order = numpy.argsort(dist[..., 0])
            nbrs = nbrs[order]
            cand = free[order]
            for p, choices in zip(cand, nbrs):
                for g in choices:
                    if counts[g] < cap:
                        owner[p] = g
                        counts[g] += 1
                        break
            free = numpy.where(owner == -1)[0]
            if n - len(free) >= target:
                break
            assert k < n_groups
            k = min(k * 2, n_groups)
    counts = numpy.bincount(owner)
    assert numpy.min(counts) in (size - 1, size) and numpy.max(counts) == size
    return [grid[..., owner == g] for g in range(n_groups)]


def shuffled(vals: t.Sequence, seed: t.Any = None, i: int = 0) -> t.Iterator:
    """Visit `vals` in a seeded random order (misc.py:84-93)."""
    order = numpy.arange(len(vals))
    create_rng(seed, f"shuffle_{i}").shuffle(order)
    for k in order:
        yield vals[int(k)]


def mask_fraction_of_groups(n_groups: int, fraction: float) -> numpy.ndarray:
    """Groups that compute the detector error: every k-th (misc.py:199-208)."""
    need = max(1, math.ceil(n_groups * fraction))
    if need >= n_groups:
        return numpy.ones(n_groups, dtype=numpy.bool_)
    mask = numpy.zeros(n_groups, dtype=numpy.bool_)
    mask[::n_groups // need] = True
    return mask


class GroupManager:
    """Regenerates or reshuffles the mini-batches each iteration
    (phaser/engines/common/simulation.py:22-53)."""

    def __init__(self, scan_shape: t.Tuple[int, ...], grouping: t.Optional[int] = None,
                 compact: bool = False, seed: t.Any = None):
        self.grouping = grouping or 64
        self.compact = compact
        self.seed = seed
        self.scan_shape = tuple(scan_shape)
        self.groups: t.Optional[t.List[numpy.ndarray]] = None
        self.n_groups = int(numpy.ceil(numpy.prod(self.scan_shape) / self.grouping))

    def _make(self, scan_host: t.Optional[numpy.ndarray], i: int) -> t.List[numpy.ndarray]:
        if self.compact:
            if scan_host is None:
                raise ValueError("compact groupings need the scan positions")
            return create_compact_groupings(scan_host, self.grouping, seed=self.seed, i=i)
        return create_sparse_groupings(self.scan_shape, self.grouping, seed=self.seed, i=i)

    def iter(self, scan_host: t.Optional[numpy.ndarray] = None, i: int = 0,
             shuffle_groups: bool = False) -> t.List[numpy.ndarray]:
        if shuffle_groups or self.groups is None:
            self.groups = self._make(scan_host, i)
            return list(self.groups)
        return list(shuffled(self.groups, seed=self.seed, i=i))

    def __len__(self) -> int:
        return self.n_groups

    def flat(self, group: numpy.ndarray) -> numpy.ndarray:
        """(ndim, B) grid indices -> flat position indices (int64)."""
        return numpy.ravel_multi_index(tuple(group), self.scan_shape).astype(numpy.int64)
