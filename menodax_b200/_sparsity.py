"""Jacobian sparsity: pattern normalisation, column colouring and slot maps.

The Rodas5P kernel fills ``-J`` by forward sweeps, one per colour group: a group
is a set of columns no two of which share a row, so seeding all of them at once
returns every one of their entries in a single sweep (the scheme of
``modax/_sparsity.py:1-20``).  This module works on one boolean *occupancy*
matrix ``M[r, c] = (r, c) is a structural nonzero`` built once per pattern:

* ``normalize_sparsity`` turns a mask, a scipy sparse matrix or ``(nnz, 2)``
  ``(row, col)`` pairs into the hashable tuple-of-row-tuples key the kernel
  caches compile on, with the reference's error messages
  (``modax/_sparsity.py:150-179``);
* ``colour_columns`` colours the column-conflict graph ``M^T M`` with NetworkX's
  greedy colouring, fewest colours over the same five strategies as the
  reference (``modax/_sparsity.py:33-39, 182-210``; same library version);
* a ``SlotMap`` is a precomputed ``(n_vars, n_colours)`` table telling where the
  value sweep ``g`` produces for row ``r`` is stored.  On the *grid* (dense
  storage) the slot is ``r * n_colours + g`` (the reference's layout,
  ``modax/_sparsity.py:42-60``) and every position is written; a sparse LU
  supplies its own CSR slots (``_sparse_direct.csr_slot_map``) and positions no
  entry claims hold ``-1``.
"""

from __future__ import annotations

import functools
from dataclasses import dataclass, field

import numpy as np

# NetworkX greedy strategies tried, in this order; fewest colours wins and a tie
# keeps the earlier strategy's colouring (modax/_sparsity.py:33-39).
STRATEGIES = (
    "largest_first",
    "smallest_last",
    "independent_set",
    "saturation_largest_first",
    "DSATUR",
)


def occupancy(pattern: tuple[tuple[int, ...], ...]) -> np.ndarray:
    """``(n, n)`` boolean matrix of a normalised pattern's structural nonzeros."""
    n = len(pattern)
    mask = np.zeros((n, n), dtype=bool)
    for r, cols in enumerate(pattern):
        mask[r, list(cols)] = True
    return mask


def _entries(sparsity, n_vars: int) -> tuple[np.ndarray, np.ndarray]:
    """Row and column index arrays of the entries, in whatever form they came."""
    if hasattr(sparsity, "tocoo"):
        coo = sparsity.tocoo()
        return np.asarray(coo.row, dtype=np.int64), np.asarray(coo.col, dtype=np.int64)
    arr = np.asarray(sparsity)
    if arr.ndim == 2 and arr.shape == (n_vars, n_vars):
        r, c = np.nonzero(arr)
        return r.astype(np.int64), c.astype(np.int64)
    if arr.ndim == 2 and arr.shape[1] == 2:
        pairs = arr.astype(np.int64)
        return pairs[:, 0], pairs[:, 1]
    raise ValueError(
        "sparsity must be an (n_vars, n_vars) mask, a scipy sparse "
        f"matrix, or an (nnz, 2) array of (row, col); got shape "
        f"{arr.shape} for n_vars={n_vars}"
    )


def normalize_sparsity(sparsity, n_vars: int) -> tuple[tuple[int, ...], ...]:
    """The pattern as one sorted tuple of column indices per row (duplicates merged)."""
    rows, cols = _entries(sparsity, n_vars)
    outside = (rows < 0) | (rows >= n_vars) | (cols < 0) | (cols >= n_vars)
    if outside.any():
        k = int(np.flatnonzero(outside)[0])
        raise ValueError(
            f"sparsity entry ({int(rows[k])}, {int(cols[k])}) lies outside an {n_vars}x{n_vars} Jacobian"
        )
    mask = np.zeros((n_vars, n_vars), dtype=bool)
    mask[rows, cols] = True
    return tuple(tuple(int(c) for c in np.flatnonzero(row)) for row in mask)


@dataclass(frozen=True)
class ColourPartition:
    """Which sweep seeds each column: ``colour[c]`` in ``0 .. n_colours - 1``."""

    colour: tuple[int, ...]

    @property
    def n_vars(self) -> int:
        return len(self.colour)

    @property
    def n_colours(self) -> int:
        return 1 + max(self.colour) if self.colour else 0

    def seed_table(self, min_width: int = 0) -> np.ndarray:
        """``(n_colours + 1, max(n_vars, min_width))``: row ``g`` seeds group ``g``; the
        last row is zero (the direction of a sweep along ``t`` or a parameter)."""
        width = max(self.n_vars, min_width)
        seeds = np.zeros((self.n_colours + 1, width), dtype=np.float64)
        seeds[np.asarray(self.colour, dtype=np.int64), np.arange(self.n_vars)] = 1.0
        return seeds


def assert_orthogonal(pattern, colour) -> None:
    """Raise if some row holds two columns of one colour: their sweep values would
    land in one slot (``modax/_sparsity.py:213-230``)."""
    colour = np.asarray(colour, dtype=np.int64)
    for row, cols in enumerate(pattern):
        groups = colour[list(cols)]
        values, first, counts = np.unique(groups, return_index=True, return_counts=True)
        if (counts > 1).any():
            g = int(values[counts > 1][0])
            clash = [c for c in cols if colour[c] == g]
            raise ValueError(
                f"columns {clash[0]} and {clash[1]} share colour {g} but both have "
                f"an entry in row {row}; the colouring is not structurally "
                "orthogonal for this pattern"
            )


@functools.cache
def colour_columns(pattern: tuple[tuple[int, ...], ...]) -> ColourPartition:
    """Greedy colouring of the column-conflict graph; fewest colours over ``STRATEGIES``."""
    import networkx as nx

    mask = occupancy(pattern).astype(np.int32)
    conflict = (mask.T @ mask) > 0
    np.fill_diagonal(conflict, False)
    graph = nx.from_numpy_array(conflict.astype(np.int8))
    best: dict | None = None
    for strategy in STRATEGIES:
        found = nx.coloring.greedy_color(graph, strategy=strategy)
        if best is None or max(found.values(), default=0) < max(best.values(), default=0):
            best = found
    partition = ColourPartition(tuple(int(best.get(c, 0)) for c in range(len(pattern))))
    assert_orthogonal(pattern, partition.colour)
    return partition


@dataclass(frozen=True, eq=False)
class SlotMap:
    """Storage of one trajectory's ``-J`` (and, for a sparse LU, its fill).

    ``writes[r, g]`` is the slot that receives row ``r`` of sweep ``g`` (``-1``:
    that sweep has no entry in row ``r``); ``diagonal[i]`` is the slot of
    ``(i, i)``, which always exists because ``I / (h gamma)`` lands there;
    ``size`` is the buffer length, fill slots included.  ``contiguous`` marks the
    grid, where ``writes[r, g] == r * n_colours + g`` and every slot is written.
    """

    partition: ColourPartition
    writes: np.ndarray
    diagonal: tuple[int, ...]
    size: int
    contiguous: bool = field(default=False)

    @property
    def n_vars(self) -> int:
        return self.partition.n_vars

    @property
    def n_colours(self) -> int:
        return self.partition.n_colours

    @property
    def colour(self) -> tuple[int, ...]:
        return self.partition.colour

    def slot(self, row: int, col: int) -> int:
        """Slot of entry ``(row, col)``."""
        found = int(self.writes[row, self.colour[col]])
        if found < 0 and row == col:
            return self.diagonal[row]
        if found < 0:
            raise ValueError(
                f"entry ({row}, {col}) is not in the pattern, so a packed "
                "layout has no slot for it; declare it in the sparsity pattern"
            )
        return found

    def store_slots(self) -> np.ndarray | None:
        """Flattened ``writes`` for scattered storage; ``None`` on the grid."""
        return None if self.contiguous else self.writes.reshape(-1).astype(np.int32)

    def seed_table(self, min_width: int = 0) -> np.ndarray:
        return self.partition.seed_table(min_width)


def grid_slots(partition: ColourPartition) -> SlotMap:
    """Row-major ``(n_vars, n_colours)`` storage: sweep ``g`` writes column ``g``."""
    n, nc = partition.n_vars, partition.n_colours
    writes = np.arange(n * nc, dtype=np.int64).reshape(n, nc)
    diagonal = tuple(int(writes[i, partition.colour[i]]) for i in range(n))
    return SlotMap(partition, writes, diagonal, n * nc, contiguous=True)


def dense_jacobian(n_vars: int) -> SlotMap:
    """Every column its own colour: the row-major dense matrix."""
    return grid_slots(ColourPartition(tuple(range(n_vars))))


def colour_sparsity(pattern: tuple[tuple[int, ...], ...]) -> SlotMap:
    """The pattern's colouring on grid storage."""
    return grid_slots(colour_columns(pattern))
