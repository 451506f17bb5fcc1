"""Jacobian sparsity patterns: normalisation, column colouring and slot layouts.

Follows ``modax/_sparsity.py``: a pattern is normalised to a hashable tuple of
row tuples (``normalize_sparsity``, ``modax/_sparsity.py:150-179``), its column
intersection graph is greedily coloured with NetworkX taking the fewest colours
over five strategies (``colour_sparsity``, ``modax/_sparsity.py:182-210``), and
``CompressedJacobian`` maps entry ``(r, c)`` to slot ``r * n_colours +
colour[c]`` on the colour grid, or to a CSR slot of the sparse factorisation when
``packed`` is set (``modax/_sparsity.py:42-140``).  The Jacobian sweep seeded
with colour group ``g`` deposits every entry of that group in one pass.
"""

from __future__ import annotations

import functools
from dataclasses import dataclass

import numpy as np

# The NetworkX strategies tried; the colouring with the fewest colours wins,
# ties going to the earlier strategy (modax/_sparsity.py:33-39, 198-202).
STRATEGIES = (
    "largest_first",
    "smallest_last",
    "independent_set",
    "saturation_largest_first",
    "DSATUR",
)


@dataclass(frozen=True)
class CompressedJacobian:
    """Column-compressed Jacobian layout (``modax/_sparsity.py:42-140``)."""

    n_vars: int
    n_colours: int
    colour: tuple[int, ...]
    packed: tuple[int, ...] | None = None
    packed_diagonal: tuple[int, ...] | None = None
    n_slots: int | None = None

    @property
    def size(self) -> int:
        if self.n_slots is not None:
            return self.n_slots
        if self.packed is not None:
            return 1 + max(max(self.packed), max(self.packed_diagonal))
        return self.n_vars * self.n_colours

    @property
    def diagonal(self) -> tuple[int, ...]:
        return tuple(self.slot(i, i) for i in range(self.n_vars))

    def slot(self, row: int, col: int) -> int:
        grid = row * self.n_colours + self.colour[col]
        if self.packed is None:
            return grid
        slot = self.packed[grid]
        if slot < 0 and row == col:
            return self.packed_diagonal[row]
        if slot < 0:
            raise ValueError(
                f"entry ({row}, {col}) is not in the pattern, so a packed "
                "layout has no slot for it; declare it in the sparsity pattern"
            )
        return slot

    def store_slots(self) -> np.ndarray | None:
        """Slot of each ``(row, colour)`` sweep value, ``-1`` for none; ``None`` on the grid."""
        if self.packed is None:
            return None
        return np.asarray(self.packed, dtype=np.int32)

    def seed_table(self, min_width: int = 0) -> np.ndarray:
        """``(n_colours + 1, max(n_vars, min_width))`` colour indicators plus a zero row."""
        width = max(self.n_vars, min_width)
        seeds = np.zeros((self.n_colours + 1, width), dtype=np.float64)
        for c, g in enumerate(self.colour):
            seeds[g, c] = 1.0
        return seeds


def dense_jacobian(n_vars: int) -> CompressedJacobian:
    """Every column its own colour: the row-major dense matrix."""
    return CompressedJacobian(n_vars=n_vars, n_colours=n_vars, colour=tuple(range(n_vars)))


def normalize_sparsity(sparsity, n_vars: int) -> tuple[tuple[int, ...], ...]:
    """Accept a dense mask, a scipy sparse matrix, or ``(nnz, 2)`` ``(row, col)`` pairs."""
    if hasattr(sparsity, "tocoo"):
        coo = sparsity.tocoo()
        pairs = zip(coo.row.tolist(), coo.col.tolist())
    else:
        arr = np.asarray(sparsity)
        if arr.ndim == 2 and arr.shape == (n_vars, n_vars):
            rows, cols = np.nonzero(arr)
            pairs = zip(rows.tolist(), cols.tolist())
        elif arr.ndim == 2 and arr.shape[1] == 2:
            pairs = ((int(r), int(c)) for r, c in arr.tolist())
        else:
            raise ValueError(
                "sparsity must be an (n_vars, n_vars) mask, a scipy sparse "
                f"matrix, or an (nnz, 2) array of (row, col); got shape "
                f"{arr.shape} for n_vars={n_vars}"
            )
    by_row: list[set[int]] = [set() for _ in range(n_vars)]
    for r, c in pairs:
        if not (0 <= r < n_vars and 0 <= c < n_vars):
            raise ValueError(
                f"sparsity entry ({r}, {c}) lies outside an {n_vars}x{n_vars} Jacobian"
            )
        by_row[r].add(c)
    return tuple(tuple(sorted(cs)) for cs in by_row)


@functools.cache
def colour_sparsity(pattern: tuple[tuple[int, ...], ...]) -> CompressedJacobian:
    """Colour the column intersection graph; fewest colours over the strategies wins."""
    import networkx as nx

    n_vars = len(pattern)
    graph = nx.Graph()
    graph.add_nodes_from(range(n_vars))
    for cols in pattern:
        for a in range(len(cols)):
            for b in range(a + 1, len(cols)):
                graph.add_edge(cols[a], cols[b])
    best = None
    for strategy in STRATEGIES:
        colouring = nx.coloring.greedy_color(graph, strategy=strategy)
        if best is None or max(colouring.values()) < max(best.values()):
            best = colouring
    colour = tuple(int(best.get(c, 0)) for c in range(n_vars))
    compressed = CompressedJacobian(n_vars=n_vars, n_colours=max(colour) + 1, colour=colour)
    check_orthogonal(pattern, compressed)
    return compressed


def check_orthogonal(pattern, compressed: CompressedJacobian) -> None:
    """No row may hold two columns of the same colour (``modax/_sparsity.py:213-230``)."""
    for row, cols in enumerate(pattern):
        seen: dict[int, int] = {}
        for c in cols:
            g = compressed.colour[c]
            if g in seen:
                raise ValueError(
                    f"columns {seen[g]} and {c} share colour {g} but both have "
                    f"an entry in row {row}; the colouring is not structurally "
                    "orthogonal for this pattern"
                )
            seen[g] = c
