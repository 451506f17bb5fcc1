"""A sparse direct solver for the Rodas5P iteration matrix, compiled per pattern.

The kernel's matrix ``M = I / (h gamma) - J`` has the Jacobian's pattern plus
the diagonal.  Given that pattern (the ``sparsity`` argument, as in
``modax/_sparse_direct.py``), the host analyses it once:

1. **Order** (``fill_reducing_order``): a symmetric fill-reducing permutation.
   ``modax`` calls SuiteSparse AMD through cvxopt
   (``modax/_sparse_direct.py:91-152``); cvxopt is not part of this build, so
   ``minimum_degree_order`` eliminates on the explicit elimination graph with
   *exact* external degrees -- the quantity AMD approximates.  For the tens to
   hundreds of variables these solvers take the exact graph costs milliseconds.
2. **Symbolic factorisation** (``symbolic_rows``): each row of ``L + U`` is
   found the way the numeric factorisation will build it, up-looking -- row
   ``i`` starts from the pattern's row plus the diagonal and absorbs the upper
   part of every earlier row ``k`` it holds a multiplier for, smallest ``k``
   first (a heap), since absorbing row ``k`` can only add columns right of
   ``k``.  Without cancellation this is the exact fill of an unpivoted LU.
3. **Structure** (``LUStructure``): the rows stored as one CSR image of
   ``L + U`` in elimination order (``indptr``/``indices``, ``diag`` the slot of
   each pivot, which holds ``1 / U_ii`` after factorisation), and the
   ``UpdatePlan`` listing, per multiplier in execution order, the source and
   destination slots of its row update.  CSR by rows, in elimination order, with
   a reciprocal pivot, is the reference's storage (``modax/_sparse_direct.py:187-230``):
   the Jacobian sweeps write into it, so the format decides the numbers.
4. **Emit** (``emit_cuda``): the up-looking factorisation and the two triangular
   solves as CUDA device code, straight-line with literal slots below the size
   thresholds (``modax/_sparse_direct.py:468-469``), loops over ``__constant__``
   tables otherwise.  The transposed solve the discrete adjoint needs is emitted
   the same way.

No pivoting: the permutation is symmetric, so ``I / (h gamma)`` keeps every
pivot structurally present, and a Rosenbrock-W step tolerates an approximate
factorisation (``modax/_sparse_direct.py:51-61``).
"""

from __future__ import annotations

import functools
import heapq
from dataclasses import dataclass

import numpy as np

from menodax_b200._sparsity import SlotMap, colour_columns, normalize_sparsity

ORDERINGS = ("amd", "natural")

# Above these the routines are emitted as loops over constant-memory tables
# instead of straight-line code (the reference's thresholds,
# modax/_sparse_direct.py:468-469).
MAX_UNROLLED_SUBSTITUTIONS = 2048
MAX_UNROLLED_UPDATES = 8192


def minimum_degree_order(pattern: tuple[tuple[int, ...], ...]) -> tuple[int, ...]:
    """Minimum-degree elimination order of the symmetrised pattern."""
    n = len(pattern)
    adj = [set() for _ in range(n)]
    for r, cols in enumerate(pattern):
        for c in cols:
            if c != r:
                adj[r].add(c)
                adj[c].add(r)
    original = [len(a) for a in adj]
    alive = set(range(n))
    order = []
    while alive:
        v = min(alive, key=lambda u: (len(adj[u]), original[u], u))
        nbrs = adj[v]
        for a in nbrs:
            adj[a].discard(v)
            adj[a] |= nbrs - {a}
        adj[v] = set()
        alive.remove(v)
        order.append(v)
    return tuple(order)


def fill_reducing_order(pattern, ordering: str = "amd") -> tuple[int, ...]:
    """A permutation of the variables that keeps ``L + U`` small."""
    if ordering not in ORDERINGS:
        raise ValueError(f"unknown ordering {ordering!r}; expected one of {ORDERINGS}")
    if ordering == "natural":
        return tuple(range(len(pattern)))
    return minimum_degree_order(pattern)


def symbolic_rows(rows: list[list[int]] | tuple[tuple[int, ...], ...]) -> list[np.ndarray]:
    """Sorted column indices of each row of ``L + U`` (diagonal included).

    ``rows`` is the matrix's pattern in elimination indices.  Row ``i`` absorbs
    the strictly-upper structure of each row ``k < i`` in which it holds an
    entry; popping those ``k`` from a min-heap visits them in the order the
    numeric up-looking factorisation does, and any column a merge adds left of
    the diagonal is pushed for a later merge.
    """
    n = len(rows)
    upper: list[np.ndarray] = []
    out: list[np.ndarray] = []
    for i in range(n):
        present = set(int(c) for c in rows[i])
        present.add(i)
        pending = [c for c in present if c < i]
        heapq.heapify(pending)
        while pending:
            k = heapq.heappop(pending)
            for c in upper[k]:
                c = int(c)
                if c not in present:
                    present.add(c)
                    if c < i:
                        heapq.heappush(pending, c)
        cols = np.array(sorted(present), dtype=np.int32)
        out.append(cols)
        upper.append(cols[cols > i])
    return out


@dataclass(frozen=True, eq=False)
class UpdatePlan:
    """The factorisation's row updates, one entry per multiplier in execution order.

    Multiplier ``j`` sits in slot ``mult[j]`` of row ``row[j]`` at column ``k``; it
    is scaled by the reciprocal pivot in slot ``pivot[j]`` and then subtracts
    ``L_ik * lu[s]`` for the sources ``s = src_begin[j] .. src_end[j] - 1`` (row
    ``k``'s upper slots, contiguous in CSR) from the destinations
    ``dst[dst_begin[j] + (s - src_begin[j])]`` (the same columns in row ``i``).
    ``row_begin[i] .. row_begin[i + 1]`` are row ``i``'s multipliers.
    """

    row_begin: np.ndarray
    mult: np.ndarray
    pivot: np.ndarray
    src_begin: np.ndarray
    src_end: np.ndarray
    dst_begin: np.ndarray
    dst: np.ndarray

    @property
    def n_updates(self) -> int:
        return int(self.dst.size)


@dataclass(frozen=True, eq=False)
class LUStructure:
    """``L + U`` of the permuted matrix as one CSR image in elimination order.

    Row ``i`` of the image is the caller's variable ``order[i]``; ``indices`` are
    elimination indices, sorted within each row, so a row's strictly-lower slots
    run ``indptr[i] .. diag[i] - 1`` and its upper ones ``diag[i] + 1 ..
    indptr[i + 1] - 1``.
    """

    order: tuple[int, ...]
    indptr: np.ndarray
    indices: np.ndarray
    diag: np.ndarray
    plan: UpdatePlan

    @property
    def n_vars(self) -> int:
        return len(self.order)

    @property
    def nnz(self) -> int:
        return int(self.indptr[-1])

    @property
    def row_origin(self) -> np.ndarray:
        """Caller's index of each elimination row."""
        return np.asarray(self.order, dtype=np.int32)

    @property
    def col_origin(self) -> np.ndarray:
        """Caller's index of the column of each slot."""
        return self.row_origin[self.indices]

    def caller_slots(self) -> np.ndarray:
        """``(n, n)`` slot of each caller-indexed entry, ``-1`` outside ``L + U``."""
        table = np.full((self.n_vars, self.n_vars), -1, dtype=np.int64)
        rows = np.repeat(self.row_origin, np.diff(self.indptr))
        table[rows, self.col_origin] = np.arange(self.nnz)
        return table

    def counts(self) -> tuple[int, int, int]:
        """``(multipliers, updates, substitutions)``: one factorisation's scalings and
        multiply-adds, and one solve's multiply-adds (both substitutions)."""
        multipliers = int(self.plan.mult.size)
        return multipliers, self.plan.n_updates, self.nnz - self.n_vars


def _plan_updates(indptr: np.ndarray, indices: np.ndarray, diag: np.ndarray) -> UpdatePlan:
    n = indptr.size - 1
    row_begin, mult, pivot, src_begin, src_end, dst_begin, dst = [0], [], [], [], [], [], []
    for i in range(n):
        lo, hi = int(indptr[i]), int(indptr[i + 1])
        where = {int(c): s for s, c in zip(range(lo, hi), indices[lo:hi])}
        for p in range(lo, int(diag[i])):
            k = int(indices[p])
            s0, s1 = int(diag[k]) + 1, int(indptr[k + 1])
            mult.append(p)
            pivot.append(int(diag[k]))
            src_begin.append(s0)
            src_end.append(s1)
            dst_begin.append(len(dst))
            dst.extend(where[int(c)] for c in indices[s0:s1])
        row_begin.append(len(mult))
    as32 = lambda v: np.asarray(v, dtype=np.int32)  # noqa: E731
    return UpdatePlan(as32(row_begin), as32(mult), as32(pivot), as32(src_begin), as32(src_end),
                      as32(dst_begin), as32(dst))


def analyse(pattern: tuple[tuple[int, ...], ...], ordering: str = "amd") -> LUStructure:
    """Order the pattern, factorise it symbolically and lay ``L + U`` out in CSR."""
    order = fill_reducing_order(pattern, ordering)
    position = np.empty(len(order), dtype=np.int64)
    position[np.asarray(order, dtype=np.int64)] = np.arange(len(order))
    permuted = [sorted(int(position[c]) for c in pattern[v]) for v in order]
    rows = symbolic_rows(permuted)
    indptr = np.concatenate([[0], np.cumsum([r.size for r in rows])]).astype(np.int32)
    indices = np.concatenate(rows).astype(np.int32) if rows else np.zeros(0, dtype=np.int32)
    diag = np.array([int(indptr[i]) + int(np.searchsorted(r, i)) for i, r in enumerate(rows)],
                    dtype=np.int32)
    return LUStructure(tuple(int(v) for v in order), indptr, indices, diag,
                       _plan_updates(indptr, indices, diag))


def csr_slot_map(pattern, structure: LUStructure) -> SlotMap:
    """The pattern's colouring with each sweep value stored at its CSR slot.

    Fill-in slots belong to no Jacobian column and are claimed by no sweep; the
    kernel clears them before the sweeps."""
    partition = colour_columns(pattern)
    table = structure.caller_slots()
    rows = np.array([r for r, cols in enumerate(pattern) for _ in cols], dtype=np.int64)
    cols = np.array([c for cs in pattern for c in cs], dtype=np.int64)
    slots = table[rows, cols]
    if (slots < 0).any():
        k = int(np.flatnonzero(slots < 0)[0])
        raise ValueError(f"entry ({int(rows[k])}, {int(cols[k])}) is in the pattern but not in the "
                         "factorised structure")
    writes = np.full((structure.n_vars, partition.n_colours), -1, dtype=np.int64)
    writes[rows, np.asarray(partition.colour, dtype=np.int64)[cols]] = slots
    diagonal = tuple(int(s) for s in np.diagonal(table))
    return SlotMap(partition, writes, diagonal, structure.nnz)


class SparseLU:
    """One pattern's structure plus the Jacobian slot map that fills it; pivots nothing."""

    def __init__(self, structure: LUStructure, slots: SlotMap):
        self.structure = structure
        self.slots = slots

    @property
    def nnz(self) -> int:
        return self.structure.nnz

    def __repr__(self) -> str:
        m, u, s = self.structure.counts()
        return (f"SparseLU(n={self.structure.n_vars}, nnz={self.nnz}, colours={self.slots.n_colours}, "
                f"multipliers={m}, updates={u}, substitutions={s})")


@functools.cache
def sparse_lu_for(pattern, ordering: str = "amd") -> SparseLU:
    """Analysis of a normalised pattern, cached on it."""
    structure = analyse(pattern, ordering)
    return SparseLU(structure, csr_slot_map(pattern, structure))


def sparse_lu(sparsity, n_vars: int, *, ordering: str = "amd") -> SparseLU:
    """Analysis of a pattern in any form ``normalize_sparsity`` accepts."""
    return sparse_lu_for(normalize_sparsity(sparsity, n_vars), ordering)


# --- CUDA emission -------------------------------------------------------------------
def _c_array(name: str, values) -> str:
    body = ",".join(str(int(v)) for v in values) or "0"
    return f"__constant__ int {name}[{max(1, len(values))}] = {{{body}}};"


def emit_cuda(structure: LUStructure, mode: str = "auto", fast: bool = False) -> str:
    """``mdx_sparse_factorize`` / ``mdx_sparse_solve`` / ``mdx_sparse_solve_t`` for one structure.

    ``T`` is the LU element type.  Multipliers and updates run in ``T`` and the
    reciprocal pivot is formed in double, as ``modax`` does (numba's typing of
    ``1.0 / lu[pivot]``, ``modax/_sparse_direct.py:520, 545``).  ``mode`` is
    ``"auto"`` (straight-line below the size thresholds), ``"unrolled"`` or
    ``"tables"``; the two forms perform the same operations in the same order.
    ``fast`` (the FP32-LU product path, held to accuracy rather than to the
    reference's bits) takes the reciprocal pivot in ``T`` with ``mdx::fast_recip``
    and subtracts each back-substitution row's terms latest-solved last.
    """
    if mode not in ("auto", "unrolled", "tables"):
        raise ValueError(f"sparse code mode must be 'auto', 'unrolled' or 'tables'; got {mode!r}")
    n = structure.n_vars
    indptr, diag = structure.indptr, structure.diag
    origin, col_origin = structure.row_origin, structure.col_origin
    plan = structure.plan
    _, updates, substitutions = structure.counts()
    out = []
    # The reciprocal pivot: double then rounded, as the reference types it; in the
    # fast path mdx::fast_recip in the LU type (approximate in FP32).
    recip = "mdx::fast_recip(lu[{0}])" if fast else "(T)(1.0 / (double)lu[{0}])"

    unroll_factor = mode == "unrolled" or (mode == "auto" and updates <= MAX_UNROLLED_UPDATES)
    unroll_solve = mode == "unrolled" or (mode == "auto" and substitutions <= MAX_UNROLLED_SUBSTITUTIONS)
    if unroll_factor:
        lines = []
        for i in range(n):
            for j in range(int(plan.row_begin[i]), int(plan.row_begin[i + 1])):
                p, above = int(plan.mult[j]), int(plan.pivot[j])
                lines.append(f"  const T f{p} = lu[{p}] * lu[{above}]; lu[{p}] = f{p};")
                q = int(plan.dst_begin[j])
                for s in range(int(plan.src_begin[j]), int(plan.src_end[j])):
                    lines.append(f"  lu[{int(plan.dst[q])}] -= f{p} * lu[{s}];")
                    q += 1
            pivot = int(diag[i])
            lines.append(f"  lu[{pivot}] = {recip.format(pivot)};")
        out.append(
            "template <typename T, class LU> __device__ __forceinline__ void mdx_sparse_factorize(LU& lu) {\n"
            + "\n".join(lines) + "\n}"
        )
    else:
        out.append(_c_array("mdx_lu_rowj", plan.row_begin))
        out.append(_c_array("mdx_lu_diag", diag))
        out.append(_c_array("mdx_lu_mult", plan.mult))
        out.append(_c_array("mdx_lu_pivot", plan.pivot))
        out.append(_c_array("mdx_lu_src", plan.src_begin))
        out.append(_c_array("mdx_lu_srcend", plan.src_end))
        out.append(_c_array("mdx_lu_dst0", plan.dst_begin))
        out.append(_c_array("mdx_lu_dst", plan.dst))
        out.append(
            "template <typename T, class LU> __device__ __forceinline__ void mdx_sparse_factorize(LU& lu) {\n"
            f"  for (int i = 0; i < {n}; ++i) {{\n"
            "    for (int j = mdx_lu_rowj[i]; j < mdx_lu_rowj[i + 1]; ++j) {\n"
            "      const int p = mdx_lu_mult[j];\n"
            "      const T f = lu[p] * lu[mdx_lu_pivot[j]]; lu[p] = f;\n"
            "      int q = mdx_lu_dst0[j];\n"
            "      for (int s = mdx_lu_src[j]; s < mdx_lu_srcend[j]; ++s, ++q) lu[mdx_lu_dst[q]] -= f * lu[s];\n"
            "    }\n"
            "    const int pivot = mdx_lu_diag[i];\n"
            f"    lu[pivot] = {recip.format('pivot')};\n"
            "  }\n}"
        )

    if unroll_solve:
        fwd, back, tfwd, tback = [], [], [], []
        for i in range(n):
            row = int(origin[i])
            terms = "".join(
                f" - lu[{p}] * rhs[{int(col_origin[p])}]" for p in range(int(indptr[i]), int(diag[i]))
            )
            fwd.append(f"  rhs[{row}] = rhs[{row}]{terms};")
        for i in range(n - 1, -1, -1):
            row, pivot = int(origin[i]), int(diag[i])
            upper = range(pivot + 1, int(indptr[i + 1]))
            # The fast path subtracts the back substitution's terms latest-solved
            # last (descending column), so a row waits on one FMA after its last
            # input instead of on all of them; the reference's order is ascending.
            terms = "".join(f" - lu[{p}] * rhs[{int(col_origin[p])}]" for p in (reversed(upper) if fast else upper))
            back.append(f"  rhs[{row}] = (rhs[{row}]{terms}) * lu[{pivot}];")
        # Transposed: U^T z = b by rows of U in elimination order (scatter),
        # then L^T w = z by rows of L in reverse order (scatter).
        for i in range(n):
            row, pivot = int(origin[i]), int(diag[i])
            tfwd.append(f"  rhs[{row}] = rhs[{row}] * lu[{pivot}];")
            for p in range(pivot + 1, int(indptr[i + 1])):
                tfwd.append(f"  rhs[{int(col_origin[p])}] -= lu[{p}] * rhs[{row}];")
        for i in range(n - 1, -1, -1):
            row = int(origin[i])
            for p in range(int(indptr[i]), int(diag[i])):
                tback.append(f"  rhs[{int(col_origin[p])}] -= lu[{p}] * rhs[{row}];")
        out.append(
            "template <typename T, class LU, class R> __device__ __forceinline__ void mdx_sparse_solve(const LU& lu, R& rhs) {\n"
            + "\n".join(fwd + back) + "\n}"
        )
        out.append(
            "template <typename T, class LU, class R> __device__ __forceinline__ void mdx_sparse_solve_t(const LU& lu, R& rhs) {\n"
            + "\n".join(tfwd + tback) + "\n}"
        )
    else:
        out.append(_c_array("mdx_sv_row", indptr))
        out.append(_c_array("mdx_sv_diag", diag))
        out.append(_c_array("mdx_sv_origin", origin))
        out.append(_c_array("mdx_sv_col", col_origin))
        out.append(
            "template <typename T, class LU, class R> __device__ __forceinline__ void mdx_sparse_solve(const LU& lu, R& rhs) {\n"
            f"  for (int i = 0; i < {n}; ++i) {{\n"
            "    const int row = mdx_sv_origin[i]; T acc = rhs[row];\n"
            "    for (int p = mdx_sv_row[i]; p < mdx_sv_diag[i]; ++p) acc -= lu[p] * rhs[mdx_sv_col[p]];\n"
            "    rhs[row] = acc;\n  }\n"
            f"  for (int i = {n - 1}; i >= 0; --i) {{\n"
            "    const int row = mdx_sv_origin[i]; const int pivot = mdx_sv_diag[i]; T acc = rhs[row];\n"
            + ("    for (int p = mdx_sv_row[i + 1] - 1; p > pivot; --p) acc -= lu[p] * rhs[mdx_sv_col[p]];\n"
               if fast else
               "    for (int p = pivot + 1; p < mdx_sv_row[i + 1]; ++p) acc -= lu[p] * rhs[mdx_sv_col[p]];\n")
            + "    rhs[row] = acc * lu[pivot];\n  }\n}"
        )
        out.append(
            "template <typename T, class LU, class R> __device__ __forceinline__ void mdx_sparse_solve_t(const LU& lu, R& rhs) {\n"
            f"  for (int i = 0; i < {n}; ++i) {{\n"
            "    const int row = mdx_sv_origin[i]; const int pivot = mdx_sv_diag[i];\n"
            "    const T z = rhs[row] * lu[pivot]; rhs[row] = z;\n"
            "    for (int p = pivot + 1; p < mdx_sv_row[i + 1]; ++p) rhs[mdx_sv_col[p]] -= lu[p] * z;\n  }\n"
            f"  for (int i = {n - 1}; i >= 0; --i) {{\n"
            "    const int row = mdx_sv_origin[i]; const T w = rhs[row];\n"
            "    for (int p = mdx_sv_row[i]; p < mdx_sv_diag[i]; ++p) rhs[mdx_sv_col[p]] -= lu[p] * w;\n  }\n}"
        )
    return "\n".join(out)
