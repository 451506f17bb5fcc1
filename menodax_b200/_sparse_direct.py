"""A sparse direct solver for the Rodas5P iteration matrix, compiled per pattern.

Host-side analysis, once per pattern, as ``modax/_sparse_direct.py`` does it:

1. **Order** (``fill_reducing_order``): a symmetric fill-reducing permutation of
   ``S + S^T + I``.  ``modax`` calls SuiteSparse AMD through cvxopt
   (``modax/_sparse_direct.py:91-152``); cvxopt is not part of this build, so the
   ordering here is this module's own minimum-degree elimination on the
   explicit elimination graph, with *exact* external degrees -- the quantity AMD
   approximates.  For the tens-to-hundreds of variables these solvers take, the
   exact graph costs milliseconds.  Ties go to the vertex with the smaller
   original degree, then the smaller index.
2. **Fill** (``fill_pattern``): pattern-only unpivoted Gaussian elimination gives
   the exact ``L + U`` structure (``modax/_sparse_direct.py:155-184``).
3. **Layout** (``analyse``/``SparseLULayout``): one CSR image of ``L + U`` in
   elimination order, ``row_ptr``/``col_ind``/``diag_ptr``, the diagonal holding
   ``1/U_ii`` after factorisation (``modax/_sparse_direct.py:187-349``).
4. **Emit** (``emit_cuda``): the up-looking factorisation and the two
   triangular solves as CUDA device code, straight-line with literal slots when
   small (``modax/_sparse_direct.py:468-469`` thresholds), loops over
   ``__constant__`` index tables otherwise.  The transposed solve the discrete
   adjoint needs is emitted the same way.

No pivoting: the permutation is symmetric so ``I/(h*gamma)`` keeps every pivot
structurally present, and a Rosenbrock-W step tolerates an approximate
factorisation (``modax/_sparse_direct.py:51-61``).
"""

from __future__ import annotations

import functools
from dataclasses import dataclass, replace

import numpy as np

from menodax_b200._sparsity import CompressedJacobian, colour_sparsity, normalize_sparsity

ORDERINGS = ("amd", "natural")

# Above these the routines are emitted as loops over constant-memory tables
# instead of straight-line code (modax/_sparse_direct.py:468-469).
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


def fill_pattern(pattern: tuple[tuple[int, ...], ...]) -> np.ndarray:
    """Exact boolean ``L + U`` pattern of an unpivoted LU, diagonal included."""
    n = len(pattern)
    filled = np.zeros((n, n), dtype=bool)
    for row, cols in enumerate(pattern):
        filled[row, list(cols)] = True
    np.fill_diagonal(filled, True)
    for k in range(n):
        below = np.flatnonzero(filled[k + 1:, k]) + k + 1
        if below.size:
            filled[below, k + 1:] |= filled[k, k + 1:]
    return filled


@dataclass(frozen=True)
class SparseLULayout:
    """CSR image of ``L + U`` in elimination order (row ``i`` is variable ``order[i]``)."""

    n_vars: int
    order: tuple[int, ...]
    row_ptr: np.ndarray
    col_ind: np.ndarray
    diag_ptr: np.ndarray

    @property
    def nnz(self) -> int:
        return int(self.row_ptr[-1])

    @property
    def row_origin(self) -> np.ndarray:
        return np.asarray(self.order, dtype=np.int32)

    @property
    def col_origin(self) -> np.ndarray:
        return np.asarray(self.order, dtype=np.int32)[self.col_ind]

    def slot_table(self) -> np.ndarray:
        """``(n, n)`` caller-index -> slot map, ``-1`` outside the structure."""
        table = np.full((self.n_vars, self.n_vars), -1, dtype=np.int64)
        origin = np.asarray(self.order, dtype=np.int64)
        for i in range(self.n_vars):
            start, stop = int(self.row_ptr[i]), int(self.row_ptr[i + 1])
            table[origin[i], origin[self.col_ind[start:stop]]] = np.arange(start, stop)
        return table

    def factorization_ops(self):
        """``(dst_start, destination, upper_end)`` indexed by multiplier slot.

        For multiplier ``p = (i, k)`` the update ``row_i -= L_ik * U_k,k+1:`` reads
        row ``k``'s upper slots ``diag_ptr[k]+1 .. row_ptr[k+1]`` in order and
        writes ``destination[dst_start[p] + j]`` (``modax/_sparse_direct.py:241-283``).
        """
        n = self.n_vars
        dst_start = np.zeros(self.nnz, dtype=np.int64)
        upper_end = np.asarray(self.row_ptr[1:], dtype=np.int64)[np.asarray(self.col_ind, dtype=np.int64)]
        dst: list[int] = []
        table = np.full((n, n), -1, dtype=np.int64)
        for i in range(n):
            start, stop = int(self.row_ptr[i]), int(self.row_ptr[i + 1])
            table[i, self.col_ind[start:stop]] = np.arange(start, stop)
        for i in range(n):
            for p in range(int(self.row_ptr[i]), int(self.diag_ptr[i])):
                k = int(self.col_ind[p])
                dst_start[p] = len(dst)
                for q in range(int(self.diag_ptr[k]) + 1, int(self.row_ptr[k + 1])):
                    dst.append(int(table[i, int(self.col_ind[q])]))
        return (
            dst_start.astype(np.int32),
            np.asarray(dst, dtype=np.int32),
            upper_end.astype(np.int32),
        )

    def flop_counts(self) -> tuple[int, int, int]:
        """``(multipliers, updates, substitutions)`` of one factorisation / one solve."""
        lower = self.diag_ptr - self.row_ptr[:-1]
        upper = self.row_ptr[1:] - self.diag_ptr - 1
        multipliers = int(lower.sum())
        slot = np.arange(self.nnz)
        row = np.repeat(np.arange(self.n_vars), np.diff(self.row_ptr))
        lower_mask = slot < self.diag_ptr[row]
        updates = int(upper[self.col_ind[lower_mask]].sum())
        return multipliers, updates, multipliers + int(upper.sum())


def analyse(pattern: tuple[tuple[int, ...], ...], ordering: str = "amd") -> SparseLULayout:
    """Order, factorise symbolically, and lay out ``L + U`` in CSR."""
    n_vars = len(pattern)
    order = fill_reducing_order(pattern, ordering)
    forward = np.asarray(order, dtype=np.int64)
    inverse = np.empty(n_vars, dtype=np.int64)
    inverse[forward] = np.arange(n_vars)
    filled = fill_pattern(
        tuple(
            tuple(sorted(int(inverse[c]) for c in pattern[int(forward[i])]))
            for i in range(n_vars)
        )
    )
    row_ptr = np.zeros(n_vars + 1, dtype=np.int32)
    row_ptr[1:] = np.cumsum(filled.sum(axis=1))
    col_ind = np.concatenate([np.flatnonzero(filled[i]) for i in range(n_vars)]).astype(np.int32)
    diag_ptr = np.array(
        [int(row_ptr[i]) + int(np.searchsorted(col_ind[row_ptr[i]:row_ptr[i + 1]], i))
         for i in range(n_vars)],
        dtype=np.int32,
    )
    return SparseLULayout(n_vars, tuple(int(i) for i in order), row_ptr, col_ind, diag_ptr)


def compressed_jacobian(pattern, layout: SparseLULayout) -> CompressedJacobian:
    """Colour-grid positions remapped onto the factorisation's CSR slots."""
    compressed = colour_sparsity(pattern)
    table = layout.slot_table()
    packed = np.full(layout.n_vars * compressed.n_colours, -1, dtype=np.int64)
    for row, cols in enumerate(pattern):
        for col in cols:
            slot = int(table[row, col])
            if slot < 0:
                raise ValueError(
                    f"entry ({row}, {col}) is in the pattern but not in the "
                    "factorised structure"
                )
            packed[row * compressed.n_colours + compressed.colour[col]] = slot
    diagonal = np.array([int(table[i, i]) for i in range(layout.n_vars)])
    return replace(
        compressed,
        packed=tuple(int(s) for s in packed),
        packed_diagonal=tuple(int(s) for s in diagonal),
        n_slots=layout.nnz,
    )


class SparseDirectSolver:
    """A layout plus the Jacobian slot map that fills it; pivots nothing."""

    ipiv_size = 1

    def __init__(self, layout: SparseLULayout, compressed: CompressedJacobian):
        self.layout = layout
        self.compressed = compressed
        self.ops = layout.factorization_ops()

    @property
    def nnz(self) -> int:
        return self.layout.nnz

    def __repr__(self) -> str:
        m, u, s = self.layout.flop_counts()
        return (
            f"<SparseDirectSolver n_vars={self.layout.n_vars} nnz={self.nnz} "
            f"factorise={m + u} solve={s} colours={self.compressed.n_colours}>"
        )


@functools.cache
def sparse_direct_solver_for(pattern, ordering: str = "amd") -> SparseDirectSolver:
    layout = analyse(pattern, ordering)
    return SparseDirectSolver(layout, compressed_jacobian(pattern, layout))


def sparse_direct_solver(sparsity, n_vars: int, *, ordering: str = "amd") -> SparseDirectSolver:
    return sparse_direct_solver_for(normalize_sparsity(sparsity, n_vars), ordering)


# --- CUDA emission -------------------------------------------------------------------
def _c_array(name: str, values) -> str:
    body = ",".join(str(int(v)) for v in values) or "0"
    return f"__constant__ int {name}[{max(1, len(values))}] = {{{body}}};"


def emit_cuda(layout: SparseLULayout, ops, mode: str = "auto", fast: bool = False) -> str:
    """``mdx_sparse_factorize`` / ``mdx_sparse_solve`` / ``mdx_sparse_solve_t`` for one layout.

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
    n = layout.n_vars
    row_ptr, diag_ptr = layout.row_ptr, layout.diag_ptr
    origin, col_origin = layout.row_origin, layout.col_origin
    dst_start, destination, upper_end = ops
    pivot_of = diag_ptr[layout.col_ind]
    _, updates, substitutions = layout.flop_counts()
    out = []
    # The reciprocal pivot: double then rounded, as the reference types it; in the
    # fast path mdx::fast_recip in the LU type (approximate in FP32).
    recip = "mdx::fast_recip(lu[{0}])" if fast else "(T)(1.0 / (double)lu[{0}])"

    unroll_factor = mode == "unrolled" or (mode == "auto" and destination.size <= MAX_UNROLLED_UPDATES)
    unroll_solve = mode == "unrolled" or (mode == "auto" and substitutions <= MAX_UNROLLED_SUBSTITUTIONS)
    if unroll_factor:
        lines = []
        for i in range(n):
            for p in range(int(row_ptr[i]), int(diag_ptr[i])):
                above = int(pivot_of[p])
                lines.append(f"  const T f{p} = lu[{p}] * lu[{above}]; lu[{p}] = f{p};")
                q = int(dst_start[p])
                for s in range(above + 1, int(upper_end[p])):
                    lines.append(f"  lu[{int(destination[q])}] -= f{p} * lu[{s}];")
                    q += 1
            pivot = int(diag_ptr[i])
            lines.append(f"  lu[{pivot}] = {recip.format(pivot)};")
        out.append(
            "template <typename T, class LU> __device__ __forceinline__ void mdx_sparse_factorize(LU& lu) {\n"
            + "\n".join(lines) + "\n}"
        )
    else:
        out.append(_c_array("mdx_lu_row", row_ptr))
        out.append(_c_array("mdx_lu_diag", diag_ptr))
        out.append(_c_array("mdx_lu_pivot", pivot_of))
        out.append(_c_array("mdx_lu_start", dst_start))
        out.append(_c_array("mdx_lu_end", upper_end))
        out.append(_c_array("mdx_lu_dst", destination))
        out.append(
            "template <typename T, class LU> __device__ __forceinline__ void mdx_sparse_factorize(LU& lu) {\n"
            f"  for (int i = 0; i < {n}; ++i) {{\n"
            "    const int pivot = mdx_lu_diag[i];\n"
            "    for (int p = mdx_lu_row[i]; p < pivot; ++p) {\n"
            "      const int above = mdx_lu_pivot[p];\n"
            "      const T f = lu[p] * lu[above]; lu[p] = f;\n"
            "      int q = mdx_lu_start[p];\n"
            "      for (int s = above + 1; s < mdx_lu_end[p]; ++s, ++q) lu[mdx_lu_dst[q]] -= f * lu[s];\n"
            "    }\n"
            f"    lu[pivot] = {recip.format('pivot')};\n"
            "  }\n}"
        )

    if unroll_solve:
        fwd, back, tfwd, tback = [], [], [], []
        for i in range(n):
            row = int(origin[i])
            terms = "".join(
                f" - lu[{p}] * rhs[{int(col_origin[p])}]" for p in range(int(row_ptr[i]), int(diag_ptr[i]))
            )
            fwd.append(f"  rhs[{row}] = rhs[{row}]{terms};")
        for i in range(n - 1, -1, -1):
            row, pivot = int(origin[i]), int(diag_ptr[i])
            upper = range(pivot + 1, int(row_ptr[i + 1]))
            # The fast path subtracts the back substitution's terms latest-solved
            # last (descending column), so a row waits on one FMA after its last
            # input instead of on all of them; the reference's order is ascending.
            terms = "".join(f" - lu[{p}] * rhs[{int(col_origin[p])}]" for p in (reversed(upper) if fast else upper))
            back.append(f"  rhs[{row}] = (rhs[{row}]{terms}) * lu[{pivot}];")
        # Transposed: U^T z = b by rows of U in elimination order (scatter),
        # then L^T w = z by rows of L in reverse order (scatter).
        for i in range(n):
            row, pivot = int(origin[i]), int(diag_ptr[i])
            tfwd.append(f"  rhs[{row}] = rhs[{row}] * lu[{pivot}];")
            for p in range(pivot + 1, int(row_ptr[i + 1])):
                tfwd.append(f"  rhs[{int(col_origin[p])}] -= lu[{p}] * rhs[{row}];")
        for i in range(n - 1, -1, -1):
            row = int(origin[i])
            for p in range(int(row_ptr[i]), int(diag_ptr[i])):
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
        out.append(_c_array("mdx_sv_row", row_ptr))
        out.append(_c_array("mdx_sv_diag", diag_ptr))
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
