"""Host-side sparse analysis: ordering, symbolic fill, CSR layout, colouring.

Ports the reference's host-only tests (tests/test_sparse_direct.py:99-316,
tests/test_sparsity.py:65-109), including the pinned fill counts and a NumPy
replay of the factorisation tables that checks they factorise the matrix.
"""

import numpy as np
import pytest

from menodax_b200._sparse_direct import (
    ORDERINGS,
    SparseLU,
    analyse,
    csr_slot_map,
    sparse_lu,
    symbolic_rows,
)
from menodax_b200._sparsity import colour_sparsity, dense_jacobian, normalize_sparsity


def _arrow(n):
    m = np.eye(n, dtype=bool)
    m[0, :] = m[:, 0] = True
    return m


def _bordered(core, tails, length):
    n = core + tails * length
    m = np.zeros((n, n), dtype=bool)
    m[:core, :core] = True
    for t in range(tails):
        base = core + t * length
        parent = t % core
        for i in range(length):
            m[base + i, base + i] = True
            if i:
                m[base + i, base + i - 1] = True
            if i + 1 < length:
                m[base + i, base + i + 1] = True
        m[base, parent] = m[parent, base] = True
    return m


def _ring(n):
    m = np.zeros((n, n), dtype=bool)
    for i in range(n):
        m[i, i] = m[i, (i + 1) % n] = m[i, (i - 1) % n] = True
    return m


def _matrix(mask, seed=0, shift=60.0):
    rng = np.random.default_rng(seed)
    n = len(mask)
    dense = np.where(mask, rng.normal(size=(n, n)), 0.0)
    dense[np.diag_indices(n)] += shift
    return dense


def _replay(layout, dense):
    """The factorisation and solves the emitted device code performs, in NumPy."""
    n = layout.n_vars
    row_ptr, diag_ptr = layout.indptr, layout.diag
    plan = layout.plan
    origin, col_origin = layout.row_origin, layout.col_origin
    lu = np.zeros(layout.nnz)
    table = layout.caller_slots()
    rows, cols = np.nonzero(table >= 0)
    lu[table[rows, cols]] = dense[rows, cols]
    for i in range(n):
        for j in range(plan.row_begin[i], plan.row_begin[i + 1]):
            p = plan.mult[j]
            f = lu[p] * lu[plan.pivot[j]]
            lu[p] = f
            q = plan.dst_begin[j]
            for s in range(plan.src_begin[j], plan.src_end[j]):
                lu[plan.dst[q]] -= f * lu[s]
                q += 1
        lu[diag_ptr[i]] = 1.0 / lu[diag_ptr[i]]

    def solve(b):
        x = np.asarray(b, dtype=np.float64).copy()
        for i in range(n):
            row = origin[i]
            acc = x[row]
            for p in range(row_ptr[i], diag_ptr[i]):
                acc -= lu[p] * x[col_origin[p]]
            x[row] = acc
        for i in range(n - 1, -1, -1):
            row, pivot = origin[i], diag_ptr[i]
            acc = x[row]
            for p in range(pivot + 1, row_ptr[i + 1]):
                acc -= lu[p] * x[col_origin[p]]
            x[row] = acc * lu[pivot]
        return x

    def solve_t(b):
        # the emitted transposed solve: U^T by rows of U (scatter), then L^T in reverse
        x = np.asarray(b, dtype=np.float64).copy()
        for i in range(n):
            row, pivot = origin[i], diag_ptr[i]
            x[row] = x[row] * lu[pivot]
            for p in range(pivot + 1, row_ptr[i + 1]):
                x[col_origin[p]] -= lu[p] * x[row]
        for i in range(n - 1, -1, -1):
            row = origin[i]
            for p in range(row_ptr[i], diag_ptr[i]):
                x[col_origin[p]] -= lu[p] * x[row]
        return x

    return solve, solve_t


@pytest.mark.parametrize("seed", range(6))
def test_symbolic_rows_are_exactly_what_an_unpivoted_lu_touches(seed):
    """The up-looking symbolic pass against a numeric right-looking elimination of a
    random matrix with the same pattern (no cancellation at these values)."""
    rng = np.random.default_rng(seed)
    n = 12
    mask = (rng.random((n, n)) < 0.2) | np.eye(n, dtype=bool)
    rows = symbolic_rows(normalize_sparsity(mask, n))
    predicted = np.zeros((n, n), dtype=bool)
    for i, cols in enumerate(rows):
        predicted[i, cols] = True
    work = _matrix(mask, seed=seed)
    for k in range(n):
        work[k + 1:, k] /= work[k, k]
        work[k + 1:, k + 1:] -= np.outer(work[k + 1:, k], work[k, k + 1:])
    assert ((work != 0.0) == predicted).all()


def test_ordering_undoes_the_arrow_worst_case():
    pattern = normalize_sparsity(_arrow(12), 12)
    assert analyse(pattern, "natural").nnz == 144
    amd = analyse(pattern, "amd")
    assert amd.nnz == int(_arrow(12).sum())
    assert amd.order[-1] == 0


def test_bordered_block_needs_no_fill():
    mask = _bordered(5, 3, 7)
    amd = analyse(normalize_sparsity(mask, len(mask)), "amd")
    assert amd.nnz == int(mask.sum())
    assert set(amd.order[-5:]) == set(range(5))


@pytest.mark.parametrize("mask, expected", [
    (_arrow(12), 34), (_arrow(40), 118), (_ring(16), 74), (_ring(64), 314),
    (_bordered(5, 3, 7), 88), (_bordered(10, 8, 16), 484),
], ids=["arrow12", "arrow40", "ring16", "ring64", "bordered", "disco-like"])
def test_fill_counts_pinned_by_the_reference(mask, expected):
    """tests/test_sparse_direct.py:194-215 in the reference."""
    assert analyse(normalize_sparsity(mask, len(mask)), "amd").nnz == expected


def test_the_ordering_is_validated():
    with pytest.raises(ValueError, match="unknown ordering"):
        analyse(normalize_sparsity(_ring(4), 4), "minimum-degree-ish")
    assert "amd" in ORDERINGS


MASKS = [_ring(9), _arrow(8), _bordered(4, 2, 5), np.ones((5, 5), dtype=bool)]


@pytest.mark.parametrize("mask", MASKS, ids=["ring", "arrow", "bordered", "dense"])
def test_layout_is_a_consistent_csr_image(mask):
    n = len(mask)
    layout = analyse(normalize_sparsity(mask, n), "natural")
    assert layout.indptr[0] == 0 and layout.indptr[-1] == layout.nnz
    for i in range(n):
        span = layout.indices[layout.indptr[i]:layout.indptr[i + 1]]
        assert (np.diff(span) > 0).all()
        assert layout.indices[layout.diag[i]] == i
    table = layout.caller_slots()
    slots = [int(table[r, c]) for r, c in zip(*np.nonzero(mask))]
    assert min(slots) >= 0 and len(set(slots)) == len(slots) and max(slots) < layout.nnz


@pytest.mark.parametrize("ordering", ["natural", "amd"])
@pytest.mark.parametrize("mask", MASKS, ids=["ring", "arrow", "bordered", "dense"])
def test_the_tables_factorise_the_matrix(mask, ordering):
    n = len(mask)
    layout = analyse(normalize_sparsity(mask, n), ordering)
    dense = _matrix(mask)
    solve, solve_t = _replay(layout, dense)
    rng = np.random.default_rng(1)
    for _ in range(3):
        b = rng.normal(size=n)
        np.testing.assert_allclose(solve(b), np.linalg.solve(dense, b), rtol=1e-10)
        np.testing.assert_allclose(solve_t(b), np.linalg.solve(dense.T, b), rtol=1e-10)


def test_footprint_is_the_factorisation():
    mask = _ring(9)
    pattern = normalize_sparsity(mask, 9)
    layout = analyse(pattern, "natural")
    compressed = csr_slot_map(pattern, layout)
    assert compressed.size == layout.nnz
    assert int((compressed.store_slots() >= 0).sum()) == int(mask.sum()) < compressed.size
    assert len(set(compressed.diagonal)) == 9


def test_solver_object_and_cache():
    a = sparse_lu(_ring(6), 6, ordering="natural")
    assert isinstance(a, SparseLU) and "nnz=" in repr(a)
    b = sparse_lu(np.array(sorted(zip(*np.nonzero(_ring(6))))), 6, ordering="natural")
    assert a is b


def test_tridiagonal_takes_three_colours():
    """tests/test_sparsity.py:65-70."""
    n = 10
    mask = np.eye(n, dtype=bool) | np.eye(n, k=1, dtype=bool) | np.eye(n, k=-1, dtype=bool)
    assert colour_sparsity(normalize_sparsity(mask, n)).n_colours == 3


def test_decay_chain_takes_two_colours():
    """tests/test_sparsity.py:114-116: the chain's four columns in two sweeps."""
    from workloads import systems

    compressed = colour_sparsity(normalize_sparsity(systems.DECAY_CHAIN_PATTERN, 4))
    assert compressed.n_colours == 2


def test_dense_is_row_major():
    d = dense_jacobian(4)
    assert [d.slot(r, c) for r in range(4) for c in range(4)] == list(range(16))


def test_orthogonality_is_checked():
    from menodax_b200._sparsity import assert_orthogonal

    with pytest.raises(ValueError, match="share colour"):
        assert_orthogonal(((0, 1), (1,)), (0, 0))
    assert_orthogonal(((0, 1), (1,)), (0, 1))


def test_seed_table():
    c = colour_sparsity(normalize_sparsity(_ring(6), 6))
    seeds = c.seed_table(8)
    assert seeds.shape == (c.n_colours + 1, 8)
    assert (seeds[-1] == 0).all()
    assert (seeds[:-1, :6].sum(axis=0) == 1).all()


def test_sparsity_spellings_agree():
    import scipy.sparse as sp

    mask = _ring(5)
    a = normalize_sparsity(mask, 5)
    b = normalize_sparsity(np.array(list(zip(*np.nonzero(mask)))), 5)
    c = normalize_sparsity(sp.csr_matrix(mask), 5)
    assert a == b == c
    with pytest.raises(ValueError, match="lies outside"):
        normalize_sparsity(np.array([[0, 7]]), 5)
    with pytest.raises(ValueError, match="mask"):
        normalize_sparsity(np.ones((3, 4)), 5)
