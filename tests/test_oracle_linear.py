"""Pins the oracle's src/linear restatement to the reference's known answers
(src/linear/mod.rs:96-285)."""
import numpy as np
import pytest

from flursys_b200 import _abi

OPTIONS = _abi.LinearSolverOptions(1e-12, 1e-12, 1000)


def dense_to_triplets(rows):
    r, c, v = [], [], []
    for i, row in enumerate(rows):
        for j, x in enumerate(row):
            if x != 0.0:
                r.append(i); c.append(j); v.append(x)
    return r, c, v


def matrix(oracle, rows):
    r, c, v = dense_to_triplets(rows)
    st, ro, ci, va = oracle.csr_build(len(rows), len(rows), r, c, v)
    assert st == 0
    return ro, ci, va


def test_csr_builder_finalizes_a_sorted_duplicate_free_matrix(oracle):
    # mod.rs:96-113
    st, ro, ci, va = oracle.csr_build(3, 3, [0, 0, 1, 1, 1, 2, 2], [1, 0, 2, 1, 0, 2, 1],
                                      [-1.0, 4.0, -1.0, 4.0, -1.0, 3.0, -1.0])
    assert st == 0
    assert list(ro) == [0, 2, 5, 7]
    assert list(ci) == [0, 1, 0, 1, 2, 1, 2]
    assert list(va) == [4.0, -1.0, -1.0, 4.0, -1.0, -1.0, 3.0]


def test_duplicate_assembly_spmv_and_residual(oracle):
    # mod.rs:115-135
    st, ro, ci, va = oracle.csr_build(2, 2, [0, 0, 0, 1, 1], [0, 0, 1, 0, 1], [2.0, 3.0, -1.0, 1.0, 4.0])
    assert st == 0 and va.size == 4 and va[0] == 5.0
    st, y = oracle.csr_spmv(ro, ci, va, [1.0, 2.0])
    assert st == 0 and list(y) == [3.0, 9.0]
    st, y = oracle.csr_spmv(ro, ci, va, [3.0, -1.0])
    assert list(y) == [16.0, -1.0]
    st, y = oracle.csr_spmv(ro, ci, va, [1.0, 2.0])
    assert list(np.array([5.0, 10.0]) - y) == [2.0, 1.0]


def test_malformed_csr_is_rejected(oracle):
    # mod.rs:137-161
    import ctypes as C
    lib = oracle.load()
    msg = C.create_string_buffer(256)

    def validate(nrows, ncols, ro, ci, va):
        ro = np.array(ro, dtype=np.int64); ci = np.array(ci or [0], dtype=np.int64)
        va = np.array(va or [0.0], dtype=np.float64)
        nnz = len(va) if ro[-1] == len(va) else int(ro[-1]) - 1
        return lib.orc_csr_validate(nrows, ncols, nnz, _abi.i64ptr(ro), _abi.i64ptr(ci), _abi.dptr(va), msg, 256)

    assert validate(1, 1, [1, 1], [], []) == _abi.ERR_INVALID_CSR
    assert validate(1, 1, [0, 1], [1], [1.0]) == _abi.ERR_INVALID_CSR
    assert validate(1, 1, [0, 1], [0], [float("nan")]) == _abi.ERR_NON_FINITE


def test_jacobi_rejects_missing_and_zero_diagonals(oracle):
    # mod.rs:163-183
    import ctypes as C
    lib = oracle.load()
    ro, ci, va = matrix(oracle, [[0.0, 1.0], [1.0, 1.0]])
    inv = np.zeros(2)
    bad = C.c_int64()
    st = lib.orc_jacobi_inverse_diagonal(2, va.size, _abi.i64ptr(ro), _abi.i64ptr(ci), _abi.dptr(va),
                                         _abi.dptr(inv), C.byref(bad))
    assert st == _abi.ERR_MISSING_DIAGONAL and bad.value == 0
    ro = np.array([0, 2, 4], dtype=np.int64); ci = np.array([0, 1, 0, 1], dtype=np.int64)
    va = np.array([0.0, 1.0, 1.0, 2.0])
    st = lib.orc_jacobi_inverse_diagonal(2, 4, _abi.i64ptr(ro), _abi.i64ptr(ci), _abi.dptr(va), _abi.dptr(inv),
                                         C.byref(bad))
    assert st == _abi.ERR_ZERO_DIAGONAL and bad.value == 0


def test_cg_pcg_and_bicgstab_recover_known_solutions(oracle):
    # mod.rs:185-226
    spd = [[4.0, 1.0], [1.0, 3.0]]
    exact = np.array([1.0 / 11.0, 7.0 / 11.0])
    rhs = np.array(spd) @ exact
    ro, ci, va = matrix(oracle, spd)
    st, x, rep = oracle.csr_solve("cg", ro, ci, va, rhs, [0.0, 0.0], OPTIONS)
    assert st == 0 and rep.status == _abi.LINEAR_CONVERGED
    assert rep.final_residual <= 1e-12 + 1e-12 * rep.initial_residual
    assert np.all(np.abs(x - exact) < 1e-10)
    cg_its = rep.iterations
    st, x, rep = oracle.csr_solve("pcg", ro, ci, va, rhs, [0.0, 0.0], OPTIONS)
    assert st == 0 and rep.status == _abi.LINEAR_CONVERGED and rep.iterations <= cg_its
    assert np.all(np.abs(x - exact) < 1e-10)
    ns = [[4.0, 1.0, 0.0], [2.0, 3.0, 1.0], [0.0, 1.0, 2.0]]
    expected = np.array([1.0, -2.0, 3.0])
    ro, ci, va = matrix(oracle, ns)
    st, x, rep = oracle.csr_solve("bicgstab", ro, ci, va, np.array(ns) @ expected, [0.0] * 3, OPTIONS)
    assert st == 0 and rep.status == _abi.LINEAR_CONVERGED
    assert np.all(np.abs(x - expected) < 1e-10)


def tridiag(oracle, size):
    r, c, v = [], [], []
    for row in range(size):
        r.append(row); c.append(row); v.append(2.0)
        if row > 0:
            r.append(row); c.append(row - 1); v.append(-1.0)
        if row + 1 < size:
            r.append(row); c.append(row + 1); v.append(-1.0)
    st, ro, ci, va = oracle.csr_build(size, size, r, c, v)
    return ro, ci, va


def test_iterative_solvers_handle_large_initial_and_failure_cases(oracle):
    # mod.rs:228-284
    size = 32
    ro, ci, va = tridiag(oracle, size)
    exact = (np.arange(size) + 1.0) / size
    st, rhs = oracle.csr_spmv(ro, ci, va, exact)
    st, x, rep = oracle.csr_solve("cg", ro, ci, va, rhs, np.zeros(size), OPTIONS)
    assert st == 0 and rep.status == _abi.LINEAR_CONVERGED
    assert np.all(np.abs(x - exact) < 1e-10)
    st, _, rep = oracle.csr_solve("bicgstab", ro, ci, va, np.zeros(size), x, OPTIONS)
    assert rep.iterations > 0
    st, _, rep = oracle.csr_solve("cg", ro, ci, va, rhs, exact, OPTIONS)
    assert rep.iterations == 0
    st, _, rep = oracle.csr_solve("bicgstab", ro, ci, va, np.zeros(size), np.zeros(size), OPTIONS)
    assert st == 0 and rep.status == _abi.LINEAR_CONVERGED and rep.iterations == 0
    st, _, rep = oracle.csr_solve("cg", ro, ci, va, rhs, np.zeros(size), _abi.LinearSolverOptions(1e-12, 1e-12, 1))
    assert st == 0 and rep.status == _abi.LINEAR_MAX_ITERATIONS
    st, _, _ = oracle.csr_solve("bicgstab", [0, 0], np.zeros(0, dtype=np.int64), np.zeros(0), [1.0], [0.0], OPTIONS)
    assert st == _abi.ERR_BREAKDOWN
    st, _, _ = oracle.csr_solve("cg", ro, ci, va, np.full(size, np.inf), np.zeros(size), OPTIONS)
    assert st == _abi.ERR_NON_FINITE
