"""src/linear on the device (flursys_cuda_csr_*) against the oracle and the
reference's own known answers (src/linear/mod.rs:185-284)."""
import ctypes as C

import numpy as np
import pytest

from flursys_b200 import _abi

from .paritylib import rel_l2

pytestmark = pytest.mark.gpu

OPTIONS = _abi.LinearSolverOptions(1e-12, 1e-12, 1000)


def gpu_solve(lib, method, ro, ci, va, rhs, x0, opts=OPTIONS):
    ro = np.ascontiguousarray(ro, dtype=np.int64)
    ci = np.ascontiguousarray(ci, dtype=np.int64) if len(ci) else np.zeros(1, dtype=np.int64)
    va = np.ascontiguousarray(va, dtype=np.float64) if len(va) else np.zeros(1)
    b = np.ascontiguousarray(rhs, dtype=np.float64)
    x = np.array(x0, dtype=np.float64)
    rep = _abi.LinearSolveReport()
    fn = {"cg": lib.flursys_cuda_csr_cg, "pcg": lib.flursys_cuda_csr_pcg, "bicgstab": lib.flursys_cuda_csr_bicgstab}[method]
    st = fn(ro.size - 1, int(ro[-1]), _abi.i64ptr(ro), _abi.i64ptr(ci), _abi.dptr(va), _abi.dptr(b), _abi.dptr(x),
            C.byref(opts), C.byref(rep))
    return st, x, rep


def dense(oracle, rows):
    r, c, v = [], [], []
    for i, row in enumerate(rows):
        for j, val in enumerate(row):
            if val != 0.0:
                r.append(i); c.append(j); v.append(val)
    st, ro, ci, va = oracle.csr_build(len(rows), len(rows), r, c, v)
    return ro, ci, va


def test_known_solutions(oracle, cudalib):
    spd = [[4.0, 1.0], [1.0, 3.0]]
    exact = np.array([1.0 / 11.0, 7.0 / 11.0])
    ro, ci, va = dense(oracle, spd)
    st, x, rep = gpu_solve(cudalib, "cg", ro, ci, va, np.array(spd) @ exact, [0.0, 0.0])
    assert st == 0 and rep.status == _abi.LINEAR_CONVERGED and np.all(np.abs(x - exact) < 1e-10)
    cg_its = rep.iterations
    st, x, rep = gpu_solve(cudalib, "pcg", ro, ci, va, np.array(spd) @ exact, [0.0, 0.0])
    assert st == 0 and rep.iterations <= cg_its and np.all(np.abs(x - exact) < 1e-10)
    ns = [[4.0, 1.0, 0.0], [2.0, 3.0, 1.0], [0.0, 1.0, 2.0]]
    expected = np.array([1.0, -2.0, 3.0])
    ro, ci, va = dense(oracle, ns)
    st, x, rep = gpu_solve(cudalib, "bicgstab", ro, ci, va, np.array(ns) @ expected, [0.0] * 3)
    assert st == 0 and rep.status == _abi.LINEAR_CONVERGED and np.all(np.abs(x - expected) < 1e-10)


def test_failure_and_edge_cases(oracle, cudalib):
    size = 32
    r, c, v = [], [], []
    for row in range(size):
        r.append(row); c.append(row); v.append(2.0)
        if row > 0:
            r.append(row); c.append(row - 1); v.append(-1.0)
        if row + 1 < size:
            r.append(row); c.append(row + 1); v.append(-1.0)
    st, ro, ci, va = oracle.csr_build(size, size, r, c, v)
    exact = (np.arange(size) + 1.0) / size
    _, rhs = oracle.csr_spmv(ro, ci, va, exact)
    st, x, rep = gpu_solve(cudalib, "cg", ro, ci, va, rhs, np.zeros(size))
    assert st == 0 and np.all(np.abs(x - exact) < 1e-10)
    st, _, rep = gpu_solve(cudalib, "cg", ro, ci, va, rhs, exact)
    assert st == 0 and rep.iterations == 0
    st, _, rep = gpu_solve(cudalib, "bicgstab", ro, ci, va, np.zeros(size), np.zeros(size))
    assert st == 0 and rep.status == _abi.LINEAR_CONVERGED and rep.iterations == 0
    st, _, rep = gpu_solve(cudalib, "bicgstab", ro, ci, va, np.zeros(size), x)
    assert st == 0 and rep.iterations > 0
    st, _, rep = gpu_solve(cudalib, "cg", ro, ci, va, rhs, np.zeros(size), _abi.LinearSolverOptions(1e-12, 1e-12, 1))
    assert st == 0 and rep.status == _abi.LINEAR_MAX_ITERATIONS
    st, _, _ = gpu_solve(cudalib, "bicgstab", [0, 0], [], [], [1.0], [0.0])
    assert st == _abi.ERR_BREAKDOWN
    st, _, _ = gpu_solve(cudalib, "cg", ro, ci, va, np.full(size, np.inf), np.zeros(size))
    assert st == _abi.ERR_NON_FINITE
    # malformed CSR and Jacobi failures (mod.rs:137-183)
    st, _, _ = gpu_solve(cudalib, "cg", [0, 1], [1], [1.0], [1.0], [0.0])
    assert st == _abi.ERR_INVALID_CSR
    st, _, _ = gpu_solve(cudalib, "pcg", *dense(oracle, [[0.0, 1.0], [1.0, 1.0]]), [1.0, 1.0], [0.0, 0.0])
    assert st == _abi.ERR_MISSING_DIAGONAL
    st, _, _ = gpu_solve(cudalib, "pcg", [0, 2, 4], [0, 1, 0, 1], [0.0, 1.0, 1.0, 2.0], [1.0, 1.0], [0.0, 0.0])
    assert st == _abi.ERR_ZERO_DIAGONAL


def poisson_csr(nx, ny, shift=0.0):
    """5-point operator with a diagonal shift (SPD) on an nx x ny grid."""
    rows, cols, vals = [], [], []
    for j in range(ny):
        for i in range(nx):
            k = i + nx * j
            diag = shift
            for di, dj in ((1, 0), (-1, 0), (0, 1), (0, -1)):
                ii, jj = i + di, j + dj
                if 0 <= ii < nx and 0 <= jj < ny:
                    rows.append(k); cols.append(ii + nx * jj); vals.append(-1.0)
                    diag += 1.0
            rows.append(k); cols.append(k); vals.append(diag)
    return np.array(rows), np.array(cols), np.array(vals)


@pytest.mark.parametrize("method", ["cg", "pcg", "bicgstab"])
def test_five_point_systems_match_oracle(oracle, cudalib, method):
    nx, ny = 48, 40
    r, c, v = poisson_csr(nx, ny, shift=0.01)
    if method == "bicgstab":  # a non-symmetric convection-like perturbation
        v = v + np.where(c == r + 1, -0.2, 0.0) + np.where(c == r, 0.5, 0.0)
    st, ro, ci, va = oracle.csr_build(nx * ny, nx * ny, r, c, v)
    rng = np.random.default_rng(1)
    rhs = rng.standard_normal(nx * ny)
    opts = _abi.LinearSolverOptions(0.0, 1e-10, 5000)
    st, xref, rref = oracle.csr_solve(method, ro, ci, va, rhs, np.zeros_like(rhs), opts)
    assert st == 0
    st, x, rep = gpu_solve(cudalib, method, ro, ci, va, rhs, np.zeros_like(rhs), opts)
    assert st == 0 and rep.status == _abi.LINEAR_CONVERGED
    if method != "bicgstab":
        # CG iterates are stable under reduction-order changes; BiCGSTAB's
        # irregular convergence amplifies them, so only its solution is compared.
        assert abs(rep.iterations - rref.iterations) <= 2
    assert rep.final_residual <= 1e-10 * rep.initial_residual
    assert rel_l2(x, xref) < 1e-7


def test_spmv_matches_oracle(oracle, cudalib):
    r, c, v = poisson_csr(30, 20)
    st, ro, ci, va = oracle.csr_build(600, 600, r, c, v)
    xin = np.random.default_rng(2).standard_normal(600)
    _, yref = oracle.csr_spmv(ro, ci, va, xin)
    y = np.zeros(600)
    st = cudalib.flursys_cuda_csr_spmv(600, 600, va.size, _abi.i64ptr(ro), _abi.i64ptr(ci), _abi.dptr(va),
                                       _abi.dptr(xin), _abi.dptr(y))
    assert st == 0
    assert np.max(np.abs(y - yref)) <= 1e-12 * np.max(np.abs(yref))
