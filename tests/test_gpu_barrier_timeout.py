"""Bounded device waits: a grid barrier that gives up reports FLURSYS_ERR_TIMEOUT.

The fault is made on the host: flursys_cuda_debug_inject_barrier_fault makes
the next persistent 3D PCG launch wait at its grid barriers for blocks that
were never launched, with a poll limit of a few milliseconds. Every wait runs
out, the kernel returns, and the call must report a timeout rather than a
converged solve (the result record would otherwise hold a cleared or stale
record). The next call on the same context must solve normally. Nothing here
faults or hangs the GPU: each wait ends by its poll limit.
"""
import ctypes as C
import time

import numpy as np
import pytest

from flursys_b200 import _abi

pytestmark = pytest.mark.gpu

SHAPE = (24, 20, 12)


def _rhs():
    rng = np.random.default_rng(5)
    rhs = rng.standard_normal(SHAPE[0] * SHAPE[1] * SHAPE[2])
    rhs[0] = 0.0
    return rhs


def _allocating(lib, rhs):
    nx, ny, nz = SHAPE
    x = np.zeros_like(rhs)
    rep = _abi.LinearSolveReport()
    opts = _abi.LinearSolverOptions(0.0, 1e-10, 5000)
    st = lib.flursys_cuda_stencil_pcg(nx, ny, nz, 1 / nx, 1 / ny, 1 / nz, _abi.dptr(rhs), _abi.dptr(x),
                                      _abi.PRECISION_F64, C.byref(opts), C.byref(rep))
    return st, x, rep


def _no_alloc(lib, rhs):
    import torch
    nx, ny, nz = SHAPE
    d_rhs = torch.from_numpy(rhs).to("cuda")
    d_x = torch.zeros_like(d_rhs)
    rep = _abi.LinearSolveReport()
    opts = _abi.LinearSolverOptions(0.0, 1e-10, 5000)
    st = lib.flursys_cuda_stencil_pcg_noalloc(nx, ny, nz, 1 / nx, 1 / ny, 1 / nz, C.c_void_p(d_rhs.data_ptr()),
                                              C.c_void_p(d_x.data_ptr()), _abi.PRECISION_F64, C.byref(opts),
                                              C.byref(rep), C.c_void_p(torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    return st, d_x.cpu().numpy(), rep


@pytest.mark.parametrize("entry", [_allocating, _no_alloc], ids=["allocating", "no_alloc"])
def test_barrier_timeout_is_reported_and_the_context_survives(cudalib, entry):
    rhs = _rhs()
    st0, x0, r0 = entry(cudalib, rhs)
    assert st0 == 0 and r0.status == _abi.LINEAR_CONVERGED
    assert cudalib.flursys_cuda_debug_inject_barrier_fault(1) == 0
    t0 = time.perf_counter()
    st, _, _ = entry(cudalib, rhs)
    waited = time.perf_counter() - t0
    assert st == _abi.ERR_TIMEOUT
    buf = C.create_string_buffer(256)
    cudalib.flursys_cuda_global_error(buf, 256)
    assert "timed out" in buf.value.decode()
    assert waited < 30.0
    # The injection covered one launch: the next call solves as before.
    st1, x1, r1 = entry(cudalib, rhs)
    assert st1 == 0 and r1.status == _abi.LINEAR_CONVERGED and r1.iterations == r0.iterations
    assert np.array_equal(x1, x0)


def test_negative_injection_is_rejected(cudalib):
    assert cudalib.flursys_cuda_debug_inject_barrier_fault(-1) == _abi.ERR_INVALID_ARGUMENT
    assert cudalib.flursys_cuda_debug_inject_barrier_fault(0) == 0
