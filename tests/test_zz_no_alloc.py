"""The allocation-free pressure PCG (flursys_cuda_stencil_pcg_noalloc).

Some callers of this library cannot let it allocate device memory — their
own pool owns the device, a hard memory cap is in force, or a cudaFree's
device-wide synchronisation is not acceptable. For them the entry point
works out of a fixed scratch array inside the library. This test calls it
through the C ABI on device buffers that the test owns and checks, on two
calls in a row, that it returns what the allocating entry point
flursys_cuda_stencil_pcg returns for the same system. The file name makes
pytest collect it last.
"""
import ctypes as C

import numpy as np
import pytest

from flursys_b200 import _abi

pytestmark = pytest.mark.gpu

TOL = 1e-10  # the parity tolerance of the FP64 GPU tests


def reference_solve(lib, shape, rhs, precision, opts):
    nx, ny, nz = shape
    x = np.zeros_like(rhs)
    rep = _abi.LinearSolveReport()
    st = lib.flursys_cuda_stencil_pcg(nx, ny, nz, 1 / nx, 1 / ny, 1 / nz, _abi.dptr(rhs), _abi.dptr(x), precision,
                                      C.byref(opts), C.byref(rep))
    assert st == 0
    return x, rep


def noalloc_solve(lib, shape, rhs, precision, opts):
    import torch
    nx, ny, nz = shape
    dev_rhs = torch.from_numpy(rhs).to("cuda")
    dev_x = torch.zeros_like(dev_rhs)
    stream = torch.cuda.current_stream()
    rep = _abi.LinearSolveReport()
    st = lib.flursys_cuda_stencil_pcg_noalloc(nx, ny, nz, 1 / nx, 1 / ny, 1 / nz, C.c_void_p(dev_rhs.data_ptr()),
                                              C.c_void_p(dev_x.data_ptr()), precision, C.byref(opts), C.byref(rep),
                                              C.c_void_p(stream.cuda_stream))
    assert st == 0
    torch.cuda.synchronize()
    return dev_x.cpu().numpy(), rep


@pytest.mark.parametrize("precision", [_abi.PRECISION_F64, _abi.PRECISION_MIXED])
def test_noalloc_matches_the_allocating_entry_on_two_calls(cudalib, precision):
    opts = _abi.LinearSolverOptions(0.0, 1e-10, 5000)
    rng = np.random.default_rng(11)
    for shape in [(24, 20, 12), (32, 16, 8)]:  # two calls in a row, different systems
        n = shape[0] * shape[1] * shape[2]
        rhs = rng.standard_normal(n)
        rhs[0] = 0.0
        xr, rr = reference_solve(cudalib, shape, rhs, precision, opts)
        xn, rn = noalloc_solve(cudalib, shape, rhs, precision, opts)
        assert rn.status == _abi.LINEAR_CONVERGED
        assert rn.iterations == rr.iterations
        err = np.linalg.norm(xn - xr) / np.linalg.norm(xr)
        assert err <= TOL, f"{shape}: rel L2 {err:.3e}"


def test_noalloc_rejects_grids_beyond_its_limit(cudalib):
    opts = _abi.LinearSolverOptions(0.0, 1e-8, 10)
    rep = _abi.LinearSolveReport()
    st = cudalib.flursys_cuda_stencil_pcg_noalloc(65, 64, 64, 1.0, 1.0, 1.0, C.c_void_p(256), C.c_void_p(256),
                                                  _abi.PRECISION_F64, C.byref(opts), C.byref(rep), None)
    assert st == _abi.ERR_INVALID_ARGUMENT
    buf = C.create_string_buffer(256)
    cudalib.flursys_cuda_global_error(buf, 256)
    assert "262144" in buf.value.decode()
