"""Steady collocated SIMPLE channel (src/simple.rs solve_simple through
solve_incompressible): the FP64 oracle restatement on its own, and the device
solver against it."""
import numpy as np
import pytest

from flursys_b200 import _abi

from .paritylib import assert_close


def cfg_small(oracle, nx=64, ny=8, outer=20, tight=True):
    c = oracle.simple_default_config(nx=nx, ny=ny)
    c.max_outer_iterations = outer
    c.continuity_tolerance = 0.0  # run every outer iteration
    if tight:
        c.momentum_solver = _abi.LinearSolverOptions(1e-13, 1e-11, 20000)
        c.pressure_solver = _abi.LinearSolverOptions(1e-13, 1e-11, 20000)
    return c


def test_oracle_channel_approaches_poiseuille(oracle):
    c = cfg_small(oracle, outer=300, tight=False)
    c.momentum_solver.max_iterations = c.pressure_solver.max_iterations = 20000
    st, u, v, p, flux, hist, rep = oracle.simple_channel(c)
    assert st == 0 and rep.outer_iterations == 300
    nx, ny = c.nx, c.ny
    y = (np.arange(ny) + 0.5) / ny
    U = u.reshape(ny, nx)
    assert np.abs(U[:, int(0.75 * nx)] - 4 * y * (1 - y)).max() < 0.02  # developed flow downstream
    assert abs(rep.total_inflow + rep.total_outflow) < 1e-8             # global mass balance
    assert hist[-1] < 1e-9


def test_oracle_continuity_rule_stops_after_the_first_correction(oracle):
    # the continuity RMS is enforced by the pressure correction itself, so the
    # reference's stop rule is met as soon as one correction has been applied
    c = cfg_small(oracle, outer=50, tight=False)
    c.continuity_tolerance = 1e-7
    st, u, v, p, flux, hist, rep = oracle.simple_channel(c)
    assert st == 0 and rep.converged and rep.outer_iterations == 1


def test_channel_rejects_bad_configs(cudalib):
    import ctypes as C
    c = _abi.SimpleConfig()
    assert cudalib.flursys_cuda_simple_default_config(C.byref(c)) == 0
    assert (c.nx, c.ny, c.velocity_relaxation, c.pressure_relaxation) == (2048, 512, 0.7, 0.3)
    for field, value in [("nx", 1), ("pressure_relaxation", 0.0), ("max_outer_iterations", 0)]:
        bad = _abi.SimpleConfig()
        C.pointer(bad)[0] = c
        setattr(bad, field, value)
        rep = _abi.SimpleReport()
        st = cudalib.flursys_cuda_simple_channel(C.byref(bad), None, None, None, None, None, C.byref(rep))
        assert st == _abi.ERR_INVALID_CONFIG, field


@pytest.mark.gpu
@pytest.mark.parametrize("nx,ny,outer", [(64, 8, 20), (40, 16, 12)])
def test_device_channel_matches_oracle(oracle, nx, ny, outer):
    from flursys_b200.solver import solve_simple_channel
    c = cfg_small(oracle, nx=nx, ny=ny, outer=outer)
    st, u, v, p, flux, hist, rep = oracle.simple_channel(c)
    assert st == 0
    out = solve_simple_channel(c)
    r = out["report"]
    assert r.outer_iterations == rep.outer_iterations == outer
    for name, a, b in [("u", out["u"], u), ("v", out["v"], v), ("p", out["p"], p), ("flux", out["flux"], flux)]:
        assert_close(a, b, 1e-9, name)
    assert np.allclose(out["history"][1:], hist[1:], rtol=1e-3, atol=1e-13)
    assert abs(r.total_inflow - rep.total_inflow) < 1e-12


@pytest.mark.gpu
def test_device_channel_reference_options_and_stop_rule(oracle):
    # default linear options (atol 1e-10, rtol 1e-8, 1000 iterations) and the
    # continuity stop rule: both stop at the same outer iteration
    from flursys_b200.solver import solve_simple_channel
    c = oracle.simple_default_config(nx=64, ny=16)
    c.continuity_tolerance = 1e-7
    st, u, v, p, flux, hist, rep = oracle.simple_channel(c)
    out = solve_simple_channel(c)
    assert st == 0 and out["report"].converged == rep.converged == 1
    assert out["report"].outer_iterations == rep.outer_iterations
    assert_close(out["u"], u, 1e-6, "u")
