"""Learned FCG preconditioner: the numpy oracle of the network against finite
differences, the solver-data generator's field, and (GPU) the device
forward/backward kernels and the flexible CG against the oracle and the
plain PCG."""
import ctypes as C
import os

import numpy as np
import pytest

from oracle import fcgnet_oracle as fo


def small_params(seed, scale=1.0):
    rng = np.random.default_rng(seed)
    parts = [rng.standard_normal(27 * a * b) * np.sqrt(scale / (27 * a)) for a, b in zip(fo.CIN, fo.COUT)]
    return np.concatenate(parts)


def poisson_pair(n, seed):
    """(b_hat, p_hat, norm) with L p_hat = b_hat on the unit Neumann operator."""
    rng = np.random.default_rng(seed)
    p = rng.standard_normal((n, n, n))
    p -= p.mean()
    b = fo.lap_neumann(p)
    return b, p, float(np.sum(p * b))


@pytest.mark.parametrize("kind", ["energy", "residual"])
def test_oracle_gradient_matches_finite_differences(kind):
    n = 8
    params = small_params(1)
    b, p, norm = poisson_pair(n, 2)
    if kind == "residual":
        norm = float(np.sum(b * b))
    loss, grad = fo.loss_and_grad(params, b, p, norm, rounding=False, loss=kind)
    rng = np.random.default_rng(3)
    offs = np.cumsum([0] + [27 * a * c for a, c in zip(fo.CIN, fo.COUT)])
    for layer in range(7):
        for _ in range(3):
            k = int(rng.integers(offs[layer], offs[layer + 1]))
            eps = 1e-2  # the loss is quadratic in each parameter: central differences are exact
            pp = params.copy(); pp[k] += eps
            pm = params.copy(); pm[k] -= eps
            lp, _ = fo.loss_and_grad(pp, b, p, norm, rounding=False, loss=kind)
            lm, _ = fo.loss_and_grad(pm, b, p, norm, rounding=False, loss=kind)
            fd = (lp - lm) / (2 * eps)
            assert abs(fd - grad[k]) <= 1e-6 * max(1.0, abs(fd)), (layer, k, fd, grad[k])


def test_solenoidal_field_is_discretely_divergence_free():
    from flursys_b200.learned import solenoidal_field
    n = 16
    u, v, w = solenoidal_field(n, seed=5)
    U = u.reshape(n, n, n + 1)
    V = v.reshape(n, n + 1, n)
    W = w.reshape(n + 1, n, n)
    div = (U[:, :, 1:] - U[:, :, :-1]) + (V[:, 1:, :] - V[:, :-1, :]) + (W[1:] - W[:-1])
    assert np.abs(div).max() <= 1e-12 * np.abs(U).max() * n
    # no normal flow through the walls
    assert np.abs(U[:, :, 0]).max() == 0.0 and np.abs(U[:, :, -1]).max() == 0.0
    assert np.abs(V[:, 0, :]).max() == 0.0 and np.abs(W[0]).max() == 0.0
    assert abs(max(np.abs(U).max(), np.abs(V).max(), np.abs(W).max()) - 0.5) < 1e-12


def test_weights_file_round_trip(tmp_path):
    from flursys_b200 import learned
    p = np.arange(fo.param_count(), dtype=np.float32) * 1e-3
    path = str(tmp_path / "w.flnt")
    learned.write_weights(path, p)
    np.testing.assert_array_equal(learned.read_weights(path), p)


# ---------------------------------------------------------------- GPU ----
torch = pytest.importorskip("torch")


def rel_l2(a, b):
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b)) / max(np.linalg.norm(np.ravel(b)), 1e-300))


@pytest.mark.gpu
def test_net_apply_matches_oracle():
    from flursys_b200.learned import FcgNet
    n = 16
    params = small_params(7).astype(np.float32)
    rng = np.random.default_rng(8)
    r = rng.standard_normal((n, n, n)) * 1e-5
    h2 = (1.0 / n) ** 2
    net = FcgNet(params)
    rt = torch.tensor(r.ravel(), dtype=torch.float32, device="cuda")
    zt = torch.empty_like(rt)
    net.apply(rt, zt, (n, n, n), h2)
    torch.cuda.synchronize()
    z_ref = fo.apply(params.astype(np.float64), r.astype(np.float32).astype(np.float64), h2)
    assert rel_l2(zt.cpu().numpy(), z_ref) < 2e-2


@pytest.mark.gpu
@pytest.mark.parametrize("dims", [(64, 64, 64), (48, 40, 32)])
def test_tma_staged_convolutions_equal_register_staged(dims, monkeypatch):
    """The tcgen05 convolutions give the same bits whether their input planes
    arrive by TMA copies (halo zero-filled by the copy engine) or by
    register-staged loads with bounds checks."""
    monkeypatch.setenv("FLURSYS_FCG_PAIR", "0")
    out = {}
    for tma in ("0", "1"):
        monkeypatch.setenv("FLURSYS_FCG_TMA", tma)
        out[tma] = _apply_default_net(dims)
    assert np.isfinite(out["1"]).all()
    assert np.array_equal(out["0"], out["1"])


def _apply_default_net(dims):
    from flursys_b200.learned import DEFAULT_WEIGHTS, FcgNet
    net = FcgNet(path=DEFAULT_WEIGHTS)
    n = int(np.prod(dims))
    rt = torch.tensor(np.random.default_rng(3).standard_normal(n), dtype=torch.float32, device="cuda")
    zt = torch.empty_like(rt)
    net.apply(rt, zt, dims, 1.0 / dims[0] ** 2)
    torch.cuda.synchronize()
    return zt.cpu().numpy()


@pytest.mark.gpu
@pytest.mark.parametrize("dims", [(64, 64, 64), (48, 40, 32)])
def test_paired_plane_convolutions_match_single_plane(dims, monkeypatch):
    """Output planes computed in pairs (one MMA of N = 2 Cout per input plane)
    agree with the one-plane kernel up to the FP32 summation order inside the
    tensor cores, i.e. BF16 roundings of the activations."""
    out = {}
    for pair in ("0", "1"):
        monkeypatch.setenv("FLURSYS_FCG_PAIR", pair)
        out[pair] = _apply_default_net(dims)
    assert np.isfinite(out["1"]).all()
    assert rel_l2(out["1"], out["0"]) < 1e-2


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["energy", "residual"])
def test_net_gradients_match_oracle(kind):
    from flursys_b200 import _abi
    from flursys_b200.learned import FcgNet
    n = 16
    params = small_params(11).astype(np.float32)
    b, p, norm = poisson_pair(n, 12)
    b = b.astype(np.float32).astype(np.float64)
    p = p.astype(np.float32).astype(np.float64)
    if kind == "residual":
        norm = float(np.sum(b * b))
    net = FcgNet(params)
    bt = torch.tensor(b.ravel(), dtype=torch.float32, device="cuda")
    pt = torch.tensor(p.ravel(), dtype=torch.float32, device="cuda")
    g = torch.zeros(fo.param_count(), dtype=torch.float32, device="cuda")
    loss = torch.zeros(1, dtype=torch.float64, device="cuda")
    net.train_sample(bt, pt, norm, g, loss, (n, n, n),
                     loss_kind=_abi.FCG_LOSS_ENERGY if kind == "energy" else _abi.FCG_LOSS_RESIDUAL)
    torch.cuda.synchronize()
    l_ref, g_ref = fo.loss_and_grad(params.astype(np.float64), b, p, norm, loss=kind)
    assert abs(loss.item() - l_ref) <= 1e-2 * abs(l_ref)
    gd = g.cpu().numpy()
    offs = np.cumsum([0] + [27 * a * c for a, c in zip(fo.CIN, fo.COUT)])
    for layer in range(7):
        sl = slice(offs[layer], offs[layer + 1])
        assert rel_l2(gd[sl], g_ref[sl]) < 3e-2, (layer, rel_l2(gd[sl], g_ref[sl]))


def _weights_or_skip():
    from flursys_b200.learned import DEFAULT_WEIGHTS
    if not os.path.exists(DEFAULT_WEIGHTS):
        pytest.skip("no trained weights file")
    return DEFAULT_WEIGHTS


@pytest.mark.gpu
def test_fcg_falls_back_to_jacobi_pcg_when_the_network_is_zero(oracle, monkeypatch):
    # without the smoothing passes a zero network gives z = 0: the first
    # direction breaks down and the Jacobi-PCG fallback must finish the solve
    # to the same tolerance
    monkeypatch.setenv("FLURSYS_FCG_SMOOTH", "0")
    from flursys_b200 import _abi
    from flursys_b200.learned import FcgNet
    n = 16
    h = 1.0 / n
    rng = np.random.default_rng(4)
    rhs = rng.standard_normal(n ** 3)
    rhs[0] = 0.0
    net = FcgNet(np.zeros(fo.param_count(), np.float32))
    x, rep = net.solve((n, n, n), (h, h, h), rhs, np.zeros(n ** 3), rtol=1e-10, max_iterations=100)
    assert rep.fallback == 1 and rep.status == _abi.LINEAR_CONVERGED
    assert rep.relative_residual <= 1e-10
    opts = _abi.LinearSolverOptions(0.0, 1e-12, 20000)
    st, x_ref, _ = oracle.stencil_pcg(n, n, n, h, h, h, rhs, np.zeros(n ** 3), opts)
    assert st == 0
    assert rel_l2(x, x_ref) < 1e-8


def _cavity_system(n, steps=3):
    from flursys_b200.learned import cavity_config
    from flursys_b200.solver import LidDrivenCavity3DSolver
    s = LidDrivenCavity3DSolver(cavity_config(n, 400.0))
    s.advance(steps)
    rhs, p = s.field("rhs"), s.field("pressure")
    s.close()
    return rhs, p


@pytest.mark.gpu
def test_trained_fcg_needs_fewer_iterations_than_jacobi_pcg(cudalib):
    # the ablation: the same flexible CG without the network is Jacobi-PCG
    from flursys_b200 import _abi
    from flursys_b200.learned import FcgNet
    w = _weights_or_skip()
    n = 64
    h = 1.0 / n
    rhs, _ = _cavity_system(n)
    net = FcgNet(path=w)
    x, rep = net.solve((n, n, n), (h, h, h), rhs, np.zeros(n ** 3), rtol=1e-8, max_iterations=1000)
    assert rep.status == _abi.LINEAR_CONVERGED and rep.fallback == 0
    assert rep.relative_residual <= 1e-8
    xp = np.zeros(n ** 3)
    opts = _abi.LinearSolverOptions(0.0, 1e-8, 20000)
    prep = _abi.LinearSolveReport()
    assert cudalib.flursys_cuda_stencil_pcg(n, n, n, h, h, h, _abi.dptr(np.ascontiguousarray(rhs)), _abi.dptr(xp),
                                            _abi.PRECISION_F64, C.byref(opts), C.byref(prep)) == 0
    assert rep.fcg_iterations * 3 <= prep.iterations, (rep.fcg_iterations, prep.iterations)
    assert rel_l2(x, xp) < 1e-6


@pytest.mark.gpu
def test_fcg_cavity_steps_match_f64_oracle(oracle):
    from flursys_b200 import _abi
    from flursys_b200.solver import _Handle
    w = _weights_or_skip()
    from .test_gpu_cavity3d import cfg3d
    cfg = cfg3d(oracle, 32, 32, 32, rtol=1e-8, precision=_abi.PRECISION_MIXED)
    cfg.pressure_solver = _abi.PRESSURE_FCG
    cfg.fcg_weights_path = os.fsencode(w)
    gpu = _Handle(cfg)
    ref_cfg = cfg3d(oracle, 32, 32, 32, rtol=1e-12)
    ref = oracle.OracleSolver(ref_cfg)
    for _ in range(4):
        r = gpu.step(1)
        ref.step(1)
        assert r.pressure_true_relative_residual <= 1e-8 * 1.01
    for fid in (_abi.FIELD_U, _abi.FIELD_V, _abi.FIELD_W):
        assert rel_l2(gpu.download(fid), ref.get(fid)) < 1e-6


@pytest.mark.gpu
@pytest.mark.parametrize("n", [64, 128])
def test_fcg_steps_from_rest_converge_without_fallback(oracle, n):
    # the first steps from rest start from residuals 1e8 above the stop
    # threshold: the FP32 recurrence must be replaced by the FP64 residual as
    # it falls (reliable updates), or it stalls at its rounding floor and the
    # step ends in the Jacobi-PCG fallback
    from flursys_b200 import _abi
    from flursys_b200.solver import _Handle
    w = _weights_or_skip()
    from .test_gpu_cavity3d import cfg3d
    cfg = cfg3d(oracle, n, n, n, rtol=1e-8, precision=_abi.PRECISION_MIXED)
    cfg.pressure_solver = _abi.PRESSURE_FCG
    cfg.fcg_weights_path = os.fsencode(w)
    gpu = _Handle(cfg)
    for _ in range(4):
        r = gpu.step(1)
        assert r.pressure_status == _abi.LINEAR_CONVERGED
        assert r.fcg_fallback == 0
        assert r.pressure_true_relative_residual <= 1e-8 * 1.01
