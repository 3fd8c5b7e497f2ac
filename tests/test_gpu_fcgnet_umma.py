"""The learned preconditioner's convolutions on the 5th-generation tensor
cores (tcgen05.mma with the accumulator in tensor memory; the default,
FLURSYS_FCG_UMMA=0 selects mma.sync) against the mma.sync kernels and the
numpy oracle of the network, and inside the flexible CG."""
import os

import numpy as np
import pytest

from oracle import fcgnet_oracle as fo

from .test_fcgnet import _cavity_system, _weights_or_skip, rel_l2, small_params

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _apply(params, r, shape, h2, umma, monkeypatch):
    from flursys_b200.learned import FcgNet
    monkeypatch.setenv("FLURSYS_FCG_UMMA", "1" if umma else "0")
    net = FcgNet(params)
    rt = torch.tensor(r.ravel(), dtype=torch.float32, device="cuda")
    zt = torch.empty_like(rt)
    net.apply(rt, zt, shape, h2)
    torch.cuda.synchronize()
    monkeypatch.delenv("FLURSYS_FCG_UMMA")
    return zt.cpu().numpy()


@pytest.mark.parametrize("shape", [(16, 16, 16), (48, 32, 40), (64, 64, 64)])
def test_umma_forward_matches_mma_sync_and_oracle(monkeypatch, shape):
    params = small_params(21).astype(np.float32)
    rng = np.random.default_rng(22)
    nx, ny, nz = shape
    r = rng.standard_normal((nz, ny, nx)) * 1e-4
    h2 = (1.0 / nx) ** 2
    z_umma = _apply(params, r, shape, h2, True, monkeypatch)
    z_mma = _apply(params, r, shape, h2, False, monkeypatch)
    assert np.all(np.isfinite(z_umma))
    # same BF16 operands, FP32 accumulation in another order: BF16 rounding
    # of the layer outputs differs in the last place at most
    assert rel_l2(z_umma, z_mma) < 5e-3
    if nx * ny * nz <= 48 * 32 * 40:
        z_ref = fo.apply(params.astype(np.float64), r.astype(np.float32).astype(np.float64), h2)
        assert rel_l2(z_umma, z_ref) < 2e-2


def test_umma_fcg_solve_matches_mma_sync(monkeypatch):
    from flursys_b200 import _abi
    from flursys_b200.learned import FcgNet
    w = _weights_or_skip()
    n = 64
    h = 1.0 / n
    rhs, _ = _cavity_system(n)
    out = {}
    for umma in (True, False):
        monkeypatch.setenv("FLURSYS_FCG_UMMA", "1" if umma else "0")
        net = FcgNet(path=w)
        x, rep = net.solve((n, n, n), (h, h, h), rhs, np.zeros(n ** 3), rtol=1e-8, max_iterations=1000)
        assert rep.status == _abi.LINEAR_CONVERGED and rep.fallback == 0 and rep.relative_residual <= 1e-8
        out[umma] = (x, rep.fcg_iterations)
    monkeypatch.delenv("FLURSYS_FCG_UMMA")
    assert abs(out[True][1] - out[False][1]) <= max(2, out[False][1] // 10)
    assert rel_l2(out[True][0], out[False][0]) < 1e-6
