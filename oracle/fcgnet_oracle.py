"""CPU restatement (numpy, FP64) of the learned FCG preconditioner network:
forward, A-norm loss and backward, for checking the device kernels.

TEST INFRASTRUCTURE ONLY: imported by tests/ as the checker of
flursys_cuda_fcgnet_apply / flursys_cuda_fcgnet_train_sample; nothing in the
flursys_b200 package uses it.

The network has no reference counterpart (the reference solves the pressure
system with SOR and Jacobi-PCG only). The oracle mirrors the device
arithmetic's rounding points: weights of the tensor-core layers and every
stored activation and activation gradient are rounded to BF16
(round-to-nearest-even), the two CUDA-core layers use FP32 weights. Sums are
FP64 here and FP32 on the device, so the two agree to BF16 rounding flips.

Layout: arrays are (nz, ny, nx, C), x fastest then channels innermost in
memory, as on the device. Parameters: layer after layer, W[co][tap][ci] with
tap = 9 (dz+1) + 3 (dy+1) + (dx+1).
"""
from __future__ import annotations

import numpy as np

CIN = [1, 16, 32, 64, 64, 32, 16]
COUT = [16, 32, 64, 64, 32, 16, 1]


def param_count() -> int:
    return sum(27 * a * b for a, b in zip(CIN, COUT))


def split(params: np.ndarray):
    out, off = [], 0
    for a, b in zip(CIN, COUT):
        n = 27 * a * b
        out.append(np.asarray(params[off:off + n], dtype=np.float64).reshape(b, 27, a))
        off += n
    return out


def bf16(x):
    """Round to BF16 (nearest, ties to even) and back to float64."""
    a = np.ascontiguousarray(np.asarray(x, dtype=np.float32))
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def taps():
    for t in range(27):
        yield t, t // 9 - 1, (t // 3) % 3 - 1, t % 3 - 1


def conv(x, w):
    """Zero-padded 3x3x3 correlation: x (nz,ny,nx,ci), w (co,27,ci)."""
    nz, ny, nx, _ = x.shape
    xp = np.pad(x, ((1, 1), (1, 1), (1, 1), (0, 0)))
    out = np.zeros((nz, ny, nx, w.shape[0]))
    for t, dz, dy, dx in taps():
        out += xp[1 + dz:1 + dz + nz, 1 + dy:1 + dy + ny, 1 + dx:1 + dx + nx, :] @ w[:, t, :].T
    return out


def conv_t(g, w):
    """Transpose of conv with respect to its input: g (nz,ny,nx,co) -> (.., ci)."""
    wt = w[:, ::-1, :].transpose(2, 1, 0)  # [ci][26 - tap][co]
    return conv(g, wt)


def wgrad(x, g):
    """dW[co][tap][ci] = sum_v g[v][co] x[v + tap][ci]."""
    nz, ny, nx, ci = x.shape
    xp = np.pad(x, ((1, 1), (1, 1), (1, 1), (0, 0)))
    dw = np.zeros((g.shape[3], 27, ci))
    gf = g.reshape(-1, g.shape[3])
    for t, dz, dy, dx in taps():
        xs = xp[1 + dz:1 + dz + nz, 1 + dy:1 + dy + ny, 1 + dx:1 + dx + nx, :].reshape(-1, ci)
        dw[:, t, :] = gf.T @ xs
    return dw


def pool(x):
    nz, ny, nx, c = x.shape
    return x.reshape(nz // 2, 2, ny // 2, 2, nx // 2, 2, c).mean(axis=(1, 3, 5))


def sumpool(x):
    nz, ny, nx, c = x.shape
    return x.reshape(nz // 2, 2, ny // 2, 2, nx // 2, 2, c).sum(axis=(1, 3, 5))


def up(x):
    return x.repeat(2, axis=0).repeat(2, axis=1).repeat(2, axis=2)


def lap_neumann(e):
    """Unit-spacing pure-Neumann 7-point operator: (L e)_c = sum over in-range
    neighbours of (e_c - e_nb). e is (nz,ny,nx)."""
    q = np.zeros_like(e)
    for ax in range(3):
        d = np.diff(e, axis=ax)
        sl_lo = [slice(None)] * 3
        sl_hi = [slice(None)] * 3
        sl_lo[ax] = slice(0, -1)
        sl_hi[ax] = slice(1, None)
        q[tuple(sl_lo)] -= d
        q[tuple(sl_hi)] += d
    return q


def _identity(x):
    return np.asarray(x, dtype=np.float64)


def forward(params, b, rounding=True):
    """Network output and the stored activations; b is (nz,ny,nx) already
    normalised. Mirrors net_train_sample's forward; rounding=False gives the
    exact FP64 network (for finite-difference checks of the oracle)."""
    bf16 = globals()["bf16"] if rounding else _identity
    W = split(params)
    Wt = [W[0]] + [bf16(w) for w in W[1:6]] + [W[6]]
    s = {}
    s["a1"] = bf16(conv(b[..., None], Wt[0]))
    s["x2"] = bf16(pool(s["a1"]))
    s["a2"] = bf16(conv(s["x2"], Wt[1]))
    s["x3"] = bf16(pool(s["a2"]))
    s["a3"] = bf16(conv(s["x3"], Wt[2]))
    s["x4"] = bf16(pool(s["a3"]))
    s["a4"] = bf16(conv(s["x4"], Wt[3]))
    s["x5"] = bf16(up(s["a4"]) + s["a3"])
    s["b3"] = bf16(conv(s["x5"], Wt[4]))
    s["x6"] = bf16(up(s["b3"]) + s["a2"])
    s["b2"] = bf16(conv(s["x6"], Wt[5]))
    s["x7"] = bf16(up(s["b2"]) + s["a1"])
    out = conv(s["x7"], Wt[6])[..., 0]
    return out, s, Wt


def apply(params, r, h2):
    """z = N(r) as flursys_cuda_fcgnet_apply computes it (input normalised to
    unit RMS, output scaled by h2 / scale)."""
    rms = np.sqrt(np.mean(r * r))
    scale = 0.0 if rms == 0.0 else 1.0 / rms
    out, _, _ = forward(params, r * scale)
    return out * (h2 / scale if scale > 0 else 0.0)


def loss_and_grad(params, b_hat, p_hat, norm, rounding=True, loss="energy"):
    """Loss and dLoss/dparams for e = net(b_hat) - p_hat on the Neumann
    operator: "energy" (e.L e)/norm or "residual" |L e|^2/norm."""
    bf16 = globals()["bf16"] if rounding else _identity
    out, s, Wt = forward(params, b_hat, rounding=rounding)
    e = np.asarray(out - p_hat, dtype=np.float32).astype(np.float64) if rounding else out - p_hat
    q = lap_neumann(e)
    if loss == "energy":
        value = float(np.sum(e * q) / norm)
        gout = 2.0 * q / norm
    else:
        value = float(np.sum(q * q) / norm)
        gout = 2.0 * lap_neumann(q) / norm
    loss = value
    grads = [None] * 7
    grads[6] = wgrad(s["x7"], gout[..., None])
    g7 = bf16(conv_t(gout[..., None], Wt[6]))
    gb2 = bf16(sumpool(g7))
    grads[5] = wgrad(s["x6"], gb2)
    g6 = bf16(conv_t(gb2, Wt[5]))
    gb3 = bf16(sumpool(g6))
    grads[4] = wgrad(s["x5"], gb3)
    g5 = bf16(conv_t(gb3, Wt[4]))
    ga4 = bf16(sumpool(g5))
    grads[3] = wgrad(s["x4"], ga4)
    g4 = bf16(conv_t(ga4, Wt[3]))
    ga3 = bf16(g5 + 0.125 * up(g4))
    grads[2] = wgrad(s["x3"], ga3)
    g3 = bf16(conv_t(ga3, Wt[2]))
    ga2 = bf16(g6 + 0.125 * up(g3))
    grads[1] = wgrad(s["x2"], ga2)
    g2 = bf16(conv_t(ga2, Wt[1]))
    ga1 = bf16(g7 + 0.125 * up(g2))
    grads[0] = wgrad(b_hat[..., None], ga1)
    return loss, np.concatenate([g.ravel() for g in grads])
