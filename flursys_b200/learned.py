"""Learned preconditioner of the 3D flexible CG: the network handle, the
solver-generated training data and the training loop.

Every network computation (forward, A-norm loss, backward, Adam) runs in the
library's own kernels (fcgnet.cu) through the C ABI; torch only holds device
buffers. Training data are (divergence, pressure) pairs that the 3D solver
itself produces: cavities of 64^3 and 128^3 cells at Re drawn uniformly from
[100, 1000], started from a random divergence-free velocity field (the
discrete curl of a random vector potential whose sine modes have amplitude
|k|^-2, so the field is exactly discrete-divergence-free and has no normal
flow through the walls), with the pressure of every step solved to 1e-8.

    python -m flursys_b200.learned --out flursys_b200/weights/fcg3d.flnt
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import struct
import time
from dataclasses import dataclass
from typing import List, Optional

import numpy as np

from . import _abi
from .solver import BackendOptions, LidDrivenCavity3DConfig, LidDrivenCavity3DSolver, SolverError, _check

CIN = [1, 16, 32, 64, 64, 32, 16]
COUT = [16, 32, 64, 64, 32, 16, 1]
DEFAULT_WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "weights", "fcg3d.flnt")


def param_count() -> int:
    return int(_abi.load().flursys_cuda_fcgnet_param_count())


def write_weights(path: str, params: np.ndarray) -> None:
    """FLNT file: magic, version 1, layer count, (cin, cout) pairs, count, FP32."""
    p = np.ascontiguousarray(params, dtype="<f4")
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    with open(path, "wb") as f:
        f.write(b"FLNT")
        f.write(struct.pack("<II", 1, len(CIN)))
        for a, b in zip(CIN, COUT):
            f.write(struct.pack("<ii", a, b))
        f.write(struct.pack("<q", p.size))
        f.write(p.tobytes())


def read_weights(path: str) -> np.ndarray:
    with open(path, "rb") as f:
        data = f.read()
    if data[:4] != b"FLNT":
        raise ValueError(f"{path} is not an FLNT weights file")
    off = 12 + 8 * len(CIN)
    (count,) = struct.unpack_from("<q", data, off)
    return np.frombuffer(data, dtype="<f4", count=count, offset=off + 8).astype(np.float32)


def init_params(seed: int = 0) -> np.ndarray:
    """He-style initialisation of every layer (std sqrt(1 / (27 cin)))."""
    rng = np.random.default_rng(seed)
    parts = [rng.standard_normal(27 * a * b) * np.sqrt(1.0 / (27 * a)) for a, b in zip(CIN, COUT)]
    return np.concatenate(parts).astype(np.float32)


class FcgNet:
    """Owns one FlursysFcgNet (the device copy of a parameter set)."""

    def __init__(self, params: Optional[np.ndarray] = None, path: Optional[str] = None):
        self.lib = _abi.load()
        h = C.c_void_p()
        if path is not None:
            _check(self.lib, None, self.lib.flursys_cuda_fcgnet_load(os.fsencode(path), C.byref(h)))
        else:
            ptr = None
            if params is not None:
                arr = np.ascontiguousarray(params, dtype=np.float32)
                if arr.size != param_count():
                    raise ValueError("parameter count does not match the network")
                ptr = arr.ctypes.data_as(C.POINTER(C.c_float))
            _check(self.lib, None, self.lib.flursys_cuda_fcgnet_create(ptr, C.byref(h)))
        self.h = h

    def params(self) -> np.ndarray:
        out = np.empty(param_count(), dtype=np.float32)
        _check(self.lib, None, self.lib.flursys_cuda_fcgnet_get_params(
            self.h, out.ctypes.data_as(C.POINTER(C.c_float)), out.size))
        return out

    def set_params_device(self, params, stream: int = 0) -> None:
        _check(self.lib, None, self.lib.flursys_cuda_fcgnet_set_params(self.h, C.c_void_p(params.data_ptr()),
                                                                       C.c_void_p(stream)))

    def apply(self, r, z, shape, h2: float, stream: int = 0) -> None:
        nx, ny, nz = shape
        _check(self.lib, None, self.lib.flursys_cuda_fcgnet_apply(self.h, nx, ny, nz, h2, C.c_void_p(r.data_ptr()),
                                                                  C.c_void_p(z.data_ptr()), C.c_void_p(stream)))

    def train_sample(self, b_hat, p_hat, norm: float, grad, loss, shape, stream: int = 0,
                     loss_kind: int = _abi.FCG_LOSS_RESIDUAL) -> None:
        nx, ny, nz = shape
        _check(self.lib, None, self.lib.flursys_cuda_fcgnet_train_sample(
            self.h, nx, ny, nz, C.c_void_p(b_hat.data_ptr()), C.c_void_p(p_hat.data_ptr()), float(norm),
            int(loss_kind), C.c_void_p(grad.data_ptr()), C.c_void_p(loss.data_ptr()), C.c_void_p(stream)))

    def solve(self, shape, spacing, rhs: np.ndarray, x0: np.ndarray, rtol: float = 1e-8, atol: float = 0.0,
              max_iterations: int = 2000):
        """flursys_cuda_stencil_fcg on host arrays; returns (x, FcgReport)."""
        nx, ny, nz = shape
        b = np.ascontiguousarray(rhs, dtype=np.float64).ravel()
        x = np.ascontiguousarray(x0, dtype=np.float64).ravel().copy()
        opts = _abi.LinearSolverOptions(atol, rtol, max_iterations)
        rep = _abi.FcgReport()
        _check(self.lib, None, self.lib.flursys_cuda_stencil_fcg(self.h, nx, ny, nz, *spacing, _abi.dptr(b),
                                                                 _abi.dptr(x), C.byref(opts), C.byref(rep)))
        return x, rep

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.flursys_cuda_fcgnet_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# --------------------------------------------------------------------------
# solver-generated data
# --------------------------------------------------------------------------
def solenoidal_field(n: int, seed: int, kmax: int = 6, peak: float = 0.5):
    """u, v, w (MAC faces, x fastest) = discrete curl of a random vector
    potential A_c = sum_k c_k sin(k1 pi x) sin(k2 pi y) sin(k3 pi z),
    c_k ~ N(0, 1) |k|^-2, scaled so that max |velocity| = peak."""
    rng = np.random.default_rng(seed)
    h = 1.0 / n
    k = np.arange(1, kmax + 1)
    kk = np.sqrt(k[:, None, None] ** 2 + k[None, :, None] ** 2 + k[None, None, :] ** 2)
    coef = [rng.standard_normal((kmax, kmax, kmax)) / kk ** 2 for _ in range(3)]
    node = np.arange(n + 1) * h            # x = i h
    mid = (np.arange(n) + 0.5) * h         # x = (i + 1/2) h
    def S(pts):
        t = np.sin(np.pi * np.outer(pts, k))
        t[np.isclose(pts, 0.0) | np.isclose(pts, 1.0)] = 0.0  # exact zeros on the walls
        return t

    def field(c, sx, sy, sz):  # evaluated as [z][y][x]
        return np.einsum("abc,ia,jb,kc->kji", c, sx, sy, sz, optimize=True)

    ax = field(coef[0], S(mid), S(node), S(node))    # x-edges (i+1/2, j, k)
    ay = field(coef[1], S(node), S(mid), S(node))    # y-edges (i, j+1/2, k)
    az = field(coef[2], S(node), S(node), S(mid))    # z-edges (i, j, k+1/2)
    # u at (i, j+1/2, k+1/2): dAz/dy - dAy/dz
    u = (az[:, 1:, :] - az[:, :-1, :]) / h - (ay[1:, :, :] - ay[:-1, :, :]) / h
    # v at (i+1/2, j, k+1/2): dAx/dz - dAz/dx
    v = (ax[1:, :, :] - ax[:-1, :, :]) / h - (az[:, :, 1:] - az[:, :, :-1]) / h
    # w at (i+1/2, j+1/2, k): dAy/dx - dAx/dy
    w = (ay[:, :, 1:] - ay[:, :, :-1]) / h - (ax[:, 1:, :] - ax[:, :-1, :]) / h
    s = peak / max(np.abs(u).max(), np.abs(v).max(), np.abs(w).max())
    return (u * s).ravel(), (v * s).ravel(), (w * s).ravel()


@dataclass
class Pair:
    shape: tuple
    b_hat: object   # torch float32 (cuda): right-hand side, unit RMS
    p_hat: object   # solution of L p_hat = b_hat
    energy_norm: float    # p_hat . b_hat
    residual_norm: float  # b_hat . b_hat


def cavity_config(n: int, reynolds: float, solver: str = "pcg", weights: Optional[str] = None,
                  precision: str = "mixed") -> LidDrivenCavity3DConfig:
    nu = 1.0 / reynolds
    h = 1.0 / n
    dt = min(0.5 * h, 0.25 * h * h / (3.0 * nu))
    return LidDrivenCavity3DConfig(nx=n, ny=n, nz=n, reynolds=reynolds, dt=dt, pressure_solver=solver,
                                   pressure_max_iters=50000,
                                   backend=BackendOptions(precision=precision, stop_rule="rel-l2", pressure_rtol=1e-8,
                                                          fcg_weights_path=weights))


def neumann_laplacian(x: np.ndarray, n: int) -> np.ndarray:
    """Unit-spacing pure-Neumann 7-point operator on an n^3 grid: (L x)_c =
    sum over in-range neighbours of (x_c - x_nb) (h^2 times the matrix of the
    compatible Neumann form of the 3D pressure system)."""
    e = x.reshape(n, n, n)
    q = np.zeros_like(e)
    for ax in range(3):
        d = np.diff(e, axis=ax)
        lo = [slice(None)] * 3
        hi = [slice(None)] * 3
        lo[ax] = slice(0, -1)
        hi[ax] = slice(1, None)
        q[tuple(lo)] -= d
        q[tuple(hi)] += d
    return q.ravel()


def _pcg_iterate(lib, n, rhs, iterations):
    """x_k of the solver's own Jacobi-PCG after `iterations` steps from 0."""
    h = 1.0 / n
    x = np.zeros(n ** 3)
    opts = _abi.LinearSolverOptions(0.0, 0.0, int(iterations))
    rep = _abi.LinearSolveReport()
    _check(lib, None, lib.flursys_cuda_stencil_pcg(n, n, n, h, h, h, _abi.dptr(np.ascontiguousarray(rhs)),
                                                   _abi.dptr(x), _abi.PRECISION_MIXED, C.byref(opts), C.byref(rep)))
    return x


class PairSet(list):
    """Training pairs plus a subset of the pressure systems they came from
    (host arrays (n, b, p) with A p = b), kept for the FCG-iterate pairs."""
    systems: list


def _to_pair(n, b, p, device):
    """Pair of the compatible Neumann form: rows c != 0 of b are kept, row 0
    becomes -sum of the others, the solution loses its mean (constants are
    the null space)."""
    import torch
    b = b.copy()
    b[0] = -b[1:].sum()
    p = p - p.mean()
    s = float(np.sqrt(np.mean(b * b)))
    if s == 0.0:
        return None
    bh, ph = b / s, p / s
    return Pair((n, n, n), torch.from_numpy(bh.astype(np.float32)).to(device),
                torch.from_numpy(ph.astype(np.float32)).to(device), float(np.dot(ph, bh)), float(np.dot(bh, bh)))


def generate_pairs(plan, seed: int, residual_iters=(8, 32, 128), device: str = "cuda", keep_every: int = 5,
                   log=print) -> List[Pair]:
    """plan: [(n, trajectories, steps per trajectory)]. Every step gives the
    pair (divergence, pressure) of its pressure system and, for each k in
    residual_iters, the pair (r_k, p - x_k) of the solver's own Jacobi-PCG
    after k iterations from zero: exact (right-hand side, solution) pairs of
    the same system whose right-hand sides carry the rough residual content
    a preconditioner meets inside CG."""
    lib = _abi.load()
    rng = np.random.default_rng(seed)
    pairs = PairSet()
    pairs.systems = []

    def add(n, b, p):
        pr = _to_pair(n, b, p, device)
        if pr is not None:
            pairs.append(pr)

    for n, ntraj, nsteps in plan:
        h2 = (1.0 / n) ** 2
        for t in range(ntraj):
            re = float(rng.uniform(100.0, 1000.0))
            solver = LidDrivenCavity3DSolver(cavity_config(n, re))
            u, v, w = solenoidal_field(n, int(rng.integers(1 << 31)))
            solver.handle.upload(_abi.FIELD_U, u)
            solver.handle.upload(_abi.FIELD_V, v)
            solver.handle.upload(_abi.FIELD_W, w)
            for step in range(nsteps):
                solver.advance(1)
                rhs = solver.field("rhs")
                rhs[0] = 0.0
                b = -rhs * h2
                p = solver.field("pressure")
                add(n, b, p)
                if step % keep_every == keep_every - 1:
                    pairs.systems.append((n, -rhs, p))
                for k in residual_iters:
                    xk = _pcg_iterate(lib, n, rhs, k)
                    add(n, b - neumann_laplacian(xk, n), p - xk)
            solver.close()
            log(f"  pairs: n={n} trajectory {t + 1}/{ntraj} Re={re:.0f} total={len(pairs)}")
    return pairs


OMEGA = 0.8  # damped-Jacobi weight of the preconditioner's smoothing (fcg3d.cu)


def _diag_unit(n: int) -> np.ndarray:
    """Diagonal of the unit-spacing Neumann operator."""
    i = np.arange(n)
    c = (i > 0).astype(float) + (i < n - 1)
    return (c[None, None, :] + c[None, :, None] + c[:, None, None]).ravel()


def fcg_iterate_pairs(net: "FcgNet", systems, iterations: int = 24, snapshots=(2, 6, 12, 24),
                      device: str = "cuda", max_systems: int = 40) -> List[Pair]:
    """Pairs from the flexible CG's own iterates with the current network:
    at iteration k the preconditioner's network sees r1 = r_k - A z0 (z0 the
    pre-smoothing of r_k), whose exact solution is e_k - z0 with e_k = p - x_k.
    FCG(1) on the compatible Neumann form with the same two-level
    preconditioner as fcg3d.cu, in FP64 on the host around the device
    network."""
    import torch
    out = []
    if len(systems) > max_systems:  # an even spread over the kept systems
        systems = [systems[int(i)] for i in np.linspace(0, len(systems) - 1, max_systems)]
    for n, b, p in systems:
        h2 = (1.0 / n) ** 2
        dA = _diag_unit(n) / h2
        A = lambda v: neumann_laplacian(v, n) / h2  # noqa: E731
        b = b.copy()
        b[0] = -b[1:].sum()
        rt = torch.empty(n ** 3, dtype=torch.float32, device=device)
        zt = torch.empty_like(rt)

        def net_apply(v):
            rt.copy_(torch.from_numpy(v.astype(np.float32)))
            net.apply(rt, zt, (n, n, n), h2)
            return zt.cpu().numpy().astype(np.float64)

        def precondition(r):
            z0 = OMEGA * r / dA
            r1 = r - A(z0)
            z1 = z0 + net_apply(r1)
            z = z1 + OMEGA * (r - A(z1)) / dA
            return z - z.mean()

        x = np.zeros(n ** 3)
        r = b.copy()
        d = q = None
        for k in range(1, iterations + 1):
            z = precondition(r)
            if d is None:
                d = z
            else:
                d = z - (z.dot(q) / d.dot(q)) * d
            q = A(d)
            dq = d.dot(q)
            if not dq > 0.0:
                break
            alpha = d.dot(r) / dq
            x += alpha * d
            r -= alpha * q
            if k in snapshots:
                z0 = OMEGA * r / dA
                r1 = r - A(z0)
                pr = _to_pair(n, h2 * r1, (p - x) - z0, device)
                if pr is not None:
                    out.append(pr)
    return out


def train(pairs: List[Pair], params: np.ndarray, epochs: int, lr: float = 1e-3, batch: int = 8, seed: int = 0,
          loss_kind: int = _abi.FCG_LOSS_RESIDUAL, iterate_rounds=(), iterate_weight: int = 3, log=print) -> dict:
    import torch
    net = FcgNet(params)
    dev = "cuda"
    w = torch.from_numpy(params.astype(np.float32)).to(dev)
    g = torch.zeros_like(w)
    m = torch.zeros_like(w)
    v = torch.zeros_like(w)
    loss = torch.zeros(1, dtype=torch.float64, device=dev)
    net.set_params_device(w)
    rng = np.random.default_rng(seed)
    lib = _abi.load()
    step = 0
    history = []
    total_steps = epochs * ((len(pairs) + batch - 1) // batch) * 2
    t0 = time.time()
    pool = list(pairs)
    weights = [1] * len(pool)
    for ep in range(epochs):
        if ep in iterate_rounds and getattr(pairs, "systems", None):
            t1 = time.time()
            extra = fcg_iterate_pairs(net, pairs.systems)
            pool += extra
            weights += [iterate_weight] * len(extra)
            log(f"  FCG-iterate pairs: +{len(extra)} ({time.time() - t1:.1f} s), pool {len(pool)}")
        order = rng.permutation(np.repeat(np.arange(len(pool)), weights))
        ep_loss = 0.0
        nb = (len(order) + batch - 1) // batch
        for bi in range(nb):
            idx = order[bi * batch:(bi + 1) * batch]
            g.zero_()
            loss.zero_()
            for i in idx:
                pr = pool[i]
                norm = pr.residual_norm if loss_kind == _abi.FCG_LOSS_RESIDUAL else pr.energy_norm
                net.train_sample(pr.b_hat, pr.p_hat, norm, g, loss, pr.shape, loss_kind=loss_kind)
            step += 1
            cur_lr = lr * 0.5 * (1.0 + np.cos(np.pi * min(step / total_steps, 1.0)))  # cosine decay
            _check(lib, None, lib.flursys_cuda_fcgnet_adam(
                C.c_void_p(w.data_ptr()), C.c_void_p(g.data_ptr()), C.c_void_p(m.data_ptr()),
                C.c_void_p(v.data_ptr()), w.numel(), float(cur_lr), 0.9, 0.999, 1e-8, step, 1.0 / len(idx),
                C.c_void_p(0)))
            net.set_params_device(w)
            ep_loss += float(loss.item()) / len(idx)
        history.append(ep_loss / nb)
        log(f"  epoch {ep + 1}/{epochs}: mean loss {history[-1]:.4f} ({time.time() - t0:.1f} s)")
    torch.cuda.synchronize()
    return {"params": w.cpu().numpy(), "loss_history": history, "train_s": time.time() - t0, "adam_steps": step}


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--out", default=DEFAULT_WEIGHTS)
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--traj64", type=int, default=25)
    ap.add_argument("--traj128", type=int, default=15)
    ap.add_argument("--steps", type=int, default=25, help="steps per trajectory (pairs per step: 1 + residual iters)")
    ap.add_argument("--epochs", type=int, default=28)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--batch", type=int, default=8)
    ap.add_argument("--loss", choices=["residual", "energy"], default="residual")
    ap.add_argument("--residual-iters", default="8,32,128",
                    help="Jacobi-PCG iteration counts whose (residual, error) pairs join each step's pair")
    ap.add_argument("--iterate-rounds", default="2,4,8,11,16,21",
                    help="epochs before which pairs from the FCG's own iterates with the current network are added")
    ap.add_argument("--summary", default=None, help="write a JSON summary here")
    ap.add_argument("--init", default=None,
                    help="start from these weights (a .flnt file) instead of a fresh initialisation")
    args = ap.parse_args(argv)
    t0 = time.time()
    plan = [(64, args.traj64, args.steps), (128, args.traj128, args.steps)]
    print(f"generating pairs: {plan}", flush=True)
    ks = tuple(int(k) for k in args.residual_iters.split(",") if k)
    pairs = generate_pairs(plan, args.seed, residual_iters=ks, log=lambda s: print(s, flush=True))
    gen_s = time.time() - t0
    params = read_weights(args.init) if args.init else init_params(args.seed)
    kind = _abi.FCG_LOSS_RESIDUAL if args.loss == "residual" else _abi.FCG_LOSS_ENERGY
    rounds = tuple(int(k) for k in args.iterate_rounds.split(",") if k)
    res = train(pairs, params, args.epochs, lr=args.lr, batch=args.batch, seed=args.seed, loss_kind=kind,
                iterate_rounds=rounds, log=lambda s: print(s, flush=True))
    write_weights(args.out, res["params"])
    summary = {"pairs": len(pairs), "plan": plan, "residual_iters": ks, "loss": args.loss,
               "generate_s": gen_s, "train_s": res["train_s"],
               "adam_steps": res["adam_steps"], "loss_history": res["loss_history"], "out": args.out,
               "seed": args.seed, "epochs": args.epochs, "lr": args.lr, "iterate_rounds": list(rounds),
               "init": args.init}
    print(json.dumps(summary), flush=True)
    if args.summary:
        with open(args.summary, "w") as f:
            json.dump(summary, f, indent=1)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
