"""Helpers shared by the GPU parity tests."""
import numpy as np


def rel_l2(a, b):
    nb = float(np.linalg.norm(b))
    return float(np.linalg.norm(a - b)) / (nb if nb > 0 else 1.0)


def rel_max(a, b):
    mb = float(np.max(np.abs(b))) if b.size else 0.0
    return float(np.max(np.abs(a - b))) / (mb if mb > 0 else 1.0)


def assert_close(a, b, tol, what=""):
    l2, mx = rel_l2(a, b), rel_max(a, b)
    assert l2 <= tol and mx <= tol, f"{what}: rel L2 {l2:.3e}, rel max {mx:.3e} > {tol:.1e}"
    return l2, mx
