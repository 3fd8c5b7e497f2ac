"""ctypes binding of the CPU oracle (liboracle_flursys.so) — TEST INFRASTRUCTURE ONLY.

Used by tests/ as the checker, by __graft_entry__.smoke() and by bench.py's
CPU baseline. The configuration and report types are the C-ABI types of
include/flursys_cuda.h (flursys_b200._abi).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from flursys_b200 import _abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle_flursys.so")
_lib = None

_D = C.POINTER(C.c_double)
_I64P = C.POINTER(C.c_int64)
_P = C.c_void_p


def build(force: bool = False) -> str:
    """Compiles the oracle with the Makefile beside this file."""
    src = os.path.join(HERE, "flursys_oracle.cpp")
    if force or not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < max(
            os.path.getmtime(src), os.path.getmtime(os.path.join(HERE, "flursys_oracle.h"))):
        subprocess.run(["make", "-s", "-B" if force else "-s", "-C", HERE], check=True)
    return LIB_PATH


def load() -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        build()
    lib = C.CDLL(LIB_PATH)
    sig = {
        "orc_set_threads": (None, [C.c_int32]),
        "orc_get_threads": (C.c_int32, []),
        "orc_csr_validate": (C.c_int32, [C.c_int64, C.c_int64, C.c_int64, _I64P, _I64P, _D, C.c_char_p, C.c_size_t]),
        "orc_csr_build": (C.c_int32, [C.c_int64, C.c_int64, C.c_int64, _I64P, _I64P, _D, _I64P, _I64P, _D, _I64P]),
        "orc_csr_spmv": (C.c_int32, [C.c_int64, C.c_int64, C.c_int64, _I64P, _I64P, _D, _D, _D]),
        "orc_jacobi_inverse_diagonal": (C.c_int32, [C.c_int64, C.c_int64, _I64P, _I64P, _D, _D, _I64P]),
        "orc_csr_solve": (C.c_int32, [C.c_int32, C.c_int64, C.c_int64, _I64P, _I64P, _D, _D, _D,
                                      C.POINTER(_abi.LinearSolverOptions), C.POINTER(_abi.LinearSolveReport)]),
        "orc_momentum_stability_numbers": (None, [C.c_double] * 6 + [_D, _D]),
        "orc_adaptive_time_step": (C.c_int32, [C.c_double] * 12 + [_D, C.c_char_p, C.c_size_t]),
        "orc_default_config": (C.c_int32, [C.c_int32, C.POINTER(_abi.CudaConfig)]),
        "orc_create": (C.c_int32, [C.POINTER(_abi.CudaConfig), C.POINTER(_P), C.c_char_p, C.c_size_t]),
        "orc_step": (C.c_int32, [_P, C.c_int64, C.POINTER(_abi.StepReport)]),
        "orc_field_size": (C.c_size_t, [_P, C.c_int32]),
        "orc_get_field": (C.c_int32, [_P, C.c_int32, _D, C.c_size_t]),
        "orc_set_field": (C.c_int32, [_P, C.c_int32, _D, C.c_size_t]),
        "orc_last_error": (C.c_int32, [_P, C.c_char_p, C.c_size_t]),
        "orc_destroy": (None, [_P]),
        "orc_phase_predict": (C.c_int32, [_P, C.c_double]),
        "orc_phase_rhs": (C.c_int32, [_P, C.c_double]),
        "orc_phase_pressure": (C.c_int32, [_P, _D, _I64P]),
        "orc_phase_correct": (C.c_int32, [_P, C.c_double]),
        "orc_max_divergence": (C.c_double, [_P]),
        "orc_pressure_residual": (C.c_double, [_P]),
        "orc_max_speed": (C.c_double, [_P]),
        "orc_stencil_pcg": (C.c_int32, [C.c_int64, C.c_int64, C.c_int64, C.c_double, C.c_double, C.c_double, _D,
                                        _D, C.POINTER(_abi.LinearSolverOptions),
                                        C.POINTER(_abi.LinearSolveReport)]),
        "orc_simple_channel": (C.c_int32, [C.POINTER(_abi.SimpleConfig), _D, _D, _D, _D, _D,
                                           C.POINTER(_abi.SimpleReport)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


class OracleError(RuntimeError):
    def __init__(self, message: str, status: int):
        super().__init__(message)
        self.status = status


def set_threads(n: int) -> None:
    load().orc_set_threads(int(n))


class OracleSolver:
    """One oracle solver (2D IncompressibleSolver or 3D LidDrivenCavity3DSolver)."""

    def __init__(self, cfg: _abi.CudaConfig):
        self.lib = load()
        self.cfg = cfg
        h = C.c_void_p()
        msg = C.create_string_buffer(512)
        st = self.lib.orc_create(C.byref(cfg), C.byref(h), msg, len(msg))
        if st:
            raise OracleError(msg.value.decode(), st)
        self.h = h

    def __del__(self):
        try:
            if self.h:
                self.lib.orc_destroy(self.h)
                self.h = None
        except Exception:
            pass

    def _err(self, st: int) -> None:
        if st:
            msg = C.create_string_buffer(512)
            self.lib.orc_last_error(self.h, msg, len(msg))
            raise OracleError(msg.value.decode(), st)

    def step(self, n: int = 1) -> _abi.StepReport:
        rep = _abi.StepReport()
        self._err(self.lib.orc_step(self.h, n, C.byref(rep)))
        return rep

    def get(self, fid: int) -> np.ndarray:
        n = self.lib.orc_field_size(self.h, fid)
        out = np.empty(n, dtype=np.float64)
        self._err(self.lib.orc_get_field(self.h, fid, _abi.dptr(out), n))
        return out

    def set(self, fid: int, values: np.ndarray) -> None:
        a = np.ascontiguousarray(values, dtype=np.float64).ravel()
        self._err(self.lib.orc_set_field(self.h, fid, _abi.dptr(a), a.size))

    def predict(self, dt: float) -> None:
        self._err(self.lib.orc_phase_predict(self.h, dt))

    def rhs(self, dt: float) -> None:
        self._err(self.lib.orc_phase_rhs(self.h, dt))

    def pressure(self):
        res = C.c_double()
        its = C.c_int64()
        self._err(self.lib.orc_phase_pressure(self.h, C.byref(res), C.byref(its)))
        return res.value, its.value

    def correct(self, dt: float) -> None:
        self._err(self.lib.orc_phase_correct(self.h, dt))

    def max_divergence(self) -> float:
        return self.lib.orc_max_divergence(self.h)

    def pressure_residual(self) -> float:
        return self.lib.orc_pressure_residual(self.h)

    def max_speed(self) -> float:
        return self.lib.orc_max_speed(self.h)


def default_config(dimension: int) -> _abi.CudaConfig:
    cfg = _abi.CudaConfig()
    load().orc_default_config(dimension, C.byref(cfg))
    return cfg


def csr_solve(method: str, row_offsets, columns, values, rhs, x0, options=None):
    """method: "cg" | "pcg" | "bicgstab". Returns (status, x, report)."""
    lib = load()
    ro = np.ascontiguousarray(row_offsets, dtype=np.int64)
    ci = np.ascontiguousarray(columns, dtype=np.int64)
    va = np.ascontiguousarray(values, dtype=np.float64)
    b = np.ascontiguousarray(rhs, dtype=np.float64)
    x = np.array(x0, dtype=np.float64)
    opt = options or _abi.LinearSolverOptions(1e-10, 1e-8, 1000)
    rep = _abi.LinearSolveReport()
    st = lib.orc_csr_solve({"cg": 0, "pcg": 1, "bicgstab": 2}[method], ro.size - 1, va.size, _abi.i64ptr(ro),
                           _abi.i64ptr(ci), _abi.dptr(va), _abi.dptr(b), _abi.dptr(x), C.byref(opt), C.byref(rep))
    return st, x, rep


def csr_build(nrows: int, ncols: int, rows, cols, vals):
    lib = load()
    r = np.ascontiguousarray(rows, dtype=np.int64)
    c = np.ascontiguousarray(cols, dtype=np.int64)
    v = np.ascontiguousarray(vals, dtype=np.float64)
    ro = np.zeros(nrows + 1, dtype=np.int64)
    ci = np.zeros(max(1, r.size), dtype=np.int64)
    va = np.zeros(max(1, r.size), dtype=np.float64)
    nnz = C.c_int64()
    st = lib.orc_csr_build(nrows, ncols, r.size, _abi.i64ptr(r), _abi.i64ptr(c), _abi.dptr(v), _abi.i64ptr(ro),
                           _abi.i64ptr(ci), _abi.dptr(va), C.byref(nnz))
    return st, ro, ci[:nnz.value], va[:nnz.value]


def csr_spmv(row_offsets, columns, values, x, ncols=None):
    lib = load()
    ro = np.ascontiguousarray(row_offsets, dtype=np.int64)
    ci = np.ascontiguousarray(columns, dtype=np.int64)
    va = np.ascontiguousarray(values, dtype=np.float64)
    xx = np.ascontiguousarray(x, dtype=np.float64)
    y = np.zeros(ro.size - 1)
    st = lib.orc_csr_spmv(ro.size - 1, xx.size if ncols is None else ncols, va.size, _abi.i64ptr(ro),
                          _abi.i64ptr(ci), _abi.dptr(va), _abi.dptr(xx), _abi.dptr(y))
    return st, y


def stencil_pcg(nx, ny, nz, dx, dy, dz, rhs, x0, options):
    lib = load()
    b = np.ascontiguousarray(rhs, dtype=np.float64)
    x = np.array(x0, dtype=np.float64)
    rep = _abi.LinearSolveReport()
    st = lib.orc_stencil_pcg(nx, ny, nz, dx, dy, dz, _abi.dptr(b), _abi.dptr(x), C.byref(options), C.byref(rep))
    return st, x, rep


def simple_default_config(nx=64, ny=8, length=8.0, height=1.0, reynolds=200.0, peak=1.0):
    """Channel config with the IncompressibleSolverOptions defaults
    (unstructured_incompressible.rs:38-49); Re on the mean velocity 2/3 peak
    and the height, as project.rs:497-509 defines it."""
    c = _abi.SimpleConfig()
    c.abi_version = _abi.ABI_VERSION
    c.nx, c.ny = nx, ny
    c.length, c.height = length, height
    c.kinematic_viscosity = (2.0 / 3.0) * peak * height / reynolds
    c.inlet_peak_velocity = peak
    c.outlet_pressure = 0.0
    c.max_outer_iterations = 200
    c.continuity_tolerance = 1e-10
    c.velocity_relaxation, c.pressure_relaxation = 0.7, 0.3
    c.momentum_solver = _abi.LinearSolverOptions(1e-10, 1e-8, 1000)
    c.pressure_solver = _abi.LinearSolverOptions(1e-10, 1e-8, 1000)
    return c


def simple_channel(cfg):
    """orc_simple_channel: (status, u, v, p, face_flux, history, report)."""
    lib = load()
    n = cfg.nx * cfg.ny
    u, v, p = np.zeros(n), np.zeros(n), np.zeros(n)
    flux = np.zeros((cfg.nx + 1) * cfg.ny + cfg.nx * (cfg.ny + 1))
    hist = np.zeros(cfg.max_outer_iterations + 1)
    rep = _abi.SimpleReport()
    st = lib.orc_simple_channel(C.byref(cfg), _abi.dptr(u), _abi.dptr(v), _abi.dptr(p), _abi.dptr(flux),
                                _abi.dptr(hist), C.byref(rep))
    return st, u, v, p, flux, hist[:rep.outer_iterations + 1], rep


# ---------------------------------------------------------------------------
# Face-based meshes for the SIMPLE building blocks (test infrastructure)
# ---------------------------------------------------------------------------
class FvMesh:
    """UnstructuredMesh::from_cells (src/mesh.rs:317-423) for 2D polygons:
    faces are the polygons' edges in cell order and edge order, shared edges
    are merged (the first cell owns the face), the area vector is the edge
    (dy, -dx) oriented away from the owner's vertex average, the face centre
    is the edge midpoint, and cell centre and volume are the polygon's
    centroid and area (unit depth)."""

    def __init__(self, points, cells):
        pts = np.asarray(points, dtype=np.float64)
        self.nc = len(cells)
        owner, neigh, area, fc, verts = [], [], [], [], []
        lookup = {}
        cc, vol = [], []
        for c, poly in enumerate(cells):
            ref = pts[poly].mean(axis=0)
            for a, b in zip(poly, poly[1:] + poly[:1]):
                key = tuple(sorted((a, b)))
                if key in lookup:
                    neigh[lookup[key]] = c
                    continue
                e = pts[b] - pts[a]
                s = np.array([e[1], -e[0], 0.0])
                mid = 0.5 * (pts[a] + pts[b])
                if np.dot(s, mid - ref) < 0.0:
                    s = -s
                lookup[key] = len(owner)
                owner.append(c)
                neigh.append(-1)
                area.append(s)
                fc.append(mid)
                verts.append(key)
            # shoelace centroid and area
            x, y = pts[poly, 0], pts[poly, 1]
            x1, y1 = np.roll(x, -1), np.roll(y, -1)
            cr = x * y1 - x1 * y
            a2 = cr.sum()
            vol.append(0.5 * abs(a2))
            cc.append([((x + x1) * cr).sum() / (3.0 * a2), ((y + y1) * cr).sum() / (3.0 * a2), 0.0])
        self.nf = len(owner)
        self.owner = np.array(owner, dtype=np.int64)
        self.neigh = np.array(neigh, dtype=np.int64)
        self.area = np.ascontiguousarray(np.array(area), dtype=np.float64)
        self.fc = np.ascontiguousarray(np.array(fc), dtype=np.float64)
        self.cc = np.ascontiguousarray(np.array(cc), dtype=np.float64)
        self.vol = np.array(vol, dtype=np.float64)

    def args(self):
        return (self.nc, self.nf, _abi.i64ptr(self.owner), _abi.i64ptr(self.neigh), _abi.dptr(self.area),
                _abi.dptr(self.fc), _abi.dptr(self.cc), _abi.dptr(self.vol))

    def boundary_faces(self):
        return np.nonzero(self.neigh < 0)[0]

    def internal_faces(self):
        return np.nonzero(self.neigh >= 0)[0]


def quad_grid(nx, ny, x0=0.0, y0=0.0, dx=1.0, dy=1.0):
    """Cells (x fastest) of an nx x ny grid of axis-aligned quads, as the
    reference's test helpers square_grid / cavity_grid / channel build them
    (points x fastest, polygons counter-clockwise)."""
    pts = [(x0 + i * dx, y0 + j * dy, 0.0) for j in range(ny + 1) for i in range(nx + 1)]
    p = lambda i, j: i + (nx + 1) * j  # noqa: E731
    cells = [[p(i, j), p(i + 1, j), p(i + 1, j + 1), p(i, j + 1)] for j in range(ny) for i in range(nx)]
    return FvMesh(pts, cells)


_FV = [C.c_int64, C.c_int64, _I64P, _I64P, _D, _D, _D, _D]
_I32P = C.POINTER(C.c_int32)


def _fv_sigs(lib):
    sig = {
        "orc_fv_pressure_face_coefficients": _FV + [_D, _I32P, _D, _D],
        "orc_fv_correct_face_flux": _FV + [_D, _D, _D, _I32P, _D, _D],
        "orc_fv_assemble_pressure_correction": _FV + [_D, _D, _I32P, _D, C.c_int64, _I64P, _I64P, _D, C.c_int64,
                                                      _I64P, _D],
        "orc_fv_continuity_rms": _FV + [_D, _D],
        "orc_fv_correct_cell_velocity": [C.c_int64, _D, _D, _D, _D],
        "orc_fv_initial_face_flux": _FV + [_D, _D, _D],
        "orc_fv_assemble_momentum": _FV + [C.c_double, _I32P, _D, _D, _D, _D, C.c_double, _I64P, _I64P, _D,
                                           C.c_int64, _I64P, _D],
        "orc_fv_simple": _FV + [_I32P, _D, _I32P, _D, _I32P, _D, C.c_int64, C.c_double, C.c_double, C.c_double,
                                C.c_int64, C.c_double, C.POINTER(_abi.LinearSolverOptions),
                                C.POINTER(_abi.LinearSolverOptions), _D, _D, _D, _D, C.POINTER(_abi.SimpleReport)],
    }
    for name, args in sig.items():
        fn = getattr(lib, name)
        fn.restype = C.c_int32
        fn.argtypes = args


def _i32(a):
    if a is None:
        return None
    arr = np.ascontiguousarray(a, dtype=np.int32)
    return arr, arr.ctypes.data_as(_I32P)


def _dp(a):
    if a is None:
        return None
    return _abi.dptr(a)


def _bc(mesh, bc):
    """bc: None, or (fixed[nf] of 0/1, value[nf])."""
    if bc is None:
        return None, None, None
    fixed, value = bc
    f = np.ascontiguousarray(fixed, dtype=np.int32)
    v = np.ascontiguousarray(value, dtype=np.float64)
    return (f, v), f.ctypes.data_as(_I32P), _abi.dptr(v)


def fv_pressure_face_coefficients(mesh, rau, pc_bc=None):
    lib = load()
    _fv_sigs(lib)
    rau = np.ascontiguousarray(rau, dtype=np.float64)
    out = np.zeros(mesh.nf)
    keep, f, v = _bc(mesh, pc_bc)
    st = lib.orc_fv_pressure_face_coefficients(*mesh.args(), _abi.dptr(rau), f, v, _abi.dptr(out))
    return st, out


def fv_correct_face_flux(mesh, predicted, coef, correction, pc_bc=None):
    lib = load()
    _fv_sigs(lib)
    a = [np.ascontiguousarray(x, dtype=np.float64) for x in (predicted, coef, correction)]
    out = np.zeros(mesh.nf)
    keep, f, v = _bc(mesh, pc_bc)
    st = lib.orc_fv_correct_face_flux(*mesh.args(), *[_abi.dptr(x) for x in a], f, v, _abi.dptr(out))
    return st, out


def fv_assemble_pressure_correction(mesh, predicted, coef, reference_cell=0, pc_bc=None):
    """Returns (status, row_offsets, columns, values, rhs)."""
    lib = load()
    _fv_sigs(lib)
    a = [np.ascontiguousarray(x, dtype=np.float64) for x in (predicted, coef)]
    cap = 4 * mesh.nf + mesh.nc + 1
    ro = np.zeros(mesh.nc + 1, dtype=np.int64)
    ci = np.zeros(cap, dtype=np.int64)
    va = np.zeros(cap)
    rhs = np.zeros(mesh.nc)
    nnz = C.c_int64()
    keep, f, v = _bc(mesh, pc_bc)
    st = lib.orc_fv_assemble_pressure_correction(*mesh.args(), *[_abi.dptr(x) for x in a], f, v, reference_cell,
                                                 _abi.i64ptr(ro), _abi.i64ptr(ci), _abi.dptr(va), cap,
                                                 C.byref(nnz), _abi.dptr(rhs))
    return st, ro, ci[:nnz.value], va[:nnz.value], rhs


def fv_continuity_rms(mesh, flux):
    lib = load()
    _fv_sigs(lib)
    f = np.ascontiguousarray(flux, dtype=np.float64)
    out = C.c_double()
    st = lib.orc_fv_continuity_rms(*mesh.args(), _abi.dptr(f), C.byref(out))
    return st, out.value


def fv_correct_cell_velocity(predictor, rau, grad):
    lib = load()
    _fv_sigs(lib)
    p = np.ascontiguousarray(predictor, dtype=np.float64)
    r = np.ascontiguousarray(rau, dtype=np.float64)
    g = np.ascontiguousarray(grad, dtype=np.float64)
    out = np.zeros_like(p)
    st = lib.orc_fv_correct_cell_velocity(r.size, _abi.dptr(p), _abi.dptr(r), _abi.dptr(g), _abi.dptr(out))
    return st, out


def fv_initial_face_flux(mesh, velocity, wall_flux):
    lib = load()
    _fv_sigs(lib)
    u = np.ascontiguousarray(velocity, dtype=np.float64)
    w = np.ascontiguousarray(wall_flux, dtype=np.float64)
    out = np.zeros(mesh.nf)
    st = lib.orc_fv_initial_face_flux(*mesh.args(), _abi.dptr(u), _abi.dptr(w), _abi.dptr(out))
    return st, out


def fv_assemble_momentum(mesh, nu, bc, flux, source=None, current=None, alpha=1.0):
    """Returns (status, row_offsets, columns, values, rhs)."""
    lib = load()
    _fv_sigs(lib)
    fl = np.ascontiguousarray(flux, dtype=np.float64)
    src = None if source is None else np.ascontiguousarray(source, dtype=np.float64)
    cur = None if current is None else np.ascontiguousarray(current, dtype=np.float64)
    cap = 4 * mesh.nf + mesh.nc + 1
    ro = np.zeros(mesh.nc + 1, dtype=np.int64)
    ci = np.zeros(cap, dtype=np.int64)
    va = np.zeros(cap)
    rhs = np.zeros(mesh.nc)
    nnz = C.c_int64()
    keep, f, v = _bc(mesh, bc)
    st = lib.orc_fv_assemble_momentum(*mesh.args(), nu, f, v, _abi.dptr(fl), _dp(src), _dp(cur), alpha,
                                      _abi.i64ptr(ro), _abi.i64ptr(ci), _abi.dptr(va), cap, C.byref(nnz),
                                      _abi.dptr(rhs))
    return st, ro, ci[:nnz.value], va[:nnz.value], rhs


def fv_simple(mesh, vel_bc, p_bc, pc_bc=None, reference_cell=0, nu=0.1, velocity_relaxation=0.7,
              pressure_relaxation=0.3, max_outer=200, continuity_tolerance=1e-10,
              momentum_solver=(1e-10, 1e-8, 1000), pressure_solver=(1e-10, 1e-8, 1000), velocity=None,
              pressure=None, face_flux=None):
    """solve_simple on `mesh`. vel_bc = (fixed[nf], value[nf, 3]); p_bc and
    pc_bc = (fixed[nf], value[nf]) or None. Returns (status, velocity[nc, 3],
    pressure, face_flux, history, report)."""
    lib = load()
    _fv_sigs(lib)
    u = np.zeros((mesh.nc, 3)) if velocity is None else np.array(velocity, dtype=np.float64).reshape(mesh.nc, 3)
    u = np.ascontiguousarray(u)
    p = np.zeros(mesh.nc) if pressure is None else np.array(pressure, dtype=np.float64)
    fl = np.zeros(mesh.nf) if face_flux is None else np.array(face_flux, dtype=np.float64)
    hist = np.zeros(max_outer + 1)
    rep = _abi.SimpleReport()
    vf = np.ascontiguousarray(vel_bc[0], dtype=np.int32)
    vv = np.ascontiguousarray(np.asarray(vel_bc[1], dtype=np.float64).reshape(mesh.nf, 3))
    kp, pf, pv = _bc(mesh, p_bc if p_bc is not None else (np.zeros(mesh.nf), np.zeros(mesh.nf)))
    kc, cf, cv = _bc(mesh, pc_bc)
    st = lib.orc_fv_simple(*mesh.args(), vf.ctypes.data_as(_I32P), _abi.dptr(vv), pf, pv, cf, cv, reference_cell,
                           nu, velocity_relaxation, pressure_relaxation, max_outer, continuity_tolerance,
                           C.byref(_abi.LinearSolverOptions(*momentum_solver)),
                           C.byref(_abi.LinearSolverOptions(*pressure_solver)), _abi.dptr(u), _abi.dptr(p),
                           _abi.dptr(fl), _abi.dptr(hist), C.byref(rep))
    return st, u, p, fl, hist[:rep.outer_iterations + 1], rep
