"""Pins the oracle's restatement of the collocated SIMPLE path to the
reference's own tests of it, on the reference's own test meshes:
src/simple.rs:989-1260 (two-cell hand calculations: rAU face coefficient,
flux correction, pressure-correction matrix and signs, velocity-correction
sign, continuity RMS, initial face flux, closed two-cell cases),
src/simple.rs:1406-1532 (closed cavities without wall leakage, orthogonal
and skewed), tests/unstructured_incompressible.rs:345-388 (velocity-inlet /
pressure-outlet channel mass balance) and src/momentum.rs:718-764,888-965
(upwind coefficients, Couette and Poiseuille profiles). The meshes are built
as UnstructuredMesh::from_cells builds them (oracle.binding.FvMesh)."""
import numpy as np
import pytest


def two_cells(ob):
    """simple.rs:817-846: two unit squares side by side."""
    pts = [(0, 0, 0), (1, 0, 0), (2, 0, 0), (0, 1, 0), (1, 1, 0), (2, 1, 0)]
    return ob.FvMesh(pts, [[0, 1, 4, 3], [1, 2, 5, 4]])


def on_internal(mesh, value):
    return np.where(mesh.neigh >= 0, value, 0.0)


def csr_get(ro, ci, va, r, c):
    for k in range(ro[r], ro[r + 1]):
        if ci[k] == c:
            return va[k]
    return None


def test_pressure_face_coefficient_two_cell(oracle):
    m = two_cells(oracle)
    st, coef = oracle.fv_pressure_face_coefficients(m, [0.5, 1.5])
    assert st == 0
    f = m.internal_faces()[0]
    assert coef[f] == 1.0  # rAU_f = (0.5 + 1.5) / 2, |S| = |d| = 1
    assert all(coef[g] == 0.0 for g in range(m.nf) if g != f)


def test_pressure_flux_correction_two_cell(oracle):
    m = two_cells(oracle)
    st, out = oracle.fv_correct_face_flux(m, on_internal(m, 3.0), on_internal(m, 2.0), [0.0, 1.5])
    assert st == 0
    assert np.all(out == 0.0)  # 3 - 2 * 1.5 = 0 on the internal face, walls untouched


def test_pressure_correction_two_cell_matrix_rhs_and_signs(oracle):
    m = two_cells(oracle)
    st, ro, ci, va, rhs = oracle.fv_assemble_pressure_correction(m, on_internal(m, 3.0), on_internal(m, 2.0), 0)
    assert st == 0
    assert csr_get(ro, ci, va, 0, 0) == 1.0
    assert csr_get(ro, ci, va, 0, 1) is None and csr_get(ro, ci, va, 1, 0) is None
    assert csr_get(ro, ci, va, 1, 1) == 2.0
    assert list(rhs) == [0.0, 3.0]  # A p' = -div(Phi*), reference row 0 eliminated


def test_pressure_correction_solve_removes_the_two_cell_imbalance(oracle):
    from flursys_b200 import _abi
    m = two_cells(oracle)
    pred, coef = on_internal(m, 3.0), on_internal(m, 2.0)
    st, ro, ci, va, rhs = oracle.fv_assemble_pressure_correction(m, pred, coef, 0)
    st, x, rep = oracle.csr_solve("pcg", ro, ci, va, rhs, np.zeros(2), _abi.LinearSolverOptions(1e-14, 1e-14, 20))
    assert st == 0 and rep.status == _abi.LINEAR_CONVERGED
    assert list(x) == [0.0, 1.5]
    st, corrected = oracle.fv_correct_face_flux(m, pred, coef, x)
    st, rms = oracle.fv_continuity_rms(m, corrected)
    assert st == 0 and rms < 1e-12
    st, ax = oracle.csr_spmv(ro, ci, va, x)
    assert np.all(np.abs(rhs - ax) < 1e-12)


def test_velocity_pressure_correction_has_the_negative_gradient_sign(oracle):
    st, out = oracle.fv_correct_cell_velocity([[4.0, -1.0, 2.0], [1.0, 3.0, -2.0]], [0.5, 2.0],
                                              [[2.0, -4.0, 1.0], [-1.0, 0.5, 3.0]])
    assert st == 0
    assert out.tolist() == [[3.0, 1.0, 1.5], [3.0, 2.0, -8.0]]


def test_continuity_rms_is_the_integrated_imbalance_norm(oracle):
    m = two_cells(oracle)
    st, rms = oracle.fv_continuity_rms(m, on_internal(m, 3.0))
    assert st == 0 and rms == 3.0  # residuals [+3, -3]


def test_initial_face_flux_interpolates_but_keeps_wall_fluxes(oracle):
    m = two_cells(oracle)
    vel = np.array([[1.0, 0.0, 0.0], [1.0, 0.0, 0.0]])
    st, flux = oracle.fv_initial_face_flux(m, vel, np.where(m.neigh < 0, 4.0, 0.0))
    assert st == 0
    for f in range(m.nf):
        assert flux[f] == (float(vel[0] @ m.area[f]) if m.neigh[f] >= 0 else 4.0)


def closed_walls(mesh, lid=None, p_fixed=False):
    """Every boundary face a fixed-velocity wall (lid velocity (1, 0, 0) on
    faces whose centre has y == lid); pressure zero gradient, or fixed 0."""
    nf = mesh.nf
    fixed = (mesh.neigh < 0).astype(np.int32)
    val = np.zeros((nf, 3))
    if lid is not None:
        val[(mesh.neigh < 0) & (np.abs(mesh.fc[:, 1] - lid) < 1e-12), 0] = 1.0
    p_bc = (fixed if p_fixed else np.zeros(nf, dtype=np.int32), np.zeros(nf))
    return (fixed, val), p_bc


def test_zero_velocity_closed_two_cell_case_stays_at_rest(oracle):
    m = two_cells(oracle)
    vel_bc, p_bc = closed_walls(m, p_fixed=True)
    st, u, p, flux, hist, rep = oracle.fv_simple(m, vel_bc, p_bc, nu=1.0)
    assert st == 0 and rep.converged and rep.final_continuity_rms < 1e-12
    assert np.all(u == 0.0) and np.all(p == 0.0) and np.all(flux == 0.0)


def test_corrected_face_flux_removes_a_nonzero_initial_two_cell_imbalance(oracle):
    m = two_cells(oracle)
    vel_bc, p_bc = closed_walls(m, p_fixed=True)
    st, u, p, flux, hist, rep = oracle.fv_simple(m, vel_bc, p_bc, nu=1.0, face_flux=on_internal(m, 3.0))
    assert st == 0 and rep.converged
    assert hist[0] == 3.0 and rep.final_continuity_rms < 1e-10


@pytest.mark.parametrize("skew", [0.0, 0.2])
def test_low_reynolds_closed_cavity_converges_without_wall_leakage(oracle, skew):
    # simple.rs:1406-1532: 3 x 3 cavity (orthogonal, or skewed x + 0.2 y),
    # lid (1, 0, 0) on the top faces, zero-gradient pressure, nu 0.1
    pts = [(x + skew * y, y, 0.0) for y in range(4) for x in range(4)]
    p_ = lambda x, y: x + 4 * y  # noqa: E731
    m = oracle.FvMesh(pts, [[p_(x, y), p_(x + 1, y), p_(x + 1, y + 1), p_(x, y + 1)] for y in range(3) for x in range(3)])
    vel_bc, p_bc = closed_walls(m, lid=3.0)
    tol = 1e-9 if skew == 0.0 else 1e-8
    st, u, p, flux, hist, rep = oracle.fv_simple(m, vel_bc, p_bc, nu=0.1, max_outer=300 if skew == 0.0 else 500,
                                                 continuity_tolerance=tol, momentum_solver=(1e-12, 1e-8, 1000),
                                                 pressure_solver=(1e-12, 1e-8, 1000))
    assert st == 0 and rep.converged and rep.final_continuity_rms < tol
    if skew == 0.0:
        assert np.any(np.sum(u * u, axis=1) > 1e-12)
    assert np.all(np.isfinite(u)) and np.all(np.isfinite(p))
    assert np.all(np.abs(flux[m.neigh < 0]) < 1e-12)


def test_velocity_inlet_pressure_outlet_channel_balances_boundary_flow(oracle):
    # tests/unstructured_incompressible.rs:345-388 on the 2 x 2 mesh of :65-116:
    # inlet u = (1, 0, 0) on x = 0, outlet p = 0 on x = 2, no-slip walls, nu 0.1
    m = oracle.quad_grid(2, 2)
    b = m.neigh < 0
    left, right = b & (m.fc[:, 0] == 0.0), b & (m.fc[:, 0] == 2.0)
    vfix = (b & ~right).astype(np.int32)
    vval = np.zeros((m.nf, 3))
    vval[left, 0] = 1.0
    p_bc = (right.astype(np.int32), np.zeros(m.nf))
    wall_flux = np.where(left, vval[:, 0] * m.area[:, 0], 0.0)
    st, u, p, flux, hist, rep = oracle.fv_simple(m, (vfix, vval), p_bc, pc_bc=p_bc, nu=0.1, max_outer=500,
                                                 continuity_tolerance=1e-9, face_flux=wall_flux)
    assert st == 0 and rep.converged
    inlet, outlet = flux[left].sum(), flux[right].sum()
    assert abs(inlet + outlet) <= 1e-8 and outlet > 0.0
    assert abs(flux[b].sum()) <= 1e-8
    assert flux[b][flux[b] < 0].sum() < 0.0 and flux[b][flux[b] > 0].sum() > 0.0
    assert 0.5 * (p[0] + p[2]) > 0.5 * (p[1] + p[3])


@pytest.mark.parametrize("flux_value", [2.0, -2.0])
def test_upwind_internal_coefficients_two_cell(oracle, flux_value):
    # momentum.rs:718-764, zero-gradient boundary, nu 1
    m = two_cells(oracle)
    bc = (np.zeros(m.nf, dtype=np.int32), np.zeros(m.nf))
    st, ro, ci, va, rhs = oracle.fv_assemble_momentum(m, 1.0, bc, on_internal(m, flux_value))
    assert st == 0
    f = m.internal_faces()[0]
    o, n = m.owner[f], m.neigh[f]
    pos = flux_value > 0
    assert csr_get(ro, ci, va, o, o) == 1.0 + (2.0 if pos else 0.0)
    assert csr_get(ro, ci, va, n, n) == 1.0 + (0.0 if pos else 2.0)
    assert csr_get(ro, ci, va, o, n) == -1.0 + min(flux_value, 0.0)
    assert csr_get(ro, ci, va, n, o) == -1.0 - max(flux_value, 0.0)


def channel(oracle, ny):
    """momentum.rs:530-560: one column of ny cells on the unit square."""
    pts = []
    for y in range(ny + 1):
        pts += [(0.0, y / ny, 0.0), (1.0, y / ny, 0.0)]
    return oracle.FvMesh(pts, [[2 * y, 2 * y + 1, 2 * y + 3, 2 * y + 2] for y in range(ny)])


def solve_component(oracle, m, bc, source=None):
    from flursys_b200 import _abi
    st, ro, ci, va, rhs = oracle.fv_assemble_momentum(m, 1.0, bc, np.zeros(m.nf), source=source)
    assert st == 0
    st, x, rep = oracle.csr_solve("bicgstab", ro, ci, va, rhs, np.zeros(m.nc),
                                  _abi.LinearSolverOptions(1e-13, 1e-13, 10000))
    assert st == 0 and rep.status == _abi.LINEAR_CONVERGED
    return x


def test_steady_diffusion_recovers_the_couette_profile(oracle):
    m = channel(oracle, 12)
    y = m.fc[:, 1]
    b = m.neigh < 0
    fixed = (b & ((y < 1e-12) | (np.abs(y - 1.0) < 1e-12))).astype(np.int32)
    value = np.where(np.abs(y - 1.0) < 1e-12, 1.0, 0.0)
    u = solve_component(oracle, m, (fixed, value))
    assert np.all(np.abs(u - m.cc[:, 1]) < 1e-10)


def test_poiseuille_source_profile_converges_under_refinement(oracle):
    errors = []
    for n in (8, 16, 32):
        m = channel(oracle, n)
        y = m.fc[:, 1]
        fixed = ((m.neigh < 0) & ((y < 1e-12) | (np.abs(y - 1.0) < 1e-12))).astype(np.int32)
        u = solve_component(oracle, m, (fixed, np.zeros(m.nf)), source=np.full(m.nc, 2.0))
        yc = m.cc[:, 1]
        errors.append(float(np.sqrt(np.sum((u - yc * (1.0 - yc)) ** 2) / n)))
    assert errors[2] < errors[1] < errors[0]
