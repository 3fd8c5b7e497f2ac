"""Field writers of src/output.rs for device snapshots (legacy VTK, CSV, history).

Numbers are printed the way Rust's ``{:.12e}`` prints them (no '+' sign and
no zero padding in the exponent) so files compare byte-for-byte with the
reference's writers.
"""
from __future__ import annotations

import os

import numpy as np


def rust_e12(x: float) -> str:
    """Rust's ``format!("{:.12e}", x)``."""
    if x != x:
        return "NaN"
    if x in (float("inf"), float("-inf")):
        return "inf" if x > 0 else "-inf"
    s = "%.12e" % x
    mant, exp = s.split("e")
    return f"{mant}e{int(exp)}"


def write_legacy_vtk_3d(path: str, title: str, solver) -> None:
    """write_legacy_vtk_3d (src/output.rs:127-176) of a LidDrivenCavity3DSolver."""
    cfg = solver.cfg
    nx, ny, nz = cfg.nx, cfg.ny, cfg.nz
    dx, dy, dz = cfg.length / nx, cfg.height / ny, cfg.depth / nz
    p = solver.field("pressure")
    u = solver.field("u").reshape(nz, ny, nx + 1)
    v = solver.field("v").reshape(nz, ny + 1, nx)
    w = solver.field("w").reshape(nz + 1, ny, nx)
    uc = (0.5 * (u[:, :, :-1] + u[:, :, 1:])).ravel()
    vc = (0.5 * (v[:, :-1, :] + v[:, 1:, :])).ravel()
    wc = (0.5 * (w[:-1, :, :] + w[1:, :, :])).ravel()
    with open(path, "w") as f:
        f.write("# vtk DataFile Version 3.0\n")
        f.write(f"{title}\nASCII\nDATASET STRUCTURED_POINTS\n")
        f.write(f"DIMENSIONS {nx} {ny} {nz}\n")
        f.write("ORIGIN %.12f %.12f %.12f\n" % (0.5 * dx, 0.5 * dy, 0.5 * dz))
        f.write("SPACING %.12f %.12f %.12f\n" % (dx, dy, dz))
        f.write(f"POINT_DATA {nx * ny * nz}\n")
        f.write("SCALARS pressure double 1\nLOOKUP_TABLE default\n")
        f.write("".join(rust_e12(float(x)) + "\n" for x in p))
        f.write("VECTORS velocity double\n")
        f.write("".join(f"{rust_e12(float(a))} {rust_e12(float(b))} {rust_e12(float(c))}\n"
                        for a, b, c in zip(uc, vc, wc)))


def append_history(path: str, header: str, row: str) -> None:
    """append_history (src/output.rs:186-199)."""
    new = not os.path.exists(path)
    with open(path, "a") as f:
        if new:
            f.write(header + "\n")
        f.write(row + "\n")


def write_field_csv(path: str, solver, fu=None) -> None:
    """write_field_csv (src/output.rs:31-73) of a 2D IncompressibleSolver
    snapshot (a FieldUpdate; taken from the solver when not given), with the
    temperature column when the energy equation is on."""
    cfg = solver.cfg
    nx, ny = cfg.nx, cfg.ny
    length, height = cfg.case.domain()
    dx, dy = length / nx, height / ny
    fu = fu if fu is not None else solver.field_update()
    solid = fu.solid
    temp = fu.temperature
    with open(path, "w") as f:
        f.write("i,j,x,y,solid,p,u,v,speed,vorticity" + (",temperature" if temp is not None else "") + "\n")
        for j in range(ny):
            for i in range(nx):
                k = i + nx * j
                uu, vv = float(fu.velocity_x[k]), float(fu.velocity_y[k])
                speed = float(np.sqrt(uu * uu + vv * vv))
                f.write("%d,%d,%.12f,%.12f,%d,%s,%s,%s,%s,%s" % (
                    i, j, (i + 0.5) * dx, (j + 0.5) * dy, 1 if solid[k] else 0, rust_e12(float(fu.pressure[k])),
                    rust_e12(uu), rust_e12(vv), rust_e12(speed), rust_e12(float(fu.vorticity[k]))))
                if temp is not None:
                    f.write("," + rust_e12(float(temp[k])))
                f.write("\n")


def write_legacy_vtk(path: str, title: str, solver, fu=None) -> None:
    """write_legacy_vtk (src/output.rs:75-125) of a 2D IncompressibleSolver
    snapshot: pressure, speed, vorticity, temperature (when on), solid mask
    and the cell velocity on the cell-centre structured points."""
    cfg = solver.cfg
    nx, ny = cfg.nx, cfg.ny
    length, height = cfg.case.domain()
    dx, dy = length / nx, height / ny
    fu = fu if fu is not None else solver.field_update()
    u, v = fu.velocity_x, fu.velocity_y
    speed = np.sqrt(u * u + v * v)
    with open(path, "w") as f:
        f.write("# vtk DataFile Version 3.0\n")
        f.write(f"{title}\nASCII\nDATASET STRUCTURED_POINTS\n")
        f.write(f"DIMENSIONS {nx} {ny} 1\n")
        f.write("ORIGIN %.12f %.12f 0\n" % (0.5 * dx, 0.5 * dy))
        f.write("SPACING %.12f %.12f 1\n" % (dx, dy))
        f.write(f"POINT_DATA {nx * ny}\n")
        for name, values in (("pressure", fu.pressure), ("speed", speed), ("vorticity", fu.vorticity)) + (
                (("temperature", fu.temperature),) if fu.temperature is not None else ()):
            f.write(f"SCALARS {name} double 1\nLOOKUP_TABLE default\n")
            f.write("".join(rust_e12(float(x)) + "\n" for x in values))
        f.write("SCALARS solid int 1\nLOOKUP_TABLE default\n")
        f.write("".join(("1" if s_ else "0") + "\n" for s_ in fu.solid))
        f.write("VECTORS velocity double\n")
        f.write("".join(f"{rust_e12(float(a))} {rust_e12(float(b))} 0\n" for a, b in zip(u, v)))
