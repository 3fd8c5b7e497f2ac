"""The C ABI: the library loads, exports every symbol include/*.h declares,
and the ctypes structures match the C layouts (no device calls)."""
import ctypes as C
import os
import re
import subprocess
import tempfile

import pytest

from flursys_b200 import _abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "flursys_cuda.h")


def declared_symbols():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(flursys_cuda_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = _abi.load()
    syms = declared_symbols()
    assert len(syms) >= 15
    for s in syms:
        assert hasattr(lib, s), s
        assert s in _abi.SIGNATURES, f"{s} has no ctypes signature"
    assert lib.flursys_cuda_abi_version() == _abi.ABI_VERSION


STRUCTS = {
    "FlursysLinearSolverOptions": _abi.LinearSolverOptions,
    "FlursysLinearSolveReport": _abi.LinearSolveReport,
    "FlursysCaseParams": _abi.CaseParams,
    "FlursysBoundaryOverride": _abi.BoundaryOverride,
    "FlursysCudaConfig": _abi.CudaConfig,
    "FlursysStepReport": _abi.StepReport,
    "FlursysThermalBoundary": _abi.ThermalBoundary,
    "FlursysPhysicsSettings": _abi.PhysicsSettings,
}


def test_ctypes_structures_match_the_header_layout():
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "flursys_cuda.h"', "int main(void){"]
    for cname, py in STRUCTS.items():
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, _ in py._fields_:
            lines.append(f'printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines.append("return 0;}")
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "layout.c")
        exe = os.path.join(d, "layout")
        open(src, "w").write("\n".join(lines))
        subprocess.run(["/usr/bin/gcc", "-I", os.path.join(ROOT, "include"), src, "-o", exe], check=True)
        out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout
    got = {}
    for line in out.splitlines():
        s, f, v = line.split()
        got[(s, f)] = int(v)
    for cname, py in STRUCTS.items():
        assert got[(cname, "size")] == C.sizeof(py), cname
        for fname, _ in py._fields_:
            assert got[(cname, fname)] == getattr(py, fname).offset, (cname, fname)


def test_default_config_mirrors_reference_defaults():
    lib = _abi.load()
    cfg = _abi.CudaConfig()
    assert lib.flursys_cuda_default_config(3, C.byref(cfg)) == 0
    # LidDrivenCavity3DConfig::default (incompressible_3d.rs:27-47)
    assert (cfg.nx, cfg.ny, cfg.nz) == (32, 32, 32)
    assert cfg.dt == 5e-4 and cfg.max_steps == 10000 and cfg.pressure_max_iters == 2000
    assert cfg.pressure_tolerance == 1e-6 and cfg.pressure_omega == 1.7
    assert cfg.case_params.reynolds == 100.0 and cfg.pressure_solver == _abi.PRESSURE_SOR
    assert lib.flursys_cuda_default_config(2, C.byref(cfg)) == 0
    assert (cfg.nx, cfg.ny) == (64, 64) and cfg.pressure_tolerance == 1e-5 and cfg.pressure_max_iters == 1200
    # ThermalSettings::default / BuoyancyModel::default (src/physics.rs:43-56,59-70)
    ph = cfg.physics
    assert ph.energy_model == _abi.ENERGY_OFF and ph.buoyancy == _abi.BUOYANCY_OFF
    assert ph.initial_temperature == 293.15 and ph.thermal_diffusivity == 2.2e-5
    assert ph.source_temperature_rate == 0.0
    assert all(ph.thermal[s].kind == _abi.THERMAL_ADIABATIC for s in range(4))


def test_create_rejects_invalid_configs_before_touching_a_device():
    lib = _abi.load()
    cfg = _abi.CudaConfig()
    lib.flursys_cuda_default_config(3, C.byref(cfg))
    cfg.nx = 3
    h = C.c_void_p()
    assert lib.flursys_cuda_create(C.byref(cfg), C.byref(h)) == _abi.ERR_INVALID_CONFIG
    buf = C.create_string_buffer(256)
    lib.flursys_cuda_global_error(buf, 256)
    assert buf.value.decode() == "nx, ny, and nz must all be at least 4"
    lib.flursys_cuda_default_config(3, C.byref(cfg))
    cfg.pressure_omega = 2.0
    assert lib.flursys_cuda_create(C.byref(cfg), C.byref(h)) == _abi.ERR_INVALID_CONFIG
    lib.flursys_cuda_default_config(2, C.byref(cfg))
    cfg.t_end = 0.0
    assert lib.flursys_cuda_create(C.byref(cfg), C.byref(h)) == _abi.ERR_INVALID_CONFIG
    lib.flursys_cuda_global_error(buf, 256)
    assert buf.value.decode() == "t_end must be positive for projection coupling"
