"""bench.py's reference arm: the oracle alone builds and runs the workload.

The reference arm times the CPU restatement of the reference path; nothing
of the CUDA library may be loaded on that path, not even to fill in the
configuration. Its config must equal the one the CUDA arm builds through the
package's public API, field for field, except the precision knob.
"""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_config_equals_the_product_config(oracle):
    sys.path.insert(0, ROOT)
    import bench
    from flursys_b200 import _abi
    for n in (16, 128):
        ref = bench.oracle_workload_config(n)
        _, ours = bench.workload_config(n, "f64")
        assert bytes(ref) == bytes(ours), n
        _, mixed = bench.workload_config(n, "mixed")
        assert mixed.precision == _abi.PRECISION_MIXED and ref.precision == _abi.PRECISION_F64


def test_reference_arm_runs_without_the_cuda_library(oracle):
    code = (
        "import runpy, sys\n"
        f"sys.argv = ['bench.py', '--impl', 'reference', '--size', '8', '--steps', '2', '--warmup', '3']\n"
        f"runpy.run_path({os.path.join(ROOT, 'bench.py')!r}, run_name='__main__')\n"
        "maps = open('/proc/self/maps').read()\n"
        "print('CUDA_LIB_LOADED' if 'libflursys_cuda' in maps else 'CUDA_LIB_ABSENT')\n")
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, cwd=ROOT, timeout=300)
    assert out.returncode == 0, out.stderr
    lines = out.stdout.strip().splitlines()
    assert lines[-1] == "CUDA_LIB_ABSENT"
    rec = json.loads(lines[-2])
    assert rec["impl"] == "reference" and rec["warmup"] == 3 and rec["steps"] == 2
    assert set(rec["config"]) == {"workload", "cells", "precision", "l2", "parallelism"}
    assert rec["config"]["workload"] == "3D lid-driven cavity 8^3, Re 400, central, PCG to 1e-8 rel L2"
    assert rec["e2e"]["h2d_bytes_per_step"] == 0
