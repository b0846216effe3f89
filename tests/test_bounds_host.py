"""The per-cell index check of the bounds-checked build (cell_stencil_ok in
gpu-vh_b200/csrc/gvh_stage.cuh) on the CPU: consistent lattices pass everywhere, inconsistent
strides and cells outside the lattice are flagged (tests/bounds_check.cu, built with nvcc,
run on the host). The GPU side -- the bounds-checked library on a lattice, no bit raised and
the same values as the plain build -- is tests/test_bounds_gpu.py."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "gpu-vh_b200", "csrc")


@pytest.mark.skipif(shutil.which("nvcc") is None, reason="nvcc not found")
def test_cell_stencil_check_on_host(tmp_path):
    exe = tmp_path / "bounds_check"
    subprocess.run(["nvcc", "-std=c++17", "-I", CSRC, "-o", str(exe), os.path.join(HERE, "bounds_check.cu")],
                   check=True, capture_output=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "0 errors" in r.stdout
