"""The reference-side drop-in (gpu-vh_b200/dropin/twoStepRungeKutta_gvh.cu) compiles
against the reference's own headers, as a maintainer would build it in rhic/src."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
from oracle.build_ref import REF_ROOT  # noqa: E402

REF_SRC = os.path.join(REF_ROOT, "rhic", "src")


@pytest.mark.skipif(not os.path.isdir(REF_SRC), reason="reference tree not present")
@pytest.mark.parametrize("defines", [[], ["-DCONFORMAL_EOS"]])
def test_dropin_compiles_against_reference_headers(tmp_path, defines):
    out = tmp_path / "dropin.o"
    cmd = ["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-std=c++14", "-rdc=true", "-c", *defines,
           "-I", os.path.join(ROOT, "include"), "-I", REF_SRC, "-o", str(out),
           os.path.join(ROOT, "gpu-vh_b200", "dropin", "twoStepRungeKutta_gvh.cu")]
    r = subprocess.run(cmd, cwd=REF_SRC, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert out.exists()
