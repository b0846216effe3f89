"""The surface.dat number formatter (gpu-vh_b200/csrc/gvh_format.hpp) writes the characters
of printf's "%g", which is what the reference's ofstream writes (HydroPlugin.cpp:315-372).
Compiled with the host compiler and run on the CPU."""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "gpu-vh_b200", "csrc")


def test_g6_matches_printf(tmp_path):
    exe = tmp_path / "format_check"
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-I", CSRC, "-o", str(exe),
                    os.path.join(HERE, "format_check.cpp")], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert " 0 mismatches" in r.stdout


def test_device_text_splice(tmp_path):
    """format_rows with the device's text and its host rows (gvh_surface_host.cpp) gives the
    text of formatting every row on the host, for pools of 1, 3 and 8 threads, synchronous
    and asynchronous, with no, some, runs of and only host rows, rows kept or not."""
    exe = tmp_path / "surface_splice_check"
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-pthread", "-I", CSRC, "-o", str(exe),
                    os.path.join(HERE, "surface_splice_check.cpp"), os.path.join(CSRC, "gvh_surface_host.cpp")],
                   check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert " 0 mismatches" in r.stdout
