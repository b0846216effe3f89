"""Builds libgvh.so (the CUDA stage kernels + C ABI) in-tree for sm_100a."""
from __future__ import annotations

import os
import subprocess

PKG_ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))  # gpu-vh_b200/
REPO_ROOT = os.path.dirname(PKG_ROOT)
CSRC = os.path.join(PKG_ROOT, "csrc")
LIB = os.path.join(PKG_ROOT, "libgvh.so")
# the same sources with every stage cell's stencil indices checked (GVH_BOUNDS_CHECK): a cell
# whose indices leave the arrays is skipped and raises GVH_STATUS_BOUNDS; for debugging
BOUNDS_LIB = os.path.join(PKG_ROOT, "libgvh_bounds.so")
EXE = os.path.join(PKG_ROOT, "gvh-run")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC,-ffp-contract=off", "-shared",
]


def sources() -> list[str]:
    return [os.path.join(CSRC, "gvh_capi.cu"), os.path.join(CSRC, "gvh_batch.cu"), os.path.join(CSRC, "gvh_plugin.cpp"),
            os.path.join(CSRC, "gvh_noalloc.cu"), os.path.join(CSRC, "gvh_surface.cu"),
            os.path.join(CSRC, "gvh_surface_host.cpp"), os.path.join(CSRC, "gvh_surface_rows.cu")]


# per-file flags: the device surface rows repeat the host's arithmetic operation for operation
# (the host side is compiled with -ffp-contract=off), so no multiply-add contraction there
FILE_FLAGS = {"gvh_surface_rows.cu": ["-fmad=false"]}


def needs_rebuild() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(REPO_ROOT, "include", "gvh.h")]
    return any(os.path.getmtime(d) > t for d in deps if os.path.isfile(d))


def build(verbose: bool = True, ptxas_info: bool = False, bounds_check: bool = False) -> str:
    """Compiles every source to an object in parallel (gpu-vh_b200/_build/), then links.
    bounds_check builds BOUNDS_LIB instead of LIB (and no executable)."""
    from concurrent.futures import ThreadPoolExecutor

    nvcc = os.environ.get("NVCC", "nvcc")
    obj_dir = os.path.join(PKG_ROOT, "_build", "bounds" if bounds_check else "")
    os.makedirs(obj_dir, exist_ok=True)
    compile_flags = [f for f in NVCC_FLAGS if f != "-shared"] + (["-DGVH_BOUNDS_CHECK"] if bounds_check else [])
    lib = BOUNDS_LIB if bounds_check else LIB

    def compile_one(src):
        obj = os.path.join(obj_dir, os.path.basename(src) + ".o")
        cmd = [nvcc] + compile_flags + FILE_FLAGS.get(os.path.basename(src), []) + \
              (["-Xptxas", "-v"] if ptxas_info else []) + ["-c", src, "-o", obj]
        r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
        if r.returncode != 0:
            raise RuntimeError("libgvh build failed:\n" + r.stdout)
        return obj, r.stdout

    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        results = list(ex.map(compile_one, sources()))
    objs = [o for o, _ in results]
    log = "".join(out for _, out in results)
    r = subprocess.run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", lib] + objs,
                       stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        raise RuntimeError("libgvh link failed:\n" + r.stdout)
    if bounds_check:
        if verbose:
            print(f"[gvh] built {lib}")
        return log
    exe = [nvcc, "-O2", "-std=c++17", "-o", EXE, os.path.join(CSRC, "gvh_run_main.cpp"), "-L" + PKG_ROOT, "-lgvh",
           "-Xlinker", "-rpath=$ORIGIN"]
    r2 = subprocess.run(exe, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r2.returncode != 0:
        raise RuntimeError("gvh-run build failed:\n" + r2.stdout)
    if verbose:
        print(f"[gvh] built {LIB} and {EXE}")
    return log
