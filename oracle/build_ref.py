"""Build recipe for oracle/_ref: the reference's own hot-path sources compiled for the CPU
(and, further down, with nvcc for the GPU, as shipped and in FP64).

Test infrastructure only (the pinning oracle and the benchmark's reference arm). It
compiles gpu-vh's rhic/src/*.cu files IN PLACE from the reference tree with g++ through
the host shim in oracle/ref_shim, links them with oracle/ref_driver.cpp, and writes one
shared library per physics variant into oracle/_ref/ (git-ignored; it travels with the
working tree to the GPU host like every other built .so).

Two files need a generated overlay copy, written to oracle/_ref/overlay/: FluxLimiter.cu
hard-codes `#define THETA 2.0` (FluxLimiter.cu:15) after its includes, so no header can
override it; the copy only turns THETA into a runtime double so one build serves both the
shipped theta=2.0 and the theta=1.8 configuration. HydrodynamicValidity.cu ends with a
<<<>>> launcher; its copy stops before that function. Every other source is compiled
unchanged.

Variants (compile-time switches the reference exposes as macros):
  precision  fp64 (PRECISION double + double intrinsics, via the shim) | fp32 (as shipped)
  eos        conf (CONFORMAL_EOS, EquationOfState.cuh:16) | qcd (default WB fit)
  physics    bulk (PIMUNU+PI: 15 components) | shear (PI off: 14) | ideal (4)
  coords     Milne (as shipped) | _cart suffix: USE_CARTESIAN_COORDINATES defined on the
             command line (SourceTerms.cu:25 leaves it commented out; its #ifdef at 738-743
             then takes the Cartesian source terms), for three FP64 physics variants
"""
from __future__ import annotations

import itertools
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
# Where this recipe reads the reference tree: $GVH_REFERENCE_ROOT, else the location the
# build container mounts it at. This is the only place the location is written down; the
# fixture scripts and the compile test take it from here. Hosts without the tree (the GPU
# hosts) skip every step that needs it and use the libraries built before.
REF_ROOT = os.environ.get("GVH_REFERENCE_ROOT") or "/root/reference"
OUT = os.path.join(HERE, "_ref")

SOURCES = [
    "EulerStep.cu",
    "SemiDiscreteKurganovTadmorScheme.cu",
    "HalfSiteExtrapolation.cu",
    "LocalPropagationSpeed.cu",
    "SpectralRadius.cu",
    "FluxFunctions.cu",
    "SourceTerms.cu",
    "TransportCoefficients.cu",
    "EnergyMomentumTensor.cu",
    "EquationOfState.cu",
    "RegulateDissipativeCurrents.cu",
]

PRECISIONS = {"fp64": ["-DGVH_REF_FP64"], "fp32": []}
EOS = {"conf": ["-DCONFORMAL_EOS"], "qcd": []}
PHYSICS = {"bulk": [], "shear": ["-DGVH_REF_NO_BULK"], "ideal": ["-DGVH_REF_IDEAL"]}


CARTESIAN_VARIANTS = ["fp64_conf_ideal_cart", "fp64_conf_shear_cart", "fp64_qcd_bulk_cart"]


def variant_names():
    return ["_".join(v) for v in itertools.product(PRECISIONS, EOS, PHYSICS)] + CARTESIAN_VARIANTS


def lib_path(name: str) -> str:
    return os.path.join(OUT, f"libref_{name}.so")


def _overlay_flux_limiter() -> str:
    src = os.path.join(REF_ROOT, "rhic", "src", "FluxLimiter.cu")
    with open(src) as f:
        text = f.read()
    needle = "#define THETA 2.0"
    if needle not in text:
        raise RuntimeError(f"{src}: expected '{needle}' not found")
    text = text.replace(needle, "extern double gvh_ref_theta;\n#define THETA gvh_ref_theta")
    d = os.path.join(OUT, "overlay")
    os.makedirs(d, exist_ok=True)
    dst = os.path.join(d, "FluxLimiter.cu")
    with open(dst, "w") as f:
        f.write(text)
    return dst


def _overlay_validity() -> str:
    """HydrodynamicValidity.cu ends with its host launcher, a <<<>>> launch that g++ cannot
    compile (HydrodynamicValidity.cu:231-235); the copy stops before it, the kernel itself is
    unchanged (the driver launches it over the interior)."""
    src = os.path.join(REF_ROOT, "rhic", "src", "HydrodynamicValidity.cu")
    with open(src) as f:
        text = f.read()
    cut = text.find("void checkValidity(")
    if cut < 0:
        raise RuntimeError(f"{src}: launcher 'void checkValidity(' not found")
    d = os.path.join(OUT, "overlay")
    os.makedirs(d, exist_ok=True)
    dst = os.path.join(d, "HydrodynamicValidity.cu")
    with open(dst, "w") as f:
        f.write(text[:cut])
    return dst


def _run(cmd):
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        raise RuntimeError("command failed: " + " ".join(cmd) + "\n" + r.stdout)


def build_variant(name: str, flux_limiter: str, validity: str) -> str:
    prec, eos, phys, *coords = name.split("_")
    flags = PRECISIONS[prec] + EOS[eos] + PHYSICS[phys] + (["-DUSE_CARTESIAN_COORDINATES"] if coords == ["cart"] else [])
    obj_dir = os.path.join(OUT, "obj", name)
    os.makedirs(obj_dir, exist_ok=True)
    src_dir = os.path.join(REF_ROOT, "rhic", "src")
    inc = [
        "-I", os.path.join(HERE, "ref_shim"),
        "-I", os.path.join(REF_ROOT, "rhic", "include"),
        "-I", src_dir,
    ]
    common = ["g++", "-std=c++14", "-O2", "-fPIC", "-fopenmp", "-ffp-contract=off", "-w"] + inc + flags
    objs = []
    for s in [os.path.join(src_dir, x) for x in SOURCES] + [flux_limiter, validity]:
        o = os.path.join(obj_dir, os.path.basename(s) + ".o")
        _run(common + ["-x", "c++", "-c", s, "-o", o])
        objs.append(o)
    o = os.path.join(obj_dir, "ref_driver.o")
    _run(common + ["-c", os.path.join(HERE, "ref_driver.cpp"), "-o", o])
    objs.append(o)
    # the freeze-out replay includes FreezeOut.cpp, Memory.cpp and cornelius.cpp from the
    # reference's freezeout/ directory, as HydroPlugin.cpp does
    o = os.path.join(obj_dir, "ref_surface.o")
    _run(common + ["-I", os.path.join(REF_ROOT, "freezeout"), "-c", os.path.join(HERE, "ref_surface.cpp"), "-o", o])
    objs.append(o)
    lib = lib_path(name)
    _run(["g++", "-shared", "-fopenmp", "-o", lib] + objs)
    return lib


def build_cornelius() -> str:
    """The reference's cornelius (freezeout/cornelius-c++-1.3/cornelius.cpp, included by
    oracle/ref_cornelius.cpp from its place in the reference tree)."""
    lib = os.path.join(OUT, "libref_cornelius.so")
    inc = os.path.join(REF_ROOT, "freezeout", "cornelius-c++-1.3")
    _run(["g++", "-std=c++14", "-O2", "-fPIC", "-shared", "-ffp-contract=off", "-w", "-I", inc,
          os.path.join(HERE, "ref_cornelius.cpp"), "-o", lib])
    return lib


# ---- the reference's own CUDA build (nvcc, sm_100a) -------------------------------------
# The same hot-path sources plus the files that hold its launches and device state, compiled
# with relocatable device code and linked with oracle/ref_gpu_driver.cu into one shared
# library per variant (oracle/_ref/libref_gpu_<variant>.so). "fp32" is the build as shipped;
# "fp64" adds the PRECISION double overlay (oracle/ref_gpu_shim). The limiter slope is a
# literal in FluxLimiter.cu:15 (THETA 2.0): the 2.0 variants compile that file unchanged,
# the 1.8 variants compile a generated overlay copy whose only change is the literal.
GPU_SOURCES = SOURCES + [
    "HydrodynamicValidity.cu",
    "FullyDiscreteKurganovTadmorScheme.cu",
    "GhostCells.cu",
    "DynamicalVariables.cu",
    "CudaConfiguration.cu",
]
# (precision, eos, physics, theta): the benchmark event's physics as shipped and in FP64,
# and the 33x33x17 conformal configuration (theta 1.8) in both precisions
GPU_VARIANTS = [
    ("fp32", "qcd", "bulk", "2.0"),
    ("fp64", "qcd", "bulk", "2.0"),
    ("fp32", "conf", "shear", "1.8"),
    ("fp64", "conf", "shear", "1.8"),
]
NVCC_ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def gpu_variant_name(prec: str, eos: str, phys: str, theta: str) -> str:
    return f"{prec}_{eos}_{phys}_th{theta}"


def gpu_lib_path(name: str) -> str:
    return os.path.join(OUT, f"libref_gpu_{name}.so")


def _overlay_flux_limiter_theta(theta: str) -> str:
    src = os.path.join(REF_ROOT, "rhic", "src", "FluxLimiter.cu")
    with open(src) as f:
        text = f.read()
    needle = "#define THETA 2.0"
    if needle not in text:
        raise RuntimeError(f"{src}: expected '{needle}' not found")
    d = os.path.join(OUT, "overlay", f"theta{theta}")
    os.makedirs(d, exist_ok=True)
    dst = os.path.join(d, "FluxLimiter.cu")
    with open(dst, "w") as f:
        f.write(text.replace(needle, f"#define THETA {theta}"))
    return dst


def build_gpu_variant(prec: str, eos: str, phys: str, theta: str) -> str:
    name = gpu_variant_name(prec, eos, phys, theta)
    flags = PRECISIONS[prec] + EOS[eos] + PHYSICS[phys] + [f"-DGVH_REF_THETA={theta}"]
    obj_dir = os.path.join(OUT, "obj", "gpu_" + name)
    os.makedirs(obj_dir, exist_ok=True)
    src_dir = os.path.join(REF_ROOT, "rhic", "src")
    inc = ["-I", os.path.join(HERE, "ref_gpu_shim"), "-I", os.path.join(REF_ROOT, "rhic", "include"), "-I", src_dir]
    common = ["nvcc"] + NVCC_ARCH + ["-O3", "-rdc=true", "-Xcompiler", "-fPIC", "-w", "-std=c++14"] + inc + flags
    flux = os.path.join(src_dir, "FluxLimiter.cu") if theta == "2.0" else _overlay_flux_limiter_theta(theta)
    objs = []
    for s in [os.path.join(src_dir, x) for x in GPU_SOURCES] + [flux, os.path.join(HERE, "ref_gpu_driver.cu")]:
        o = os.path.join(obj_dir, os.path.basename(s) + ".o")
        extra = []
        if prec == "fp64" and os.path.basename(s) == "HydrodynamicValidity.cu":
            # checkValidityKernel is launched with a fixed 16x16x2 = 512-thread block
            # (HydrodynamicValidity.cu:233, CudaConfiguration.cuh:36-38), which fits an SM's
            # 65536 registers only at <= 128 per thread; in double precision nvcc gives it 134
            # and the launch fails (the reference ignores the error). The as-shipped FP32
            # build needs 79 and is compiled unchanged.
            extra = ["-maxrregcount=128"]
        _run(common + extra + ["-x", "cu", "-c", s, "-o", o])
        objs.append(o)
    lib = gpu_lib_path(name)
    _run(["nvcc"] + NVCC_ARCH + ["-shared", "-rdc=true", "-Xcompiler", "-fPIC", "-o", lib] + objs)
    return lib


# The drop-in (gpu-vh_b200/dropin/twoStepRungeKutta_gvh.cu) built into the reference's own
# program in place of FullyDiscreteKurganovTadmorScheme.cu, as a maintainer would build it,
# and linked against libgvh.so: the same driver then runs the reference's allocation, set-up
# and step loop with libgvh's step behind twoStepRungeKutta.
DROPIN_VARIANTS = [
    ("fp64", "conf", "shear", "1.8"),
    ("fp64", "qcd", "bulk", "2.0"),
    ("fp32", "qcd", "bulk", "2.0"),
]
REPO = os.path.dirname(HERE)
PKG = os.path.join(REPO, "gpu-vh_b200")


def gpu_dropin_lib_path(name: str) -> str:
    return os.path.join(OUT, f"libref_gpu_dropin_{name}.so")


def build_gpu_dropin_variant(prec: str, eos: str, phys: str, theta: str) -> str:
    name = gpu_variant_name(prec, eos, phys, theta)
    flags = PRECISIONS[prec] + EOS[eos] + PHYSICS[phys] + [f"-DGVH_REF_THETA={theta}", f"-DGVH_THETA={theta}"]
    obj_dir = os.path.join(OUT, "obj", "gpu_dropin_" + name)
    os.makedirs(obj_dir, exist_ok=True)
    src_dir = os.path.join(REF_ROOT, "rhic", "src")
    inc = ["-I", os.path.join(HERE, "ref_gpu_shim"), "-I", os.path.join(REF_ROOT, "rhic", "include"), "-I", src_dir,
           "-I", os.path.join(REPO, "include")]
    common = ["nvcc"] + NVCC_ARCH + ["-O3", "-rdc=true", "-Xcompiler", "-fPIC", "-w", "-std=c++14"] + inc + flags
    flux = os.path.join(src_dir, "FluxLimiter.cu") if theta == "2.0" else _overlay_flux_limiter_theta(theta)
    sources = [os.path.join(src_dir, x) for x in GPU_SOURCES if x != "FullyDiscreteKurganovTadmorScheme.cu"]
    sources += [flux, os.path.join(PKG, "dropin", "twoStepRungeKutta_gvh.cu"), os.path.join(HERE, "ref_gpu_driver.cu")]
    objs = []
    for s in sources:
        o = os.path.join(obj_dir, os.path.basename(s) + ".o")
        extra = ["-maxrregcount=128"] if prec == "fp64" and os.path.basename(s) == "HydrodynamicValidity.cu" else []
        _run(common + extra + ["-x", "cu", "-c", s, "-o", o])
        objs.append(o)
    lib = gpu_dropin_lib_path(name)
    _run(["nvcc"] + NVCC_ARCH + ["-shared", "-rdc=true", "-Xcompiler", "-fPIC", "-o", lib] + objs +
         ["-L" + PKG, "-lgvh", "-Xlinker", "-rpath=$ORIGIN/../../gpu-vh_b200"])
    return lib


def build_gpu(jobs: int | None = None, verbose: bool = True) -> list[str]:
    """Build the reference's CUDA variants (nvcc cross-compiles without a GPU). Skips
    (returns []) when the reference tree is not present."""
    if not os.path.isdir(os.path.join(REF_ROOT, "rhic", "src")):
        return []
    os.makedirs(OUT, exist_ok=True)
    with ThreadPoolExecutor(max_workers=jobs or min(4, os.cpu_count() or 4)) as ex:
        libs = list(ex.map(lambda v: build_gpu_variant(*v), GPU_VARIANTS))
        if os.path.exists(os.path.join(PKG, "libgvh.so")):
            libs += list(ex.map(lambda v: build_gpu_dropin_variant(*v), DROPIN_VARIANTS))
    if verbose:
        print(f"[oracle/_ref] built {len(libs)} CUDA variants of the reference into {OUT}")
    return libs


def build(jobs: int | None = None, verbose: bool = True) -> list[str]:
    """Build every variant; returns the library paths. Skips (returns []) when the
    reference tree is not present, e.g. on a host that only runs prebuilt files."""
    if not os.path.isdir(os.path.join(REF_ROOT, "rhic", "src")):
        if verbose:
            print(f"[oracle/_ref] reference tree not found at {REF_ROOT}; skipping")
        return []
    os.makedirs(OUT, exist_ok=True)
    fl = _overlay_flux_limiter()
    va = _overlay_validity()
    names = variant_names()
    with ThreadPoolExecutor(max_workers=jobs or min(12, os.cpu_count() or 4)) as ex:
        libs = list(ex.map(lambda n: build_variant(n, fl, va), names))
    libs.append(build_cornelius())
    libs += build_gpu(jobs=4, verbose=verbose)
    shutil.rmtree(os.path.join(OUT, "obj"), ignore_errors=True)
    if verbose:
        print(f"[oracle/_ref] built {len(libs)} variants into {OUT}")
    return libs


if __name__ == "__main__":
    build()
    sys.exit(0)
