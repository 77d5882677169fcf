"""Build oracle/_ref/libref.so from the reference's own double-precision OpenCL kernels.

TEST INFRASTRUCTURE ONLY. The reference (clTEM) cannot be built here: its host code needs the OpenCL
C++ bindings, an OpenCL platform, clFFT, libtiff, Eigen and easylogging++. Its kernels, though, are
OpenCL C, close enough to C++ that g++ compiles them with a small shim. This script
  1. reads kernels/<name>_d.cl from the reference tree (argv[1], else $CLTEM_REFERENCE, else the build
     container's mount point below),
  2. applies clTEM's own source transform for the default math mode: delete "native_"
     (KernelSource::BuildToKernel, src/simulation/kernels.h:37-45),
  3. applies two syntax shims that OpenCL C needs and C++ lacks: the vector literal
     "(double2)(a, b)" becomes "make_double2(a, b)", and a __local array declared in a kernel body
     becomes a function-static array (shared by the threads that emulate one work group),
  4. writes the results to oracle/_ref/src/<name>_d.inc and compiles oracle/ref_host.cpp with them into
     oracle/_ref/libref.so (g++ -O2 -ffp-contract=off, matching the oracle's floating-point mode).
Nothing from the reference is written outside oracle/_ref/, which git ignores.
"""
import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
KERNELS = ["atom_sort", "band_limit", "band_pass", "bilinear_translate", "complex_multiply", "complex_to_real", "fft_shift",
           "init_plane_wave", "init_probe_wave", "propagator", "sqabs", "sum_reduction",
           "transmission_potentials_projected", "transmission_potentials_full_3d", "ctem_image"]


# Where the build container mounts the reference tree (read-only). This recipe is the one place that names
# it; the fixture scripts and the package build ask reference_root().
_CONTAINER_MOUNT = "/root/reference"


def reference_root(arg=None):
    """The clTEM source tree to read: `arg`, else $CLTEM_REFERENCE, else the build container's mount point;
    None when that directory holds no kernels/ (machines without the reference, such as the GPU box)."""
    root = arg or os.environ.get("CLTEM_REFERENCE") or _CONTAINER_MOUNT
    return root if os.path.isdir(os.path.join(root, "kernels")) else None


def transform(src: str) -> str:
    src = src.replace("native_", "")
    src = re.sub(r"\(double2\)\s*\(", "make_double2(", src)
    src = re.sub(r"(^|\n)(\s*)__local\s+(double|int)\s+(\w+)\s*\[", r"\1\2static \3 \4[", src)
    return src


def build(ref_root=None, quiet=False):
    ref_root = reference_root(ref_root)
    if ref_root is None:
        raise FileNotFoundError("reference tree not found: pass its path or set CLTEM_REFERENCE")
    kdir = os.path.join(ref_root, "kernels")
    if not os.path.isdir(kdir):
        raise FileNotFoundError(f"reference kernels not found under {kdir}")
    srcdir = os.path.join(OUT, "src")
    os.makedirs(srcdir, exist_ok=True)
    for k in KERNELS:
        with open(os.path.join(kdir, f"{k}_d.cl")) as f:
            txt = transform(f.read())
        with open(os.path.join(srcdir, f"{k}_d.inc"), "w") as f:
            f.write(txt)
    cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
    cmd = [cxx, "-O2", "-std=c++20", "-fPIC", "-shared", "-ffp-contract=off", "-pthread", "-w",
           "-I", srcdir, "-I", HERE, os.path.join(HERE, "ref_host.cpp"), "-o", os.path.join(OUT, "libref.so")]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("building the reference kernels failed:\n" + r.stderr)
    if not quiet:
        print("built", os.path.join(OUT, "libref.so"))
    return os.path.join(OUT, "libref.so")


if __name__ == "__main__":
    build(sys.argv[1] if len(sys.argv) > 1 else None)
