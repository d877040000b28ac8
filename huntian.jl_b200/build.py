"""Build recipe for libhuntian_b200.so (sm_100a), in-tree next to this file.

    python huntian.jl_b200/build.py [--verbose] [--checked]

Compiles every .cu under csrc/ with nvcc for sm_100a only (no fast-math: the collapse
criterion needs IEEE divisions, square roots and NaN propagation) and links them into
one shared library with a plain C ABI (include/huntian_b200.h).  The files listed in
FILE_FLAGS are compiled to objects of their own with extra flags first (ht_collapse.cu
with -fmad=false: the ellipsoid integration keeps every product unfused, as the
reference's Julia arithmetic does).

--checked builds libhuntian_b200_checked.so from the same sources with -DHT_CHECKED: the
data-dependent indices of the shell walk and of the peak scan's output are checked before
each access, and a failed check records status 2 (ht_device_status) and skips the access
instead of trapping.  The bindings load it when HT_CHECKED=1 is set in the environment.
"""
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libhuntian_b200.so")
LIB_CHECKED = os.path.join(HERE, "libhuntian_b200_checked.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
         "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden", "-shared",
         "-cudart", "shared", "-I", os.path.join(ROOT, "include"), "-lcufft"]


FILE_FLAGS = {"ht_collapse.cu": ["-fmad=false"]}
OBJDIR = os.path.join(HERE, "_build")
CHECKED_FLAGS = ["-DHT_CHECKED"]


def sources():
    return sorted(glob.glob(os.path.join(HERE, "csrc", "*.cu")))


def _split_sources(srcs):
    plain = [f for f in srcs if os.path.basename(f) not in FILE_FLAGS]
    special = [f for f in srcs if os.path.basename(f) in FILE_FLAGS]
    return plain, special


def _objects(special, flags, objdir=OBJDIR):
    """Compile the FILE_FLAGS sources to position-independent objects."""
    os.makedirs(objdir, exist_ok=True)
    objs = []
    base = [f for f in flags if f not in ("-shared", "-cudart", "shared", "-lcufft", "-lcuda")]
    for src in special:
        obj = os.path.join(objdir, os.path.basename(src)[:-3] + ".o")
        subprocess.run([NVCC] + base + FILE_FLAGS[os.path.basename(src)] +
                       ["-Xcompiler", "-fPIC", "-c", src, "-o", obj], check=True)
        objs.append(obj)
    return objs


def deps():
    return sources() + sorted(glob.glob(os.path.join(HERE, "csrc", "*.cuh"))) + \
        [os.path.join(ROOT, "include", "huntian_b200.h")]


def needs_build(checked: bool = False) -> bool:
    lib = LIB_CHECKED if checked else LIB
    if not os.path.exists(lib):
        return True
    t = os.path.getmtime(lib)
    return any(os.path.getmtime(d) > t for d in deps())


def build(force: bool = False, verbose: bool = False, checked: bool = False) -> str:
    lib = LIB_CHECKED if checked else LIB
    if force or needs_build(checked):
        plain, special = _split_sources(sources())
        extra = (["-Xptxas", "-v"] if verbose else []) + (CHECKED_FLAGS if checked else [])
        objs = _objects(special, FLAGS + extra, OBJDIR + ("_checked" if checked else ""))
        cmd = [NVCC] + FLAGS + extra + plain + objs + ["-o", lib]
        subprocess.run(cmd, check=True)
    return lib


if __name__ == "__main__":
    print(build(force=True, verbose="--verbose" in sys.argv, checked="--checked" in sys.argv))
