"""Builds the engine's shared library, in tree, for sm_100a.

    python -m emptyheaded_b200.build          # -> emptyheaded_b200/_lib/libeh_b200.so

Each csrc/*.cu is compiled with nvcc (-gencode arch=compute_100a,code=sm_100a
-O3 -lineinfo) to an object in _lib/obj, in parallel, then linked into one
shared library that exports the C ABI of include/eh_b200.h.  Objects are
rebuilt when their source or any header is newer.
"""
import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "_lib")
OBJDIR = os.path.join(LIBDIR, "obj")
LIB = os.path.join(LIBDIR, "libeh_b200.so")
INCLUDE = os.path.join(ROOT, "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
              "--expt-relaxed-constexpr", "-I" + INCLUDE, "-I" + CSRC]


def nvcc():
    p = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(p):
        raise RuntimeError("nvcc not found")
    return p


def _headers():
    return glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(INCLUDE, "*.h"))


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose=False, extra_flags=(), libdir=None):
    """Compile and link; `libdir` (default _lib) and `extra_flags` let a
    variant build land elsewhere without touching the in-tree library."""
    objdir = OBJDIR if libdir is None else os.path.join(libdir, "obj")
    lib = LIB if libdir is None else os.path.join(libdir, "libeh_b200.so")
    os.makedirs(objdir, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    hdrs = _headers()
    jobs = []
    objs = []
    for s in srcs:
        o = os.path.join(objdir, os.path.basename(s)[:-3] + ".o")
        objs.append(o)
        if _stale(o, [s] + hdrs):
            jobs.append([nvcc()] + ARCH + NVCC_FLAGS + list(extra_flags) + ["-c", s, "-o", o])

    def run(cmd):
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("compile failed: %s\n%s%s" % (" ".join(cmd), r.stdout, r.stderr))
        if verbose and (r.stdout or r.stderr):
            print(r.stdout + r.stderr, file=sys.stderr)

    with cf.ThreadPoolExecutor(max_workers=min(8, max(1, len(jobs)))) as ex:
        list(ex.map(run, jobs))
    if jobs or _stale(lib, objs):
        run([nvcc()] + ARCH + ["-shared", "-o", lib] + objs + ["-lcudart"])
    return lib


if __name__ == "__main__":
    print(build(verbose=True))
