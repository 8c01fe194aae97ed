"""Build the hpx_b200 CUDA library in-tree (``cuhpx_b200/libhpx_b200.so``).

The library is one translation unit compiled by nvcc for sm_100a only and
exports the C ABI declared in ``include/hpx_b200.h``.  Python reaches it
through ctypes (``cuhpx_b200/_lib.py``); nothing here depends on torch.

    python -m cuhpx_b200.build [--force] [--debug]
"""

import argparse
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libhpx_b200.so")
SOURCES = ["hpx_plan.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc():
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _deps():
    files = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cu", ".cuh", ".h"))]
    files.append(os.path.join(REPO, "include", "hpx_b200.h"))
    files.append(os.path.abspath(__file__))
    return files


def up_to_date():
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(f) <= t for f in _deps())


def build(force=False, debug=False, verbose=False, defines=(), out=None):
    """Compile the library; ``defines``/``out`` build an instrumented copy elsewhere."""
    target = out or LIB
    if not force and out is None and not defines and up_to_date():
        return LIB
    cmd = [
        _nvcc(),
        *ARCH,
        "-O3",
        "-lineinfo",
        "-std=c++17",
        "-shared",
        "-Xcompiler",
        "-fPIC,-fvisibility=hidden",
        "-Xptxas",
        "-v" if verbose else "-O3",
        "--expt-relaxed-constexpr",
        "-I",
        os.path.join(REPO, "include"),
        "-o",
        target + ".tmp",
        *[os.path.join(CSRC, s) for s in SOURCES],
    ]
    if debug:  # the bounds-checked build (also VARIANTS["bounds"])
        cmd.insert(1, "-DHPX_CHECK_BOUNDS=1")
    for d in defines:
        cmd.insert(1, "-D" + d)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError("nvcc failed building libhpx_b200.so")
    if verbose:
        sys.stderr.write(res.stderr)
    os.replace(target + ".tmp", target)
    return target


# Checker builds of the same sources (test infrastructure, never loaded by the
# package): name -> (defines, file).
#   waittest  every bounded pipeline wait gives up after 1 ms and the tensor-core
#             kernels withhold their TMA loads, so their waits run out: the
#             failure-detection test checks that a call then ends with
#             HPX_ERR_TIMEOUT and leaves the device usable
#   bounds    every global access of the ring, layout, contraction-epilogue and
#             spin-1 kernels is checked against the call's buffer extents
#             (skipped and reported as HPX_ERR_BOUNDS by hpx_plan_check)
VARIANTS = {
    "waittest": (["HPX_WAIT_LIMIT_NS=1000000ull", "HPX_TEST_WITHHOLD_TMA_LOADS=1"],
                 os.path.join(HERE, "libhpx_b200_waittest.so")),
    "bounds": (["HPX_CHECK_BOUNDS=1"], os.path.join(HERE, "libhpx_b200_bounds.so")),
}


def build_variant(name, force=False):
    """Compile one checker build (see VARIANTS) if it is older than the sources."""
    defines, path = VARIANTS[name]
    if not force and os.path.exists(path) and all(os.path.getmtime(f) <= os.path.getmtime(path) for f in _deps()):
        return path
    return build(defines=defines, out=path)


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--debug", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    ap.add_argument("-D", dest="defines", action="append", default=[])
    ap.add_argument("--out", default=None)
    a = ap.parse_args()
    print(build(force=a.force or bool(a.out), debug=a.debug, verbose=a.verbose, defines=a.defines, out=a.out))
