"""Compile the reference's own remapping module into ``oracle/_ref`` -- TEST INFRASTRUCTURE ONLY.

cuHPX's ``cuhpx_remap`` extension is built from two source files of the
reference, ``src/data_remapping/hpx_remapping.cpp`` and
``src/data_remapping/hpx_remapping_cuda.cu`` (with torch's extension headers
only), so it is compiled here straight from where those files lie, for
sm_100a, without the reference's setup.py.  The result,
``oracle/_ref/cuhpx_remap.so``, is git-ignored and travels with the
repository to a GPU machine, where ``tests/test_remap_gpu.py`` runs the
reference's kernels beside this library's and requires identical output.
Nothing in the product imports it.

    python -m oracle.build_ref_remap --reference /path/to/cuHPX   (or set CUHPX_REFERENCE)
"""

import argparse
import os

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
# a cuHPX checkout; the build is skipped when none is given
DEFAULT_REFERENCE = os.environ.get("CUHPX_REFERENCE")
SOURCES = ["src/data_remapping/hpx_remapping.cpp", "src/data_remapping/hpx_remapping_cuda.cu"]


def built_path():
    return os.path.join(OUT, "cuhpx_remap.so")


def build(reference=DEFAULT_REFERENCE, verbose=False):
    if not reference:
        return None
    srcs = [os.path.join(reference, s) for s in SOURCES]
    if not all(os.path.exists(s) for s in srcs):
        return None  # no reference checkout on this machine: keep any prebuilt copy
    from torch.utils import cpp_extension

    os.makedirs(OUT, exist_ok=True)
    cpp_extension.load(
        name="cuhpx_remap",
        sources=srcs,
        build_directory=OUT,
        extra_cflags=["-O2"],
        extra_cuda_cflags=["-O2", "-gencode", "arch=compute_100a,code=sm_100a"],
        verbose=verbose,
    )
    return built_path()


def load():
    """Import the prebuilt reference module (None when it was not built)."""
    path = built_path()
    if not os.path.exists(path):
        return None
    import importlib.util

    import torch  # noqa: F401  (the module links against torch's libraries)

    spec = importlib.util.spec_from_file_location("cuhpx_remap", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=DEFAULT_REFERENCE)
    a = ap.parse_args()
    print(build(a.reference, verbose=True))
