"""Builds ``oracle/_ref/hs2_ref_corr*.so`` from the reference's correlation sources.

TEST INFRASTRUCTURE ONLY.  Compiles, unmodified and where they lie,
``src/correlation_kernels.cu`` and ``src/altcorr_kernel.cu`` of the HI-SLAM2
checkout (default ``/root/reference``) for sm_100a, with the binding in
``oracle/ref_corr_binding.cpp``.  Nothing is copied into the repository; the
output goes to ``oracle/_ref/`` (git-ignored) and is used by the GPU tests and
the fixture generator to pin the oracle against the reference's own kernels.

``src/droid_kernels.cu`` (ba, frame_distance) is not built: it includes Eigen,
which is absent from the checkout (empty ``thirdparty/eigen`` submodule).

Usage: ``python oracle/build_ref.py [--reference PATH]``.
"""

import argparse
import glob
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
NAME = "hs2_ref_corr"


def built_library():
    hits = sorted(glob.glob(os.path.join(OUT, NAME + "*.so")))
    return hits[0] if hits else None


def build(reference="/root/reference", verbose=False):
    src = os.path.join(reference, "src")
    sources = [os.path.join(src, "correlation_kernels.cu"), os.path.join(src, "altcorr_kernel.cu")]
    if not all(os.path.exists(s) for s in sources):
        return None
    os.makedirs(OUT, exist_ok=True)
    from torch.utils import cpp_extension
    os.environ.setdefault("TORCH_CUDA_ARCH_LIST", "10.0")
    cpp_extension.load(
        name=NAME,
        sources=[os.path.join(HERE, "ref_corr_binding.cpp")] + sources,
        build_directory=OUT,
        extra_cflags=["-O2"],
        extra_cuda_cflags=["-O3", "-gencode", "arch=compute_100a,code=sm_100a"],
        verbose=verbose,
        is_python_module=True,
    )
    return built_library()


def load():
    """Imports the built reference extension (needs torch and a GPU to call)."""
    path = built_library()
    if path is None:
        return None
    import importlib.machinery
    import importlib.util
    import torch  # noqa: F401  (the extension links against libtorch)
    loader = importlib.machinery.ExtensionFileLoader(NAME, path)
    spec = importlib.util.spec_from_file_location(NAME, path, loader=loader)
    mod = importlib.util.module_from_spec(spec)
    loader.exec_module(mod)
    return mod


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default="/root/reference")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    lib = build(a.reference, a.verbose)
    print(lib if lib else "reference sources not found; nothing built")
    sys.exit(0)
