"""Builds ``oracle/_ref/hs2_ref_droid*.so``: HI-SLAM2's own ``droid_backends``
extension, compiled unmodified from the checkout's ``src/`` for sm_100a.

TEST INFRASTRUCTURE ONLY.  Compiles, where they lie, the reference's binding
``src/droid.cpp`` and its kernels ``src/droid_kernels.cu`` (ba, pgba,
frame_distance, proj_trans, covis_distance, depth_filter, iproj, bi_inter),
``src/correlation_kernels.cu`` and ``src/altcorr_kernel.cu``.  Eigen, which
``droid_kernels.cu`` includes (``:15-17``), is absent from the checkout (empty
``thirdparty/eigen`` submodule) and from this image, so the include path puts
the self-written dense stand-in ``oracle/eigen_standin/`` in its place (its
header states what it restates and how it differs: natural instead of AMD
ordering in the LLT).  Nothing is copied into the repository; the output goes to
``oracle/_ref/`` (git-ignored) and is used by the GPU tests and the fixture
generator to pin the numpy oracle against the reference's own operators.

The checkout is found at ``$HISLAM2_REFERENCE``, else at the default below.
Usage: ``python oracle/build_ref.py [--reference PATH] [-v]``.
"""

import argparse
import glob
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
NAME = "hs2_ref_droid"
STANDIN = os.path.join(HERE, "eigen_standin")
DEFAULT_REFERENCE = "/root/reference"


def reference_path(reference=None):
    return reference or os.environ.get("HISLAM2_REFERENCE") or DEFAULT_REFERENCE


def built_library():
    hits = sorted(glob.glob(os.path.join(OUT, NAME + "*.so")))
    return hits[0] if hits else None


def build(reference=None, verbose=False):
    """Returns the built library's path, or None when the checkout is absent."""
    src = os.path.join(reference_path(reference), "src")
    sources = [os.path.join(src, f) for f in ("droid.cpp", "droid_kernels.cu", "correlation_kernels.cu",
                                              "altcorr_kernel.cu")]
    if not all(os.path.exists(s) for s in sources):
        return None
    os.makedirs(OUT, exist_ok=True)
    from torch.utils import cpp_extension
    os.environ.setdefault("TORCH_CUDA_ARCH_LIST", "10.0")
    cpp_extension.load(
        name=NAME,
        sources=sources,
        build_directory=OUT,
        extra_include_paths=[STANDIN],
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
    ap.add_argument("--reference", default=None)
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    lib = build(a.reference, a.verbose)
    print(lib if lib else "reference sources not found; nothing built")
    sys.exit(0)
