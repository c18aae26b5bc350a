"""Build the reference pygrog C++ extension from its own sources into ``oracle/_ref``.

Test infrastructure only: the product never imports or links this.  The
resulting ``_pygrog_torch_ref`` module is the reference's own CPU
implementation of the seven native entry points bound in
``csrc/torch/module.cpp:54-87`` (``grog_interpolate``, ``scatter_add``,
``scatter_add_binned``, ``gather``, ``psf_scatter_scalar``,
``psf_scatter_outer``, ``psf_scatter_outer_basis``).  It is used

* to validate the oracle restatement (``oracle/``) and generate golden
  fixtures (``tests/golden/make_golden.py``), and
* as the timed reference CPU arm of ``bench.py --impl reference``.

Recipe: compile ``csrc/torch/{module,grog_interp,sparse_ops,toep_psf}.cpp``
directly (not the reference's CMake build) with ``torch.utils.cpp_extension``.
The reference's own JIT list omits ``toep_psf.cpp`` although ``module.cpp``
binds its symbols, so it is added here.  ``-DPYGROG_MARCH_NATIVE`` selects the
single-ISA CPU path of ``sparse_ops.cpp``; the ISA is pinned to AVX2+FMA
(instead of ``-march=native``) so the built module also runs on the GPU host.

Usage:  python oracle/build_ref.py [--src /root/reference]
"""

from __future__ import annotations

import argparse
import os
import pathlib
import sys

HERE = pathlib.Path(__file__).resolve().parent
OUT = HERE / "_ref"
MODULE_NAME = "_pygrog_torch_ref"
SOURCES = ("module.cpp", "grog_interp.cpp", "sparse_ops.cpp", "toep_psf.cpp")


def built_path() -> pathlib.Path | None:
    """Return the path of the built reference module, or None."""
    if not OUT.exists():
        return None
    for p in sorted(OUT.glob(f"{MODULE_NAME}*.so")):
        return p
    return None


# Where this recipe finds the reference checkout (its sources are compiled
# where they lie; override with PYGROG_REFERENCE).
DEFAULT_SRC = os.environ.get("PYGROG_REFERENCE", "/root/reference")


def source_root() -> pathlib.Path | None:
    """The reference checkout if its C++ sources are present, else None."""
    root = pathlib.Path(DEFAULT_SRC)
    return root if (root / "csrc" / "torch").exists() else None


def build(src_root: str = DEFAULT_SRC, verbose: bool = False) -> pathlib.Path:
    import torch.utils.cpp_extension as cpp_ext

    csrc = pathlib.Path(src_root) / "csrc" / "torch"
    if not csrc.exists():
        raise FileNotFoundError(f"reference sources not found at {csrc}")
    OUT.mkdir(parents=True, exist_ok=True)
    bdir = OUT / "build"
    bdir.mkdir(exist_ok=True)
    # The gcc first on some PATHs cannot link -fopenmp; /usr/bin/g++ can.
    if os.path.exists("/usr/bin/g++"):
        os.environ["CXX"] = "/usr/bin/g++"
        os.environ["CC"] = "/usr/bin/gcc"
    cpp_ext.load(
        name=MODULE_NAME,
        sources=[str(csrc / s) for s in SOURCES],
        extra_cflags=[
            "-O3",
            "-std=c++17",
            "-fopenmp",
            "-mavx2",
            "-mfma",
            "-DPYGROG_MARCH_NATIVE",
        ],
        extra_ldflags=["-fopenmp"],
        build_directory=str(bdir),
        verbose=verbose,
    )
    so = bdir / f"{MODULE_NAME}.so"
    dst = OUT / so.name
    dst.write_bytes(so.read_bytes())
    return dst


def load():
    """Import the built reference module (``import torch`` first)."""
    import importlib.machinery
    import importlib.util

    import torch  # noqa: F401  (the module links against libtorch)

    path = built_path()
    if path is None:
        raise ImportError("oracle/_ref is not built (run python oracle/build_ref.py)")
    loader = importlib.machinery.ExtensionFileLoader(MODULE_NAME, str(path))
    spec = importlib.util.spec_from_file_location(MODULE_NAME, str(path), loader=loader)
    mod = importlib.util.module_from_spec(spec)
    loader.exec_module(mod)
    return mod


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--src", default=DEFAULT_SRC)
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    p = build(a.src, a.verbose)
    print(p)
    sys.exit(0)
