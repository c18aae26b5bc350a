"""Import the reference ``pygrog`` package from its read-only checkout.

Only for this development container (the reference checkout does not travel
to the GPU host).  Used by ``make_golden.py`` to produce the committed golden
fixtures, and by the CPU tests that cross-check the oracle against the live
reference when the checkout is present (skipped otherwise).

Steps: build/load the reference C++ extension from source (``oracle/_ref``),
register it as ``pygrog._pygrog_torch``, put the ``mrinufft`` stand-in
(``refshim/``) and the reference ``src`` tree on ``sys.path``, import.
"""

from __future__ import annotations

import os
import pathlib
import sys

REF_ROOT = pathlib.Path(os.environ.get("PYGROG_REFERENCE", "/root/reference"))
HERE = pathlib.Path(__file__).resolve().parent
REPO = HERE.parent.parent


def available() -> bool:
    return (REF_ROOT / "src" / "pygrog" / "calib" / "_grog.py").exists()


def import_reference():
    """Return the reference ``pygrog`` package (CPU path, built from source)."""
    if "pygrog" in sys.modules and hasattr(sys.modules["pygrog"], "calib"):
        return sys.modules["pygrog"]
    if not available():
        raise ImportError(f"reference checkout not found at {REF_ROOT}")
    import torch  # noqa: F401

    sys.path.insert(0, str(REPO))
    from oracle import build_ref

    if build_ref.built_path() is None:
        build_ref.build(str(REF_ROOT))
    ext = build_ref.load()
    sys.modules["pygrog._pygrog_torch"] = ext
    shim = str(HERE / "refshim")
    if shim not in sys.path:
        sys.path.insert(0, shim)
    src = str(REF_ROOT / "src")
    if src not in sys.path:
        sys.path.insert(0, src)
    import pygrog  # noqa: F401

    return sys.modules["pygrog"]
