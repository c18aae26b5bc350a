"""Build ``libpygrog_b200.so`` (sm_100a) in-tree with nvcc.

The library is a plain C-ABI shared object (see ``include/pygrog_b200.h``);
it has no torch dependency.  Output: ``pygrog_b200/_lib/libpygrog_b200.so``.

    python -m pygrog_b200.csrc.build [--force] [--verbose]
"""

from __future__ import annotations

import argparse
import os
import pathlib
import shutil
import subprocess
import sys

CSRC = pathlib.Path(__file__).resolve().parent
PKG = CSRC.parent
REPO = PKG.parent
OUT_DIR = PKG / "_lib"
LIB = OUT_DIR / "libpygrog_b200.so"
SOURCES = ["l0_ops.cu", "plan.cu", "grog_fused.cu", "grog_v6.cu", "grog_v8.cu", "grog_tc.cu", "coil.cu", "fft_stage.cu", "solver.cu", "lsmr.cu", "subspace.cu", "plan_pack.cu", "shift_chain.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    deps = list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cuh")) + [REPO / "include" / "pygrog_b200.h"]
    return any(p.stat().st_mtime > t for p in deps if p.exists())


def build(force: bool = False, verbose: bool = False, extra: list[str] | None = None) -> pathlib.Path:
    """Compile every CUDA source for sm_100a and link the shared library."""
    if not force and not _stale():
        return LIB
    OUT_DIR.mkdir(parents=True, exist_ok=True)
    objdir = OUT_DIR / "obj"
    objdir.mkdir(exist_ok=True)
    nvcc = _nvcc()
    flags = ARCH + [
        "-O3",
        "-lineinfo",
        "-std=c++17",
        "-Xcompiler",
        "-fPIC",
        "-Xcompiler",
        "-fvisibility=hidden",
        "--expt-relaxed-constexpr",
        f"-I{REPO / 'include'}",
    ] + (extra or [])
    objs = []
    procs = []
    for src in SOURCES:
        obj = objdir / (src + ".o")
        cmd = [nvcc, *flags, "-c", str(CSRC / src), "-o", str(obj)]
        if verbose:
            print(" ".join(cmd))
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
        objs.append(obj)
    failed = []
    for src, p in procs:
        out, _ = p.communicate()
        txt = out.decode(errors="replace")
        if p.returncode != 0:
            failed.append(f"--- {src} ---\n{txt}")
        elif verbose and txt.strip():
            print(txt)
    if failed:
        raise RuntimeError("nvcc failed:\n" + "\n".join(failed))
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [nvcc, *ARCH, "-shared", "-o", str(tmp), *map(str, objs), "-lcudart_static"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("link failed:\n" + r.stdout + r.stderr)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas-v", action="store_true", help="print register/smem usage")
    a = ap.parse_args()
    extra = ["-Xptxas", "-v"] if a.ptxas_v else None
    print(build(force=a.force or a.ptxas_v, verbose=a.verbose or a.ptxas_v, extra=extra))
    sys.exit(0)
