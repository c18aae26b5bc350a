"""Per-call CPU timings of the reference's own implementation on configs c0 and c2.

BASELINE INFRASTRUCTURE ONLY: runs where the reference checkout is present
(it imports the reference package through ``tests/golden/refimport.py``, with
its C++ kernels built from source into ``oracle/_ref``), never on the product
path.  The GPU counterpart is ``python bench.py --calls``; both take their
inputs from ``pygrog_b200.workloads.config0`` / ``config2``.

Calls (reference API, ``calib/_grog.py``, ``operator/_sparse_fft.py``):
``GrogInterpolator(...)`` (plan), ``calc_interp_table``, ``interpolate(data)``,
``interpolate(data, grid=True)``, ``SparseFFT(plan, smaps, toeplitz=True)``
(PSF build), ``forward``, ``adjoint``, ``normal``, ``solve(cg, 30)``.  The
reference has no adjoint of the GROG shift (degrid), so none is timed.
One warm-up, then ``reps`` repeats; median and min in ms; all host threads.

Usage: ``python oracle/time_reference_calls.py [--reps 5]`` (prints one JSON line).
"""

from __future__ import annotations

import argparse
import json
import os
import pathlib
import platform
import sys
import time

import numpy as np

REPO = pathlib.Path(__file__).resolve().parent.parent


def _timed(fn, reps, setup=None):
    """``fn(setup())`` timed after one warm-up; ``setup`` runs outside the timed region."""
    arg = setup() if setup else None
    fn(arg) if setup else fn()
    ts = []
    for _ in range(reps):
        arg = setup() if setup else None
        t0 = time.perf_counter()
        fn(arg) if setup else fn()
        ts.append((time.perf_counter() - t0) * 1e3)
    return {"median_ms": float(np.median(ts)), "min_ms": float(np.min(ts))}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reps", type=int, default=5)
    args = ap.parse_args()
    sys.path.insert(0, str(REPO))
    sys.path.insert(0, str(REPO / "tests" / "golden"))
    import torch

    import refimport
    from pygrog_b200.workloads import config0, config2

    n = os.cpu_count() or 1
    torch.set_num_threads(n)
    pg = refimport.import_reference()
    out = {}
    for name, w, damp in (("c0", config0(), 1e-2), ("c2", config2(), 1e-3)):
        res = {}
        mk = lambda: pg.calib.GrogInterpolator(shape=w.shape, coords=w.coords, oversamp=w.oversamp,  # noqa: E731
                                               kernel_width=w.kernel_width, kernel_shape=w.kernel_shape)
        res["plan"] = _timed(mk, args.reps)
        g = mk()
        # the reference drops the plan's shifts after quantising them: a fresh interpolator per call
        res["calc_interp_table"] = _timed(
            lambda gi: gi.calc_interp_table(w.acr, lamda=w.lamda, precision=w.precision), args.reps, setup=mk)
        g.calc_interp_table(w.acr, lamda=w.lamda, precision=w.precision)
        data = w.data
        res["interpolate"] = _timed(lambda: g.interpolate(data), args.reps)
        res["interpolate_grid"] = _timed(lambda: g.interpolate(data, grid=True), args.reps)
        smaps = torch.from_numpy(w.smaps.astype(np.complex64))
        res["sparsefft_build_toeplitz"] = _timed(
            lambda: pg.operator.SparseFFT(plan=g.plan, smaps=smaps, toeplitz=True), args.reps)
        op = pg.operator.SparseFFT(plan=g.plan, smaps=smaps, toeplitz=True)
        sparse = torch.as_tensor(np.asarray(g.interpolate(data)))
        b = sparse * g.plan.pre_weights.unsqueeze(0)
        x = op.adjoint(b)
        res["forward"] = _timed(lambda: op.forward(x), args.reps)
        res["adjoint"] = _timed(lambda: op.adjoint(b), args.reps)
        res["normal"] = _timed(lambda: op.normal(x), args.reps)
        bn = b.reshape(b.shape[0], *op.natural_shape)
        res["solve_cg30"] = _timed(lambda: op.solve(bn, method="cg", max_iter=30, damp=damp, tol=0.0),
                                   max(1, args.reps // 2))
        out[name] = {"shape": list(w.shape), "coils": int(data.shape[0]), "samples": int(np.prod(data.shape[1:])),
                     "calls": res}
        print(name, json.dumps(res), file=sys.stderr, flush=True)
    print(json.dumps({"impl": "reference", "calls": out, "threads": n, "cpu": platform.processor() or platform.machine()}))


if __name__ == "__main__":
    main()
