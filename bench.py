"""Benchmark: GROG fused gridding forward + adjoint (samples*coils/s) on B200.

Workload (the 3-D roofline configuration): 192^3 grid, kooshball trajectory
of 20,000 spokes x 384 samples (golden means), 12 coils (32 seeded Gaussian
coils compressed to 12 by PCA of the calibration block), kernel width 2
sphere (kw = 4), shift table precision 1 (11^3 entries), oversampling 1.
A step is one fused forward (interpolate + EGROG weight + scatter onto the
grid) plus one adjoint (gather + conjugate-transposed shift) over the whole
trajectory.  value = N_samples * C / step time, inputs resident in HBM
(737 MB of samples, 679 MB of grid: both larger than L2, so no flush needed).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Under torchrun (N > 1) every rank runs an independent replica (the path
shards by reconstruction; no data-path collective) and the max time over
ranks is reported.
"""

from __future__ import annotations

import argparse
import json
import math
import os
import pathlib
import re
import subprocess
import sys
import threading
import time

import numpy as np

REPO = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(REPO))

N_SPOKES, N_READOUT, GRID_N, N_COILS_RAW, N_COILS = 20000, 384, 192, 32, 12
CPU_SAMPLE_SPOKES = 2000
C3_LANES = (8, 16, 64)  # parallel chains of the c3 batch graph to time (the fastest is reported)
METRIC = "GROG samples*coils/s fwd+adj (3-D kooshball 192^3, C=12)"
UNIT = "samples*coils/s"


def _dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""

    QUERY = (
        "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
        "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
        "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"
    )

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "20"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True,
            )
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except (FileNotFoundError, OSError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {
            "sm_mhz": float(np.median(sm)) if sm else None,
            "sm_max_mhz": max(smax) if smax else None,
            "reasons": sorted(reasons),
            "samples": len(sm),
        }


def _peaks():
    p = REPO / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            d = json.loads(p.read_text())
            return float(d["hbm_gbs"]), "measured"
        except Exception:  # noqa: BLE001
            pass
    return 6650.0, "fallback"


def _profile_traffic(kernel: str):
    """DRAM bytes per launch of ``kernel`` recorded from an ncu capture in profiles/."""
    for f in sorted((REPO / "profiles").glob("*.md")):
        for line in f.read_text().splitlines():
            m = re.match(rf"\s*[-*]?\s*traffic_per_launch\[{re.escape(kernel)}\]\s*[:=]\s*([0-9.eE+]+)", line)
            if m:
                return float(m.group(1)), f.name
    return None, None


def aggregate_replicas(ms: float, units_per_rank: float, dist=None, device=None) -> tuple[float, float]:
    """Whole-job numbers of N independent replicas: the step time is the
    maximum over ranks and the throughput is the units of all ranks divided
    by it (one process per GPU, no data-path collective; `dist` is
    ``torch.distributed`` with an initialised group, or None for one rank)."""
    if dist is None:
        return ms, units_per_rank / (ms / 1e3)
    import torch

    t = torch.tensor([ms, units_per_rank], dtype=torch.float64, device=device)
    mx = t.clone()
    dist.all_reduce(mx, op=dist.ReduceOp.MAX)
    tot = t.clone()
    dist.all_reduce(tot, op=dist.ReduceOp.SUM)
    max_ms = float(mx[0].item())
    return max_ms, float(tot[1].item()) / (max_ms / 1e3)


def build_workload(device, seed: int = 1001):
    """Plan + table + device-resident data for the 3-D configuration."""
    import torch

    from pygrog_b200.calib import GrogInterpolator
    from pygrog_b200.workloads import kooshball

    coords = kooshball(N_SPOKES, N_READOUT, GRID_N / 2.0)
    # a small plan first, so that the timed plan excludes one-time library and
    # context initialisation
    GrogInterpolator(shape=(GRID_N,) * 3, coords=kooshball(8, 32, GRID_N / 2.0), oversamp=1.0, kernel_width=2,
                     kernel_shape="sphere", device=device)
    torch.cuda.synchronize(device)
    t0 = time.perf_counter()
    g = GrogInterpolator(shape=(GRID_N,) * 3, coords=coords, oversamp=1.0, kernel_width=2,
                         kernel_shape="sphere", device=device)
    torch.cuda.synchronize(device)
    t1 = time.perf_counter()
    acr = make_acr3d(device, seed)
    t2 = time.perf_counter()
    g.calc_interp_table(acr, lamda=0.01, precision=1)
    torch.cuda.synchronize(device)
    g.setup_ms = {"plan": (t1 - t0) * 1e3, "table": (time.perf_counter() - t2) * 1e3}
    gen = torch.Generator(device=device).manual_seed(seed)
    N = N_SPOKES * N_READOUT
    data = torch.randn(1, N_COILS, N, dtype=torch.complex64, device=device, generator=gen)
    return g, coords, acr, data


def make_acr3d(device, seed: int):
    """Centre 24^3 of the k-space of 32 Gaussian-coil images of a random
    ellipsoid phantom, PCA-compressed to 12 virtual coils (host FP64 SVD)."""
    import torch

    n = GRID_N
    gen = torch.Generator(device="cpu").manual_seed(seed)
    ax = torch.linspace(-1, 1, n, device=device)
    z, y, x = torch.meshgrid(ax, ax, ax, indexing="ij")
    ph = torch.zeros(n, n, n, device=device)
    for _ in range(10):
        c = (torch.rand(3, generator=gen) * 1.2 - 0.6).tolist()
        a = (torch.rand(3, generator=gen) * 0.35 + 0.05).tolist()
        v = float(torch.rand(1, generator=gen) * 0.9 + 0.1)
        m = ((x - c[0]) / a[0]) ** 2 + ((y - c[1]) / a[1]) ** 2 + ((z - c[2]) / a[2]) ** 2 <= 1
        ph = ph + v * m
    acr = torch.empty(N_COILS_RAW, 24, 24, 24, dtype=torch.complex64)
    lo = (n - 24) // 2
    for k in range(N_COILS_RAW):
        u = torch.randn(3, generator=gen)
        u = (0.7 * u / u.norm()).tolist()
        bump = torch.exp(-((x - u[0]) ** 2 + (y - u[1]) ** 2 + (z - u[2]) ** 2) / (2 * 0.7**2))
        phase = float(torch.rand(1, generator=gen)) * 2 * math.pi
        img = (ph * bump).to(torch.complex64) * complex(math.cos(phase), math.sin(phase))
        k3 = torch.fft.fftshift(torch.fft.fftn(torch.fft.ifftshift(img), norm="ortho"))
        acr[k] = k3[lo:lo + 24, lo:lo + 24, lo:lo + 24].cpu()
    flat = acr.reshape(N_COILS_RAW, -1).to(torch.complex128)
    u, s, vh = torch.linalg.svd(flat, full_matrices=False)
    comp = u[:, :N_COILS].conj().T  # (12, 32)
    return (comp @ flat).reshape(N_COILS, 24, 24, 24).to(torch.complex64).numpy()


class Fp64Check:
    """FP64 restatement of the fused operator on the GPU (torch, complex128),
    chunked over the valid replicas: grid[c, cell] += w * (T[e] x)_c and its
    adjoint.  Used to report the relative L2 error of the measured path."""

    def __init__(self, g, N: int, C: int):
        import torch

        plan = g.plan
        self.kw = int(plan.target_idx.shape[-1])
        self.tgt = plan.target_idx.reshape(-1)
        sw = torch.sqrt(plan.weights.reshape(-1).clamp(min=0.0))
        self.rw = (sw * sw).double()
        self.idx = g._interp_idx.reshape(-1)
        self.T = g._interp_kernel.to(self.tgt.device).to(torch.complex128)
        self.valid = torch.nonzero(self.tgt >= 0).squeeze(1)
        self.N, self.C = N, C
        self.G = int(np.prod(plan.grid_shape))

    def forward(self, x):
        import torch

        x = x.to(torch.complex128)
        out = torch.zeros(self.C, self.G, dtype=torch.complex128, device=x.device)
        for s in range(0, self.valid.numel(), 1 << 20):
            r = self.valid[s:s + (1 << 20)]
            y = torch.einsum("nrc,cn->rn", self.T[self.idx[r]], x[:, r // self.kw]) * self.rw[r]
            out.index_add_(1, self.tgt[r], y)
        return out

    def adjoint(self, y):
        import torch

        y = y.to(torch.complex128)
        out = torch.zeros(self.C, self.N, dtype=torch.complex128, device=y.device)
        for s in range(0, self.valid.numel(), 1 << 20):
            r = self.valid[s:s + (1 << 20)]
            v = torch.einsum("nrc,rn->cn", self.T[self.idx[r]].conj(), y[:, self.tgt[r]]) * self.rw[r]
            out.index_add_(1, r // self.kw, v)
        return out

    @staticmethod
    def rel(a, b) -> float:
        import torch

        return float((a.to(torch.complex128) - b).norm() / b.norm())


def time_modes(g, data, modes, ref_fwd, chk, reps: int = 6, warm: int = 3) -> dict:
    """Forward / adjoint CUDA-event times and FP64 errors of several gridders."""
    import torch

    B, C, N = data.shape
    G = int(np.prod(g.plan.grid_shape))
    res = {}
    saved = getattr(g, "gridder_mode", None)
    for mode in modes:
        g.gridder_mode = mode
        g._brick_plans = None
        bp = g._brick(0)
        kg = torch.empty(B, C, G, dtype=torch.complex64, device=data.device)
        out = torch.empty(B, C, N, dtype=torch.complex64, device=data.device)
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        tf, ta = [], []
        for it in range(warm + reps):
            ev[0].record()
            bp.forward(data, kg)
            ev[1].record()
            bp.adjoint(kg, out)
            ev[2].record()
            torch.cuda.synchronize()
            if it >= warm:
                tf.append(ev[0].elapsed_time(ev[1]))
                ta.append(ev[1].elapsed_time(ev[2]))
        ef = chk.rel(kg[0], ref_fwd)
        ea = chk.rel(out[0], chk.adjoint(kg[0]))
        fm, am = float(np.median(tf)), float(np.median(ta))
        res[mode] = {"kernels": list(bp.kernel_names()), "fwd_ms": fm, "adj_ms": am,
                     "value": N * C * B / ((fm + am) / 1e3), "rel_err_fwd_vs_fp64": ef, "rel_err_adj_vs_fp64": ea}
        del kg, out
    g.gridder_mode = saved
    g._brick_plans = None
    return res


def coil_compress_c1(dev, reps: int = 5) -> dict:
    """The step before the path at the 3-D configuration: 32 raw coils of all
    7.68 M samples compressed to 12 virtual coils (FP64 covariance of every
    sample, host eigendecomposition, one HBM-bound compression pass)."""
    import torch

    from pygrog_b200 import _lib
    from pygrog_b200.utils import compression_matrix

    N = N_SPOKES * N_READOUT
    gen = torch.Generator(device=dev).manual_seed(7)
    raw = torch.randn(N_COILS_RAW, N, dtype=torch.complex64, device=dev, generator=gen)
    out = torch.empty(N_COILS, N, dtype=torch.complex64, device=dev)
    st = _lib.stream_ptr(dev)
    t0 = time.perf_counter()
    mat = compression_matrix(raw, N_COILS)
    torch.cuda.synchronize(dev)
    fit_s = time.perf_counter() - t0
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    ts = []
    for it in range(reps + 2):
        ev[0].record()
        _lib.call("pgb_coil_compress", raw.data_ptr(), N, N_COILS_RAW, N_COILS, 1, mat.data_ptr(), out.data_ptr(), st)
        ev[1].record()
        torch.cuda.synchronize(dev)
        if it >= 2:
            ts.append(ev[0].elapsed_time(ev[1]))
    ms = float(np.median(ts))
    ref = out.clone()
    ts = []
    for it in range(reps + 2):
        ev[0].record()
        _lib.call("pgb_coil_compress_tc", raw.data_ptr(), N, N_COILS_RAW, N_COILS, 1, mat.data_ptr(), out.data_ptr(),
                  st)
        ev[1].record()
        torch.cuda.synchronize(dev)
        if it >= 2:
            ts.append(ev[0].elapsed_time(ev[1]))
    ms_tc = float(np.median(ts))
    err_tc = float((out - ref).norm() / ref.norm())
    nbytes = N * (N_COILS_RAW + N_COILS) * 8
    peak, kind = _peaks()
    gbs, gbs_tc = nbytes / (ms / 1e3) / 1e9, nbytes / (ms_tc / 1e3) / 1e9
    del raw, out, ref
    return {"coils": [N_COILS_RAW, N_COILS], "samples": N, "algorithmic_bytes": nbytes,
            "fp32": {"kernel": "coil_compress_kernel<32>", "ms": ms, "achieved_gbs": gbs, "roofline_frac": gbs / peak},
            "bf16x3": {"kernel": "coil_compress_tc_kernel<32,2>", "ms": ms_tc, "achieved_gbs": gbs_tc,
                       "roofline_frac": gbs_tc / peak, "rel_err_vs_fp32_kernel": err_tc},
            "peak_source": kind, "fit_s_incl_fp64_covariance": fit_s,
            "tc_ms": ms_tc, "tc_gbs": gbs_tc, "tc_frac": gbs_tc / peak, "fp32_ms": ms, "tc_rel_err_vs_fp32": err_tc}


def cpu_baseline(coords, acr, spokes: int):
    """Reference CPU implementation timed on a bounded sample of the trajectory."""
    from oracle.ref_cpu import ReferenceCPU

    sub = coords[:spokes]
    rc = ReferenceCPU((GRID_N,) * 3, sub, 1.0, 2, "sphere", acr, 1, 0.01)
    rng = np.random.default_rng(7)
    data = (rng.standard_normal((N_COILS, sub.shape[0] * sub.shape[1]))
            + 1j * rng.standard_normal((N_COILS, sub.shape[0] * sub.shape[1]))).astype(np.complex64)
    rc.time_step(data, 1)  # warm-up
    dt = rc.time_step(data, 2)
    v = sub.shape[0] * sub.shape[1] * N_COILS / dt
    return {
        "value": v,
        "unit": UNIT,
        "cores": rc.threads,
        "kind": rc.kind,
        "sample": f"{spokes} of {N_SPOKES} spokes x {N_READOUT} samples, C={N_COILS}, fwd+adj, best of 2",
    }


def run_reference_arm(args):
    ws, rank, local = _dist_env()
    if rank != 0:
        return 0
    from pygrog_b200.workloads import kooshball

    coords = kooshball(N_SPOKES, N_READOUT, GRID_N / 2.0)
    rng = np.random.default_rng(1001)
    acr = (rng.standard_normal((N_COILS, 24, 24, 24)) + 1j * rng.standard_normal((N_COILS, 24, 24, 24))).astype(np.complex64)
    try:
        import torch

        if torch.cuda.is_available():
            dev = torch.device("cuda", local)
            acr = make_acr3d(dev, 1001)
    except Exception:  # noqa: BLE001
        pass
    from oracle.ref_cpu import ReferenceCPU

    spokes = CPU_SAMPLE_SPOKES
    sub = coords[:spokes]
    rc = ReferenceCPU((GRID_N,) * 3, sub, 1.0, 2, "sphere", acr, 1, 0.01)
    data = (rng.standard_normal((N_COILS, sub.shape[0] * sub.shape[1]))
            + 1j * rng.standard_normal((N_COILS, sub.shape[0] * sub.shape[1]))).astype(np.complex64)
    for _ in range(max(args.warmup, 1)):
        rc.time_step(data, 1)
    times = [rc.time_step(data, 1) for _ in range(args.steps)]
    t = float(np.mean(times))
    v = sub.shape[0] * sub.shape[1] * N_COILS / t
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": v,
        "unit": UNIT,
        "n_gpus": args.gpus,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": t * 1e3,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "c64",
        "data": "synthetic",
        "config": {"workload": "grog3d_kooshball_192c12_fwd_adj", "grid": [GRID_N] * 3,
                   "spokes": N_SPOKES, "readout": N_READOUT, "coils": N_COILS, "kw": 4, "precision": 1,
                   "reference_sample_spokes": spokes},
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": rc.threads, "kind": rc.kind,
                         "sample": f"{spokes} of {N_SPOKES} spokes per step (reference CPU path, "
                                   f"{rc.threads} threads)"},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_serving(dev, seconds: float, rate: float = 200.0, seed: int = 1004) -> dict:
    """Served GROG + CG-SENSE mix (c0, c2 and two c3 slices) on this GPU.

    Closed-loop capacity (all requests queued at t=0) of the batched server
    (8 frames per batch, 4 streams) and of the plain single-instance path
    (one request at a time, one stream), then an open loop of Poisson arrivals
    at ``rate`` per second for ``seconds`` with p50 / p95 / p99 latency."""
    import torch

    from pygrog_b200.serve import ReconProtocol, ReconServer, Request, poisson_arrivals
    from pygrog_b200.workloads import serving_protocols, subspace_protocol

    specs = serving_protocols(seed) + [subspace_protocol()]
    protos = {}
    for sp in specs:
        kw = dict(sp)
        name = kw.pop("name")
        protos[name] = ReconProtocol(name, kw.pop("shape"), kw.pop("coords"), kw.pop("acr"), kw.pop("smaps"),
                                     device=dev, **kw)
    names = list(protos)
    # 20% of the requests use the rank-4 subspace protocol, the rest spread evenly
    others = [k for k in names if not protos[k].subspace]
    prob = np.array([0.2 if protos[k].subspace else 0.8 / len(others) for k in names])
    rng = np.random.default_rng(seed)

    def make(n, arrivals=None):
        out = []
        for i in range(n):
            p = protos[names[int(rng.choice(len(names), p=prob))]]
            d = (torch.randn(p.data_shape, dtype=torch.complex64)).pin_memory()
            out.append(Request(i, p.name, float(arrivals[i]) if arrivals is not None else 0.0, d))
        return out

    n_closed = 400
    single = ReconServer(protos, mem_budget=150 << 30, max_batch=1, n_slots=1, device=dev)
    rep_single = single.run(make(n_closed), realtime=False)
    del single
    batched = ReconServer(protos, mem_budget=150 << 30, max_batch=8, n_slots=4, device=dev)
    rep_batched = batched.run(make(n_closed), realtime=False)
    arr = poisson_arrivals(rate, seconds, rng)
    rep_open = batched.run(make(len(arr), arr), realtime=True)
    return {
        "mix": {k: {"coils": p.C, "image": list(p.image_shape), "cg_iters": p.max_iter,
                     "samples": int(np.prod(p.spatial)), "share": float(prob[i])}
                for i, (k, p) in enumerate(protos.items())},
        "memory_budget_gb": 150,
        "closed_loop_recons_per_s": rep_batched["recons_per_s"],
        "single_instance_recons_per_s": rep_single["recons_per_s"],
        "batched_over_single": rep_batched["recons_per_s"] / rep_single["recons_per_s"],
        "open_loop": {"rate_per_s": rate, "seconds": seconds, **{k: rep_open[k] for k in
                      ("requests", "recons_per_s", "p50_ms", "p95_ms", "p99_ms", "mean_batch")}},
        "precision": "complex64 operators, FP64 CG scalars",
    }


def c3_batch(dev, n_slices: int = 64, seed: int = 1004) -> dict:
    """Config c3: ``n_slices`` uneven 2-D radial slices (spokes U{13..233}, readout
    U{256..768}, grid U{128..384}, coils U{8..32}), each GROG interpolation +
    SparseFFT adjoint + 20 CG iterations, reconstructed as one batch: one CUDA
    graph launch whose branches are the slices (``pygrog_b200.batch.UnevenBatch``),
    k-space from and images to page-locked host memory (the copies are graph
    nodes).  Wall time of the launch, best of 5; the previous path (independent
    requests on 4 streams, one graph per slice) is timed beside it."""
    import torch

    from pygrog_b200.batch import UnevenBatch
    from pygrog_b200.serve import ReconProtocol, ReconServer, Request
    from pygrog_b200.workloads import c3_protocols

    specs = c3_protocols(seed, n_slices)  # synthetic trajectories, phantoms and coil maps (not setup)
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    protos = {}
    for sp in specs:
        kw = dict(sp)
        name = kw.pop("name")
        protos[name] = ReconProtocol(name, kw.pop("shape"), kw.pop("coords"), kw.pop("acr"), kw.pop("smaps"),
                                     device=dev, **kw)
    torch.cuda.synchronize(dev)
    t_proto = time.perf_counter() - t0
    gen = torch.Generator().manual_seed(seed)
    host_in = [torch.randn(p.data_shape, dtype=torch.complex64, generator=gen).pin_memory() for p in protos.values()]
    best = None
    by_lanes = {}
    for lanes in C3_LANES:
        batch = UnevenBatch(list(protos.values()), dev, lanes=lanes)
        batch.host_in = host_in  # the caller's page-locked k-space, read by the graph's copies
        t1 = time.perf_counter()
        batch.capture()
        torch.cuda.synchronize(dev)
        t_capture = time.perf_counter() - t1
        walls = []
        for _ in range(6):  # first run warms
            t2 = time.perf_counter()
            batch.run()
            walls.append(time.perf_counter() - t2)
        by_lanes[str(lanes)] = min(walls[1:]) * 1e3
        if best is None or min(walls[1:]) < best[0]:
            best = (min(walls[1:]), lanes, t_capture)
        del batch
        torch.cuda.empty_cache()
    wall, lanes_best, t_capture = best
    sc = sum(p.C * int(np.prod(p.spatial)) for p in protos.values())
    cg_bytes = sum(p.max_iter * _cg_iter_bytes(int(np.prod(p.op.grid_shape)), int(np.prod(p.image_shape)), p.C)
                   for p in protos.values())
    peak, _ = _peaks()
    # the per-request path on 4 streams, for comparison
    server = ReconServer(protos, mem_budget=150 << 30, max_batch=1, n_slots=4, device=dev)
    data = {k: h for k, h in zip(protos, host_in)}
    prev = []
    for _ in range(3):
        reqs = [Request(i, k, 0.0, data[k]) for i, k in enumerate(protos)]
        prev.append(server.run(reqs, realtime=False)["wall_s"])
    del server
    torch.cuda.empty_cache()
    return {"slices": n_slices, "ms_per_batch": wall * 1e3, "lanes": lanes_best, "ms_by_lanes": by_lanes,
            "sample_coils": sc,
            "sample_coils_per_s": sc / wall, "recons_per_s": n_slices / wall, "cg_iters": 20,
            "cg_bytes": cg_bytes, "cg_gbs": cg_bytes / wall / 1e9, "cg_roofline_frac": cg_bytes / wall / 1e9 / peak,
            "setup_s": t_proto + t_capture, "protocols_s": t_proto, "capture_s": t_capture,
            "protocol_ms_per_slice": t_proto * 1e3 / n_slices,
            "per_request_streams_ms": min(prev[1:]) * 1e3, "mode": "one graph, slices as branches",
            "note": "wall time incl. host<->device copies; plans, tables, PSFs and the graph built in setup"}


def _cg_iter_bytes(G: int, img: int, C: int) -> int:
    """Algorithmic bytes of one CG iteration on the Toeplitz normal operator:
    coil expansion into the (padded) grid, the forward and inverse 2-D FFTs as
    two passes of read + write each, the PSF multiply, the crop + SENSE
    combine, and the CG vectors (dots and updates)."""
    grid_b = C * G * 8
    return (img * 8 + C * img * 8 + grid_b  # expand: x, maps in, padded coil grid out
            + 4 * grid_b + 2 * grid_b + G * 4 + 4 * grid_b  # FFT (2 passes), PSF (r + w, PSF), IFFT
            + 2 * C * img * 8 + 2 * img * 8  # crop + combine (coil images, maps), damp add
            + 8 * img * 8)  # CG: the dots and the x / r / p updates


def cg_sense_c2(dev, iters: int = 30) -> dict:
    """Config c2 (spiral 320^2, 16 coils, Toeplitz PSF on 640^2, 30 CG
    iterations): time per reconstruction (GROG interpolation + SparseFFT
    adjoint + the graph-replayed CG) and per CG iteration (the captured
    iterations alone), CUDA events; the iteration's roofline from the bytes
    its passes move: coil expansion into the padded grid, the forward and
    inverse 2-D FFTs (two passes each, read + write), the PSF multiply
    (read + write), the crop + coil combine, and the CG vector updates."""
    import torch

    from pygrog_b200.serve import ReconProtocol
    from pygrog_b200.workloads import serving_protocols

    sp = dict(serving_protocols()[1])
    name = sp.pop("name")
    p = ReconProtocol(name, sp.pop("shape"), sp.pop("coords"), sp.pop("acr"), sp.pop("smaps"), device=dev, **sp)
    p.prepare(1, 1, graphs=True)
    d = torch.randn((1, *p.data_shape), dtype=torch.complex64, device=dev)
    for _ in range(3):
        p.recon(d, 0)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize(dev)
    reps = 5
    e0.record()
    for _ in range(reps):
        p.recon(d, 0)
    e1.record()
    torch.cuda.synchronize(dev)
    ms = e0.elapsed_time(e1) / reps
    cg = p._solvers[0]  # the captured CG iterations alone (state from the last recon)
    e0.record()
    for _ in range(reps):
        cg.run(p.max_iter)
    e1.record()
    torch.cuda.synchronize(dev)
    ms_iter = e0.elapsed_time(e1) / reps / p.max_iter
    G = int(np.prod(p.op.grid_shape))
    img = int(np.prod(p.image_shape))
    C = p.C
    iter_bytes = _cg_iter_bytes(G, img, C)
    peak, _ = _peaks()
    gbs = iter_bytes / (ms_iter / 1e3) / 1e9
    return {"ms_per_recon": ms, "ms_per_iter": ms_iter, "cg_iters": p.max_iter, "coils": C,
            "grid": list(p.op.grid_shape), "iter_bytes": iter_bytes, "iter_gbs": gbs,
            "iter_roofline_frac": gbs / peak, "fft_gflop_per_iter": 2 * C * 5 * G * float(np.log2(G)) / 1e9,
            "note": "recon = GROG interpolate + SparseFFT adjoint + graph-replayed CG (Toeplitz normal)"}


def serve_sweep(dev, rates=(200.0, 300.0, 400.0, 600.0), seconds: float = 5.0, seed: int = 1004) -> dict:
    """Open-loop Poisson arrivals of the c4 mix at several rates, served by the
    batched server (8 frames per batch, 4 streams) and by the plain
    single-instance path (one request at a time, one stream): p50 / p95 / p99
    latency and served recons/s per rate."""
    import torch

    from pygrog_b200.serve import ReconProtocol, ReconServer, Request, poisson_arrivals
    from pygrog_b200.workloads import serving_protocols, subspace_protocol

    specs = serving_protocols(seed) + [subspace_protocol()]
    protos = {}
    for sp in specs:
        kw = dict(sp)
        name = kw.pop("name")
        protos[name] = ReconProtocol(name, kw.pop("shape"), kw.pop("coords"), kw.pop("acr"), kw.pop("smaps"),
                                     device=dev, **kw)
    names = list(protos)
    others = [k for k in names if not protos[k].subspace]
    prob = np.array([0.2 if protos[k].subspace else 0.8 / len(others) for k in names])
    rng = np.random.default_rng(seed)
    servers = {"batched": ReconServer(protos, mem_budget=150 << 30, max_batch=8, n_slots=4, device=dev),
               "single": ReconServer(protos, mem_budget=150 << 30, max_batch=1, n_slots=1, device=dev)}
    out = {}
    arrivals = {rate: poisson_arrivals(rate, seconds, rng) for rate in rates}
    # one page-locked k-space per protocol, shared by its requests (timing does not depend on the values)
    kspace = {k: torch.randn(p.data_shape, dtype=torch.complex64).pin_memory() for k, p in protos.items()}
    for kind, srv in servers.items():
        for rate in rates:
            arr = arrivals[rate]
            reqs = []
            for i, t in enumerate(arr):
                p = protos[names[int(rng.choice(len(names), p=prob))]]
                reqs.append(Request(i, p.name, float(t), kspace[p.name]))
            rep = srv.run(reqs, realtime=True)
            out[f"{kind}@{int(rate)}"] = {k: rep[k] for k in ("requests", "recons_per_s", "p50_ms", "p95_ms", "p99_ms",
                                                            "mean_batch")}
    return {"seconds_per_rate": seconds, "rates": list(rates), "results": out}


def _call_workloads():
    """(name, Workload, CG damp) of the per-call timings: configs c0 and c2."""
    from pygrog_b200.workloads import config0, config2

    return [("c0", config0(), 1e-2), ("c2", config2(), 1e-3)]


def time_calls(dev, reps: int = 5) -> dict:
    """Per-call device times of the public API on configs c0 and c2, inputs
    resident on the GPU: plan, table fit (host FP64 and device), interpolate,
    interpolate(grid=True), degrid, SparseFFT build (Toeplitz PSF), forward,
    adjoint, normal, solve(cg, 30).  One warm-up, then ``reps`` repeats, each
    bracketed by a synchronize; median and min in ms."""
    import torch

    from pygrog_b200.calib import GrogInterpolator
    from pygrog_b200.operator import SparseFFT

    def timed(fn, setup=None):
        """``fn(setup())`` after one warm-up; ``setup`` runs outside the timed region."""
        fn(setup()) if setup else fn()
        torch.cuda.synchronize(dev)
        ts = []
        for _ in range(reps):
            arg = setup() if setup else None
            torch.cuda.synchronize(dev)
            t0 = time.perf_counter()
            fn(arg) if setup else fn()
            torch.cuda.synchronize(dev)
            ts.append((time.perf_counter() - t0) * 1e3)
        return {"median_ms": float(np.median(ts)), "min_ms": float(np.min(ts))}

    out = {}
    for name, w, damp in _call_workloads():
        res = {}
        mk = lambda: GrogInterpolator(shape=w.shape, coords=w.coords, oversamp=w.oversamp,  # noqa: E731
                                      kernel_width=w.kernel_width, kernel_shape=w.kernel_shape, device=dev)
        res["plan"] = timed(mk)
        res["calc_interp_table"] = timed(
            lambda gi: gi.calc_interp_table(w.acr, lamda=w.lamda, precision=w.precision), setup=mk)
        res["calc_interp_table_device_fit"] = timed(
            lambda gi: gi.calc_interp_table(w.acr, lamda=w.lamda, precision=w.precision, fit_on_device=True),
            setup=mk)
        g = mk()
        g.calc_interp_table(w.acr, lamda=w.lamda, precision=w.precision)
        data = torch.from_numpy(w.data).to(dev)
        res["interpolate"] = timed(lambda: g.interpolate(data))
        res["interpolate_grid"] = timed(lambda: g.interpolate(data, grid=True))
        kg = g.grid(data)
        res["degrid"] = timed(lambda: g.degrid(kg))
        smaps = torch.from_numpy(w.smaps.astype(np.complex64)).to(dev)
        res["sparsefft_build_toeplitz"] = timed(lambda: SparseFFT(plan=g.plan, smaps=smaps, toeplitz=True))
        op = SparseFFT(plan=g.plan, smaps=smaps, toeplitz=True)
        sparse = torch.as_tensor(g.interpolate(data))
        b = sparse * g.plan.pre_weights.unsqueeze(0)
        x = op.adjoint(b)
        res["forward"] = timed(lambda: op.forward(x))
        res["adjoint"] = timed(lambda: op.adjoint(b))
        res["normal"] = timed(lambda: op.normal(x))
        bn = b.reshape(b.shape[0], *op.natural_shape)
        res["solve_cg30"] = timed(lambda: op.solve(bn, method="cg", max_iter=30, damp=damp, tol=0.0))
        out[name] = {"shape": list(w.shape), "coils": int(w.data.shape[0]), "samples": int(np.prod(w.data.shape[1:])),
                     "calls": res}
        del g, op
        torch.cuda.empty_cache()
    return out


def chain_compare(dev, n_rep: int = 7_680_208, coils=(12, 32), reps: int = 5, seed: int = 1007) -> dict:
    """The eigen-factored shift chain alone (``pgb_shift_chain``) with mma.sync and
    with tcgen05 (accumulator in tensor memory), on ``n_rep`` replicas (the c1
    valid-replica count) at 12 and 32 coils: CUDA-event time of one launch
    applying the chain once and four times (best of ``reps``), the chain's own
    time per application ((t4 - t1) / 3, loads and stores excluded), and the
    relative error of the single chain against an FP64 restatement on every
    997th replica.  Random unitary W and unit-modulus phases keep repeated
    chains bounded."""
    import torch

    from pygrog_b200.calib import _chain

    rng = np.random.default_rng(seed)
    res = {"replicas": n_rep}
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    for C in coils:
        W = np.stack([np.linalg.qr(rng.standard_normal((C, C)) + 1j * rng.standard_normal((C, C)))[0]
                      for _ in range(4)])
        ph = np.exp(1j * rng.uniform(-np.pi, np.pi, (3, _chain.STEPS, C)))
        Wd, phd = _chain.chain_operands(W, ph, dev)
        gen = torch.Generator(device=dev).manual_seed(seed + C)
        x = torch.randn(2 * C, n_rep, device=dev, generator=gen)
        ijk = torch.randint(0, _chain.STEPS, (3, n_rep), device=dev, generator=gen)
        idx = _chain.pack_shift_indices(ijk)
        out = torch.empty_like(x)
        rows = np.arange(0, n_rep, 997)
        xs = x[:, rows].double().cpu().numpy()
        y = xs[0::2] + 1j * xs[1::2]
        ii = ijk[:, rows].cpu().numpy()
        for s in range(4):
            y = W[s] @ y
            if s < 3:
                y = y * ph[s][ii[s]].T
        for variant in ("mma", "tcgen05"):
            key = f"c{C}_{variant}"
            t = torch.zeros(1, dtype=torch.int32, device=dev)
            for rep in (1, 4):
                ts = []
                for it in range(reps + 2):
                    ev[0].record()
                    _chain.shift_chain(x, idx, Wd, phd, out, rep=rep, variant=variant, timeouts=t)
                    ev[1].record()
                    torch.cuda.synchronize(dev)
                    if it >= 2:
                        ts.append(ev[0].elapsed_time(ev[1]))
                res[f"{key}_rep{rep}_ms"] = min(ts)
                if rep == 1:
                    o = out[:, rows].double().cpu().numpy()
                    res[f"{key}_rel_err_vs_fp64"] = float(np.linalg.norm(o[0::2] + 1j * o[1::2] - y) / np.linalg.norm(y))
            _chain.check_timeouts(t)
            res[f"{key}_chain_ms"] = (res[f"{key}_rep4_ms"] - res[f"{key}_rep1_ms"]) / 3
        res[f"c{C}_tcgen05_speedup"] = res[f"c{C}_mma_chain_ms"] / res[f"c{C}_tcgen05_chain_ms"]
        del x, out, idx, ijk
        torch.cuda.empty_cache()
    return res


def _r(v, nd=4):
    """Round floats for the one-line summary (None and non-floats pass)."""
    return float(f"{v:.{nd}g}") if isinstance(v, float) else v


def _rounded(d, nd=5):
    """``d`` with its float values (one level deep) rounded for the one-line summary."""
    if not isinstance(d, dict):
        return _r(d, nd)
    return {k: _r(v, nd) for k, v in d.items()}


def _compact_modes(modes):
    """{mode: [fwd_ms, adj_ms, rel_err_fwd, rel_err_adj]} of the precision comparison."""
    if not isinstance(modes, dict) or "error" in modes:
        return modes
    return {m: [_r(v["fwd_ms"]), _r(v["adj_ms"]), _r(v["rel_err_fwd_vs_fp64"], 2), _r(v["rel_err_adj_vs_fp64"], 2)]
            for m, v in modes.items()}


def _compact_sections(coilc, cg2, c3, serving, tune):
    """Headline numbers of the secondary sections, short enough for one line."""
    out = {}

    def pick(d, keys):
        if not isinstance(d, dict):
            return d
        if "error" in d:
            return {"error": str(d["error"])[:160]}
        return {k: _r(d[k]) for k in keys if k in d}

    out["coil_compress_c1"] = pick(coilc, ("tc_ms", "tc_gbs", "tc_frac", "fp32_ms", "tc_rel_err_vs_fp32"))
    out["cg_sense_c2"] = pick(cg2, ("ms_per_recon", "ms_per_iter", "iter_gbs", "iter_roofline_frac"))
    out["c3_batch"] = pick(c3, ("ms_per_batch", "recons_per_s", "cg_roofline_frac", "protocol_ms_per_slice",
                                "capture_s", "per_request_streams_ms"))
    if isinstance(serving, dict) and "error" not in serving:
        o = serving.get("open_loop", {})
        out["serving"] = {k: _r(serving.get(k)) for k in ("closed_loop_recons_per_s", "single_instance_recons_per_s",
                                                         "batched_over_single")}
        out["serving"].update({k: _r(o.get(k)) for k in ("rate_per_s", "p50_ms", "p95_ms", "p99_ms", "mean_batch")})
    else:
        out["serving"] = pick(serving, ())
    if tune:
        out["autotune"] = {"mode": tune.get("mode"), "brick": tune.get("brick"), "ms": _r(tune.get("ms"))}
    return out


def main():
    global N_SPOKES, N_READOUT, GRID_N, N_COILS
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--table-mode", default="tc",
                    choices=["auto", "tc", "tc1", "v8", "v8pair", "v6", "global"],
                    help="gridder: tc = tensor-core bf16x3 (default), tc1 = bf16, v8 = FP32 CUDA cores, auto")
    ap.add_argument("--no-precision-modes", action="store_true", help="skip the FP32 / bf16 comparison")
    ap.add_argument("--autotune", action="store_true",
                    help="report the gridder autotuner's trials (families x bricks) on this workload")
    ap.add_argument("--spokes", type=int, default=N_SPOKES, help="smaller cases for profiling only")
    ap.add_argument("--readout", type=int, default=N_READOUT)
    ap.add_argument("--grid", type=int, default=GRID_N)
    ap.add_argument("--coils", type=int, default=N_COILS, help=f"virtual coils after PCA of {N_COILS_RAW} (1..32)")
    ap.add_argument("--serve-seconds", type=float, default=5.0, help="open-loop serving duration (0: skip)")
    ap.add_argument("--c3-slices", type=int, default=64, help="slices of the c3 batch (0: skip)")
    ap.add_argument("--calls", action="store_true",
                    help="only time the public API call by call on configs c0 and c2 (one JSON line)")
    ap.add_argument("--coil-only", action="store_true",
                    help="only time the coil compression (32 -> --coils) of --spokes x --readout samples (one JSON line)")
    ap.add_argument("--chain", action="store_true",
                    help="only time the shift chain alone, mma.sync against tcgen05, at 12 and 32 coils (one JSON line)")
    ap.add_argument("--chain-replicas", type=int, default=7_680_208, help="replicas of --chain (default: c1's valid replicas)")
    ap.add_argument("--chain-coils", default="12,32", help="coil counts of --chain (12 and / or 32)")
    ap.add_argument("--serve-sweep", action="store_true",
                    help="only sweep open-loop arrival rates of the served mix, batched vs single-instance (one JSON line)")
    ap.add_argument("--details", default=None,
                    help="also write the full per-section results (precision modes, serving, c2, c3) to this file")
    args = ap.parse_args()
    resized = (args.spokes, args.readout, args.grid, args.coils) != (N_SPOKES, N_READOUT, GRID_N, N_COILS)
    if not 1 <= args.coils <= N_COILS_RAW:
        ap.error(f"--coils must be 1..{N_COILS_RAW}")
    N_SPOKES, N_READOUT, GRID_N, N_COILS = args.spokes, args.readout, args.grid, args.coils
    if args.warmup < 3 and args.impl == "b200":
        args.warmup = 3
    if args.impl == "reference":
        return run_reference_arm(args)

    import torch

    ws, rank, local = _dist_env()
    dist = None
    if ws > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    if args.coil_only:
        if rank == 0:
            r = coil_compress_c1(dev)
            print(json.dumps({"coil_compress": {k: v for k, v in r.items() if not isinstance(v, dict)},
                              "samples": N_SPOKES * N_READOUT}), flush=True)
        return 0
    if args.chain:
        if rank == 0:
            coils = tuple(int(c) for c in args.chain_coils.split(","))
            r = chain_compare(dev, n_rep=args.chain_replicas, coils=coils)
            print(json.dumps({"shift_chain": {k: _r(v) for k, v in r.items()},
                              "device": torch.cuda.get_device_name(dev)}), flush=True)
        return 0
    if args.serve_sweep:
        if rank == 0:
            print(json.dumps({"serve_sweep": serve_sweep(dev), "device": torch.cuda.get_device_name(dev)}), flush=True)
        return 0
    if args.calls:
        if rank == 0:
            print(json.dumps({"calls": time_calls(dev), "device": torch.cuda.get_device_name(dev),
                              "inputs": "device-resident", "timing": "synchronize around each call"}), flush=True)
        return 0

    g, coords, acr, data = build_workload(dev)
    if args.table_mode and args.table_mode != "auto":
        g.gridder_mode = args.table_mode
    t0 = time.perf_counter()
    bp = g._brick(0)
    torch.cuda.synchronize(dev)
    g.setup_ms["gridder_plans"] = (time.perf_counter() - t0) * 1e3
    G = int(np.prod(g.plan.grid_shape))
    B, C, N = data.shape
    kgrid = torch.empty(B, C, G, dtype=torch.complex64, device=dev)
    out = torch.empty(B, C, N, dtype=torch.complex64, device=dev)
    stream = torch.cuda.current_stream(dev)

    def step(evs=None):
        if evs is not None:
            evs[0].record(stream)
        bp.forward(data, kgrid)
        if evs is not None:
            evs[1].record(stream)
        bp.adjoint(kgrid, out)
        if evs is not None:
            evs[2].record(stream)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize(dev)

    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(args.steps)]
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize(dev)
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    t_start.record(stream)
    for k in range(args.steps):
        step(evs[k])
    t_end.record(stream)
    torch.cuda.synchronize(dev)
    if dist is not None:
        dist.barrier()
    clocks = sampler.stop()
    total_ms = t_start.elapsed_time(t_end)
    fwd_ms = float(np.mean([e[0].elapsed_time(e[1]) for e in evs]))
    adj_ms = float(np.mean([e[1].elapsed_time(e[2]) for e in evs]))
    ms = total_ms / args.steps
    ms, value = aggregate_replicas(ms, float(N * C * B), dist, dev)

    # algorithmic bytes per launch (both directions): samples + per-replica metadata + grid
    alg_bytes = N * C * 8 * B + bp.n_valid * 12 + G * C * 8 * B
    k_fwd, k_adj = bp.kernel_names()
    dom = k_fwd if fwd_ms >= adj_ms else k_adj
    dom_ms = max(fwd_ms, adj_ms)
    peak, peak_kind = _peaks()
    achieved = alg_bytes / (dom_ms / 1e3) / 1e9
    # DRAM traffic per launch from the committed launch-list profile of the default workload
    traffic, tsrc = _profile_traffic(dom) if not resized else (None, None)
    n_launch = bp.launches_per_call(False) + bp.launches_per_call(True)

    # end to end through the public API with host buffers (pinned)
    e2e = None
    if args.e2e_steps > 0:
        x_host = data[0].cpu().reshape(C, N_SPOKES, N_READOUT).pin_memory()
        torch.cuda.synchronize(dev)
        kg = g.grid(x_host)
        g.degrid(kg)
        torch.cuda.synchronize(dev)
        ts = []
        for _ in range(args.e2e_steps):
            t0 = time.perf_counter()
            kg = g.grid(x_host)  # H2D samples, fused forward, D2H grid
            y = g.degrid(kg)  # H2D grid, fused adjoint, D2H samples
            torch.cuda.synchronize(dev)
            ts.append(time.perf_counter() - t0)
        t_e2e = float(np.median(ts))
        e2e = {
            "value": ws * N * C / t_e2e,
            "unit": UNIT,
            "h2d_bytes_per_step": int(x_host.numel() * 8 + kg.numel() * 8),
            "d2h_bytes_per_step": int(kg.numel() * 8 + y.numel() * 8),
            "api": "GrogInterpolator.grid(pinned host tensor) + GrogInterpolator.degrid(host tensor)",
        }

    # relative L2 error of the measured path against an FP64 restatement, and
    # the FP32 CUDA-core / plain bf16 gridders on the same data
    chk = Fp64Check(g, N, C)
    ref_fwd = chk.forward(data[0])
    accuracy = {"rel_err_fwd_vs_fp64": chk.rel(kgrid[0], ref_fwd),
                "rel_err_adj_vs_fp64": chk.rel(out[0], chk.adjoint(kgrid[0])),
                "tolerance": 1e-4}
    modes = None
    if ws == 1 and not args.no_precision_modes:
        try:
            fp32 = "v8" if N_COILS <= 16 else "global"  # the shared-memory FP32 families stop at 16 coils
            modes = time_modes(g, data, [fp32, "tc", "tc1"], ref_fwd, chk)
        except Exception as exc:  # noqa: BLE001
            modes = {"error": f"{type(exc).__name__}: {exc}"}
    del ref_fwd, chk
    torch.cuda.empty_cache()
    tune = None
    if args.autotune and ws == 1:
        from pygrog_b200.calib import autotune_gridder

        saved_mode = getattr(g, "gridder_mode", None)
        tune = autotune_gridder(g, batch=B, tolerance=1e-4, reps=3)
        tune["trials"] = [[m, list(b), t, e] for m, b, t, e in tune["trials"]]
        tune["rejected"] = [[m, list(b), e] for m, b, e in tune["rejected"]]
        tune["brick"] = list(tune["brick"])
        g.gridder_mode, g.gridder_brick, g._brick_plans = saved_mode, None, None
        torch.cuda.empty_cache()

    coilc = None
    if ws == 1 and not resized:
        try:
            coilc = coil_compress_c1(dev)
        except Exception as exc:  # noqa: BLE001
            coilc = {"error": f"{type(exc).__name__}: {exc}"}
        torch.cuda.empty_cache()

    serving = cg2 = c3 = None
    if ws == 1 and args.serve_seconds > 0 and not resized:
        try:
            cg2 = cg_sense_c2(dev)
            serving = run_serving(dev, args.serve_seconds)
        except Exception as exc:  # noqa: BLE001
            serving = {"error": f"{type(exc).__name__}: {exc}"}
    if ws == 1 and args.c3_slices > 0 and not resized:
        try:
            c3 = c3_batch(dev, args.c3_slices)
        except Exception as exc:  # noqa: BLE001
            c3 = {"error": f"{type(exc).__name__}: {exc}"}

    if rank == 0:
        cpu = None
        if ws == 1 and not args.no_cpu_baseline:
            try:
                cpu = cpu_baseline(coords, acr, CPU_SAMPLE_SPOKES)
            except Exception as exc:  # noqa: BLE001
                cpu = {"value": None, "unit": UNIT, "cores": os.cpu_count(), "kind": "unavailable",
                       "sample": f"failed: {exc}"}
        details = {"precision_modes": modes, "autotune": tune, "coil_compress_c1": coilc, "cg_sense_c2": cg2,
                   "c3_batch": c3, "serving": serving}
        if args.details:
            pathlib.Path(args.details).write_text(json.dumps(details, indent=1))
        line = {
            "metric": METRIC if not resized else METRIC.replace("192^3, C=12", f"{GRID_N}^3, C={N_COILS}"),
            "value": value,
            "unit": UNIT,
            "n_gpus": ws,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": ms,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": {"tc": "bf16x3 (fp32 accumulate)", "tc1": "bf16 (fp32 accumulate)"}.get(bp.mode, "fp32"),
            "data": "synthetic",
            "config": {
                "workload": (f"grog3d_kooshball_{GRID_N}c{N_COILS}_{N_SPOKES}x{N_READOUT}_fwd_adj" if resized
                             else "grog3d_kooshball_192c12_fwd_adj"),
                "grid": [GRID_N] * 3, "spokes": N_SPOKES, "readout": N_READOUT, "coils": N_COILS,
                "kernel": "sphere w=2 (kw=4)", "precision": 1, "oversamp": 1.0,
                "n_valid_replicas": bp.n_valid, "table_mode": bp.mode, "kernels": list(bp.kernel_names()),
                "l2": f"inputs > L2 ({N * C * 8 / 1e6:.0f} MB samples, {G * C * 8 / 1e6:.0f} MB grid)",
                "parallelism": f"replicas x{ws}",
            },
            "roofline": _rounded({
                "bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_source": peak_kind,
                "algorithmic_bytes": alg_bytes,
                "traffic": traffic, "traffic_source": tsrc,
            }),
            "clocks": clocks,
            "gpu_launches": n_launch * args.steps,
            "e2e": _rounded(e2e),
            "cpu_baseline": _rounded(cpu),
            "fwd_ms": _r(fwd_ms),
            "adj_ms": _r(adj_ms),
            "setup_ms": {k: round(v, 1) for k, v in g.setup_ms.items()},
            "summary": _compact_sections(coilc, cg2, c3, serving, tune),
            # last, so that a reader keeping only the end of the output keeps them
            "precision_modes": _compact_modes(modes),
            "accuracy": _rounded(accuracy, 3),
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
