"""Oracle: CPU restatement of the reference GROG path (numpy).

TEST INFRASTRUCTURE ONLY.  Nothing in the product imports this module; only
``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg
call it, as the checker.  Parity status: pinned -- ``tests/golden/`` holds
fixtures produced by running the reference implementation itself
(``tests/golden/make_golden.py``), and ``tests/test_oracle_golden.py``
checks this module against them (integer keys bit-exact, floats to
tolerance).

Each function cites the reference (FiRMLAB-Pisa/pygrog) lines it follows.
Float32 semantics follow torch's CPU evaluation: one IEEE-rounded float32
operation per elementwise op, round-half-to-even, true division.
"""

from __future__ import annotations

import numpy as np

f32 = np.float32


# ---------------------------------------------------------------------------
# Plan (calib/_grog.py:1081-1277)
# ---------------------------------------------------------------------------
def kernel_offsets(ndim: int, width: int, shape: str) -> np.ndarray:
    """calib/_grog.py:1240-1277."""
    half = (width - 1) / 2.0
    axis = np.arange(width) - int(np.floor(half))
    mesh = np.meshgrid(*([axis] * ndim), indexing="ij")
    allo = np.stack([m.ravel() for m in mesh], axis=-1).astype(np.int32)
    s = shape.lower()
    if s in ("square", "cube"):
        return allo
    if s in ("circle", "sphere"):
        rad = np.sqrt((allo.astype(np.float32) ** 2).sum(axis=-1))
        return allo[rad <= half + 0.5]
    if s == "cross":
        return allo[(allo != 0).sum(axis=-1) <= 1]
    raise ValueError(shape)


def default_oversamp(ndim, oversamp):
    """calib/_grog.py:1306-1315."""
    if oversamp is None:
        oversamp = (1.0, 1.0) if ndim == 2 else (1.0, 1.0, 1.2)
    if np.isscalar(oversamp):
        oversamp = ndim * [oversamp]
    return tuple(oversamp)


def create_plan(shape, coords, oversamp=None, kernel_width=2, kernel_shape="circle"):
    """calib/_grog.py:1081-1234 (single, unstacked trajectory).

    Returns dict with grid_shape, target_idx (..., kw) int64, distances
    (..., kw, ndim) float32, weights (..., kw) float32.
    """
    coords = np.asarray(coords, dtype=np.float32)
    ndim = coords.shape[-1]
    if np.isscalar(shape):
        shape = ndim * [shape]
    shape = tuple(int(s) for s in shape)
    oversamp = default_oversamp(ndim, oversamp)
    grid_shape = tuple(int(np.ceil(s * o)) for s, o in zip(shape, oversamp))
    amp = [2 * (s - 1 - s // 2) for s in shape]
    cmax = np.abs(coords).reshape(-1, ndim).max(axis=0)
    cs = 0.5 * np.asarray(amp, dtype=np.float32) * coords / cmax  # float32 chain
    offs = kernel_offsets(ndim, kernel_width, kernel_shape)
    origins = np.asarray([-(s // 2) for s in shape], dtype=np.float32)
    steps = np.asarray(
        [(s - 1) / (gs - 1) if gs > 1 else 1.0 for s, gs in zip(shape, grid_shape)], dtype=np.float32
    )
    frac = (cs - origins) / steps
    nearest = np.rint(frac).astype(np.int32)
    tnd = nearest[..., None, :] + offs  # (..., kw, ndim) int32
    tcoord = origins + tnd.astype(np.float32) * steps
    dist = (tcoord - cs[..., None, :]).astype(np.float32)
    inb = ((tnd >= 0) & (tnd < np.asarray(grid_shape, dtype=np.int32))).all(axis=-1)
    ok = inb & (np.abs(dist) <= f32(0.5)).all(axis=-1)
    strides = np.asarray([int(np.prod(grid_shape[d + 1:])) for d in range(ndim)], dtype=np.int64)
    flat = (tnd.astype(np.int64) * strides).sum(axis=-1)
    flat[~ok] = -1
    G = int(np.prod(grid_shape))
    dg = dist / steps
    dsq = np.zeros(dg.shape[:-1], dtype=np.float32)
    for d in range(ndim):
        dsq = (dsq + dg[..., d] * dg[..., d]).astype(np.float32)
    gauss = np.exp(f32(-0.5) * dsq).astype(np.float32)
    gauss[~ok] = 0.0
    ft = flat.reshape(-1)
    fg = gauss.reshape(-1)
    v = ft >= 0
    gsum = np.zeros(G, dtype=np.float64)
    np.add.at(gsum, ft[v], fg[v].astype(np.float64))
    w = np.zeros_like(gauss)
    wf = w.reshape(-1)
    wf[v] = fg[v] / np.maximum(gsum[ft[v]], 1e-12).astype(np.float32)
    return dict(shape=shape, grid_shape=grid_shape, target_idx=flat, distances=dist, weights=w, kw=offs.shape[0])


def fft_plan(plan):
    """calib/_grog.py:918-998: sorted cell indices and sqrt-weights (stable sort)."""
    idx = plan["target_idx"].reshape(-1).astype(np.int64).copy()
    w = plan["weights"].reshape(-1).astype(np.float32)
    sw = np.sqrt(np.maximum(w, 0)).astype(np.float32)
    bad = idx < 0
    idx[bad] = 0
    sw[bad] = 0
    perm = np.argsort(idx, kind="stable")
    inv = np.empty_like(perm)
    inv[perm] = np.arange(perm.size)
    return dict(indices=idx[perm], sqrt_weights=sw[perm], sort_perm=perm, inv_perm=inv)


def quantize(distances, precision: int, nsteps: int, K: int, radius: float = 0.5) -> np.ndarray:
    """calib/_grog.py:406-417 in float32 (torch scalar ops cast the scalar to float32)."""
    pfac = f32(10.0**precision)
    step = f32(10 ** (-precision))
    d = distances.astype(np.float32)
    a = (np.rint((d * pfac).astype(np.float32)) / pfac).astype(np.float32)
    i = np.rint(((f32(radius) + a).astype(np.float32) / step).astype(np.float32))
    strides = np.asarray([nsteps**k for k in range(d.shape[-1])], dtype=np.float32)
    s = np.rint((i * strides).astype(np.float32)).astype(np.int32).astype(np.int64).sum(axis=-1)
    return np.clip(s, 0, K - 1)


# ---------------------------------------------------------------------------
# Table (calib/_grappa.py:16-367), numpy/scipy LAPACK
# ---------------------------------------------------------------------------
def _lstsq(A, B, lamda):
    """calib/_grappa.py:16-59 (gelsd on the augmented system)."""
    n = A.shape[-1]
    if lamda > 0:
        A = np.concatenate([A, (lamda**0.5) * np.eye(n, dtype=A.dtype)], axis=0)
        B = np.concatenate([B, np.zeros((n, B.shape[-1]), dtype=B.dtype)], axis=0)
    return np.linalg.lstsq(A, B, rcond=None)[0]


def _logm(G):
    """calib/_grappa.py:62-72 (complex128 eigendecomposition)."""
    vals, vecs = np.linalg.eig(G.astype(np.complex128))
    return (vecs @ np.diag(np.log(vals)) @ np.linalg.inv(vecs)).astype(G.dtype)


def _expm(A):
    from scipy.linalg import expm

    return expm(A)


def kernel_table(train, radius=0.5, precision=1, lamda=0.01):
    """calib/_grappa.py:75-181, 264-367: table (nsteps**ndim, C, C) in train's dtype."""
    t = np.asarray(train)
    dt = t.dtype
    t = t / np.linalg.norm(t.ravel())
    t = t.astype(dt)
    cal = np.moveaxis(t, 0, -1)
    nc = cal.shape[-1]
    ndim = cal.ndim - 1
    ops = []
    for ax in range(ndim):
        m = cal.shape[ax] - 1
        src = np.take(cal, np.arange(m), axis=ax).reshape(-1, nc)
        dst = np.take(cal, np.arange(1, m + 1), axis=ax).reshape(-1, nc)
        ops.append(_lstsq(src, dst, lamda).T)
    if ndim == 2:
        gx, gy, gz = ops[0], ops[1], None
    else:
        gx, gy, gz = ops[2], ops[1], ops[0]
    step = 10 ** (-precision)
    n = int(2 * radius / step + 1)
    deltas = ((np.arange(n, dtype=np.float32) - f32((n - 1) / 2)) * f32(step)).astype(np.float32)

    def powers(G):
        L = _logm(G)
        return np.stack([_expm(d * L) for d in deltas]).astype(dt)

    Px, Py = powers(gx), powers(gy)
    if ndim == 2:
        tab = np.einsum("jab,ibc->ijac", Px, Py).reshape(-1, nc, nc)
    else:
        Pz = powers(gz)
        xy = np.einsum("kab,jbc->jkac", Px, Py)
        tab = np.einsum("jkab,ibc->ijkac", xy, Pz).reshape(-1, nc, nc)
    return tab.astype(dt), n, ndim


# ---------------------------------------------------------------------------
# Interpolation, gridding, adjoint
# ---------------------------------------------------------------------------
def interpolate(data, interp_idx, table):
    """calib/_grog.py:668-695 + grog_interp.cpp:39-73.

    data (B, C, N) -> replicas (B, C, N*kw): out[b,:,n*kw+j] = T[idx[n,j]] @ data[b,:,n].
    """
    B, C, N = data.shape
    idx = interp_idx.reshape(N, -1)
    kw = idx.shape[1]
    T = table[idx.reshape(-1)]  # (N*kw, C, C)
    x = np.repeat(data, kw, axis=-1)  # (B, C, N*kw)
    return np.einsum("rij,bjr->bir", T, x)


def grid(data, interp_idx, table, plan, fplan):
    """interpolate(grid=True): calib/_grog.py:736-902.

    kgrid[b, c, cell] = sum_r pre_w[r] * sqrt_w_sorted * (T x)_r; returns
    (kgrid (B, C, G), density (G,)).
    """
    rep = interpolate(data, interp_idx, table)
    B, C, R = rep.shape
    pre_w = fplan["sqrt_weights"][fplan["inv_perm"]]
    dc = rep * pre_w
    G = int(np.prod(plan["grid_shape"]))
    out = np.zeros((B, C, G), dtype=np.result_type(data.dtype, np.complex64))
    idx = fplan["indices"]
    sw = fplan["sqrt_weights"]
    for b in range(B):
        for c in range(C):
            np.add.at(out[b, c], idx, dc[b, c][fplan["sort_perm"]] * sw)
    dens = np.zeros(G, dtype=np.float32)
    np.add.at(dens, idx, sw * sw)
    return out, dens


def degrid(kgrid, interp_idx, table, plan):
    """Adjoint of ``grid`` (no reference counterpart; restated from the
    definition): x[b,:,n] = sum_{valid j} w[n,j] * T[idx[n,j]]^H @ kgrid[b,:,cell[n,j]],
    with w = sqrt_w**2 and sqrt_w = float32 sqrt(clamp(weights, 0)), the
    same per-replica factor the forward applies (pre_weights * sqrt_weights)."""
    B, C, G = kgrid.shape
    tgt = plan["target_idx"].reshape(-1)
    sw = np.sqrt(np.maximum(plan["weights"].reshape(-1), 0)).astype(np.float32).astype(np.float64)
    w = sw * sw
    kw = plan["kw"]
    N = tgt.size // kw
    idx = interp_idx.reshape(-1)
    out = np.zeros((B, C, N), dtype=np.complex128)
    v = np.nonzero(tgt >= 0)[0]
    TH = np.conj(np.swapaxes(table[idx[v]], -1, -2)).astype(np.complex128)
    for b in range(B):
        g = kgrid[b][:, tgt[v]].astype(np.complex128)  # (C, nv)
        contrib = np.einsum("rij,jr->ir", TH, g) * w[v]
        np.add.at(out[b].T, v // kw, contrib.T)
    return out


# ---------------------------------------------------------------------------
# L0 primitives (csrc/torch/sparse_ops*.cpp, toep_psf.cpp)
# ---------------------------------------------------------------------------
def scatter_add(grid_, data, idx, w):
    """sparse_ops_cpu_impl.inl:38-120: grid[idx] += w*data (idx outside [0,G) skipped)."""
    g = grid_.copy()
    ok = (idx >= 0) & (idx < g.size)
    np.add.at(g, idx[ok], (w * data)[ok])
    return g


def gather(grid_, idx, w):
    """sparse_ops_cpu_impl.inl:125-168."""
    out = np.zeros(idx.shape, dtype=grid_.dtype)
    ok = (idx >= 0) & (idx < grid_.size)
    out[ok] = w[ok] * grid_[idx[ok]]
    return out


def psf_scalar(G, idx, wsq):
    """toep_psf.cpp:80-118."""
    p = np.zeros(G, dtype=wsq.dtype)
    np.add.at(p, idx, wsq)
    return p


def psf_outer(G, M, idx, wsq, basis):
    """toep_psf.cpp:124-175."""
    p = np.zeros((G, M, M), dtype=basis.dtype)
    o = np.einsum("ni,nj->nij", basis.conj(), basis) * wsq[:, None, None]
    np.add.at(p, idx, o)
    return p


def psf_outer_basis(G, K, idx, wsq, basis, tix):
    """toep_psf.cpp:181-237."""
    bn = basis[:, tix].T
    return psf_outer(G, K, idx, wsq, bn)
