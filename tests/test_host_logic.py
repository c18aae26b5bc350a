"""Host-side logic that needs no GPU: brick work plan, offsets, table fit."""

import numpy as np
import pytest
import torch

from conftest import golden, golden_plan_cases, parse_meta, rel_l2
from oracle import grog as og
from pygrog_b200.calib import _grog, _grappa


@pytest.mark.parametrize("ndim,width,shape", [(2, 2, "circle"), (2, 5, "square"), (3, 2, "sphere"),
                                             (3, 3, "cube"), (2, 3, "cross"), (3, 4, "cross")])
def test_kernel_offsets_match_oracle(ndim, width, shape):
    np.testing.assert_array_equal(_grog._kernel_offsets(ndim, width, shape), og.kernel_offsets(ndim, width, shape))


@pytest.mark.parametrize("ndim,dtype", [(2, np.float32), (3, np.float32), (3, np.float64)])
def test_coordinate_rescale_is_bit_exact_with_the_oracle(ndim, dtype):
    """The plan's coordinate rescale (a torch float32 chain, run on the GPU for
    plans) equals the oracle's numpy float32 chain bit for bit, float64 input
    cast to float32 first in both."""
    rng = np.random.default_rng(ndim)
    coords = (rng.uniform(-0.5, 0.5, (777, ndim)) * rng.uniform(0.3, 3.0)).astype(dtype)
    shape = (96, 80, 64)[:ndim]
    amp = [2 * (s - 1 - s // 2) for s in shape]
    c32 = np.asarray(coords, dtype=np.float32)
    want = 0.5 * np.asarray(amp, dtype=np.float32) * c32 / np.abs(c32).reshape(-1, ndim).max(axis=0)
    got = _grog._rescale_coords(torch.from_numpy(coords).to(torch.float32), amp).numpy()
    assert got.dtype == np.float32
    np.testing.assert_array_equal(got, want)


@pytest.mark.parametrize("case", golden_plan_cases())
def test_table_fit_matches_reference(case):
    """Host LAPACK table fit == the reference's table (same library calls)."""
    z = golden(case)
    name, shape, osf, kwd, ks, prec, C = parse_meta(z["meta"])
    tab, n, nd = _grappa.KernelTable(z["in_calib"], 0.5, prec, 0.01)
    assert tab.shape == tuple(z["ref_table_size"])
    # same LAPACK calls; BLAS thread count changes the last bits (FP32 bar 1e-5)
    assert rel_l2(tab[z["ref_table_used_idx"]], z["ref_table_used"]) < 1e-5


def test_table_fit_fp64_mode_is_close_to_fp32_fit():
    z = golden("plan_p2d_circle_osf2.npz")
    t32, _, _ = _grappa.KernelTable(z["in_calib"], 0.5, 1, 0.01)
    t64, _, _ = _grappa.KernelTable(z["in_calib"], 0.5, 1, 0.01, fit_dtype=torch.complex128)
    assert t64.dtype == np.complex64
    assert rel_l2(t32, t64) < 1e-4


def _toy_plan(shape, npts, kw, rng, hot=0):
    G = int(np.prod(shape))
    tgt = rng.integers(-1, G, size=(npts, kw)).astype(np.int64)
    if hot:
        tgt[:hot, 0] = G // 2
    idx = rng.integers(0, 121, size=(npts, kw)).astype(np.int64)
    w = rng.random((npts, kw)).astype(np.float32)
    return torch.from_numpy(tgt), torch.from_numpy(idx), torch.from_numpy(w)


@pytest.mark.parametrize("shape", [(40, 70), (20, 17, 33)])
def test_brick_plan_covers_every_valid_replica_once(shape):
    rng = np.random.default_rng(1)
    tgt, idx, w = _toy_plan(shape, 3000, 3, rng, hot=2500)
    bp = _grog.BrickPlan(tgt, idx, w, 3, shape, chunk=256)
    work = bp.work.numpy()
    valid = (tgt.numpy().reshape(-1) >= 0).sum()
    assert bp.n_valid == valid
    # chunks tile [0, n_valid) exactly, in order
    spans = work[:, 1:3]
    nonempty = spans[spans[:, 1] > spans[:, 0]]
    assert nonempty[0, 0] == 0 and nonempty[-1, 1] == valid
    assert np.all(nonempty[1:, 0] == nonempty[:-1, 1])
    assert np.all(spans[:, 1] - spans[:, 0] <= 256)
    # every brick appears, hot bricks are split and flagged
    nb = int(np.prod(bp.nb))
    assert set(work[:, 0].tolist()) == set(range(nb))
    assert bp.split_bricks.numel() >= 1 and np.all(work[work[:, 3] == 1, 0] >= 0)
    # metadata decodes back to the replica's cell, entry and source
    meta = bp.rep_meta.numpy().astype(np.int64) & 0xFFFFFFFF
    entry = meta & 0xFFFFF
    cl = meta >> 20
    r_sorted = np.nonzero(tgt.numpy().reshape(-1) >= 0)[0]
    gz, gy, gx = bp.grid
    bz, by, bx = bp.brick
    src = bp.rep_src.numpy()
    # rebuild (brick, cell) from metadata and compare with the true target cell
    for i in range(0, bp.n_valid, 97):
        b = int(np.searchsorted(np.cumsum(np.bincount(work[:, 0], minlength=nb) * 0) , 0))
        del b
    brick_of = np.empty(bp.n_valid, dtype=np.int64)
    for row in work:
        brick_of[row[1]:row[2]] = row[0]
    nby, nbx = bp.nb[1], bp.nb[2]
    biz = brick_of // (nby * nbx)
    biy = (brick_of // nbx) % nby
    bix = brick_of % nbx
    lz = cl // (by * bx)
    ly = (cl // bx) % by
    lx = cl % bx
    cell = ((biz * bz + lz) * gy + (biy * by + ly)) * gx + (bix * bx + lx)
    t_all = tgt.numpy().reshape(-1)
    i_all = idx.numpy().reshape(-1)
    # the multiset of (source, cell, entry) triples is preserved
    got = sorted(zip(src.tolist(), cell.tolist(), entry.tolist()))
    exp = sorted(zip((r_sorted // 3).tolist(), t_all[r_sorted].tolist(), i_all[r_sorted].tolist()))
    assert got == exp
    # sorted by (brick, cell)
    key = brick_of * bp.cells + cl
    assert np.all(np.diff(key) >= 0)
    assert bp.multi == bool(np.bincount(r_sorted // 3).max() > 1)


def test_brick_plan_split_packing_and_first_valid_mask():
    rng = np.random.default_rng(3)
    shape = (24, 16, 40)
    kw = 4
    tgt, idx, w = _toy_plan(shape, 2000, kw, rng)
    idx = torch.from_numpy(rng.integers(0, 11 * 121, size=(2000, kw)).astype(np.int64))
    bp = _grog.BrickPlan(tgt, idx, w, kw, shape, brick=(4, 8, 8), n_outer=11, pack="split")
    meta = bp.rep_meta.numpy().astype(np.int64) & 0xFFFFFFFF
    cl = meta & 2047
    inner = (meta >> 11) & 16383
    outer = meta >> 25
    r = np.nonzero(tgt.numpy().reshape(-1) >= 0)[0]
    e_all = idx.numpy().reshape(-1)
    got = sorted(zip(bp.rep_src.numpy().tolist(), (inner * 11 + outer).tolist()))
    exp = sorted(zip((r // kw).tolist(), e_all[r].tolist()))
    assert got == exp
    assert np.all(cl < bp.cells)
    # inside each work item, replicas are ordered by (outer index, cell)
    for row in bp.work.numpy():
        key = outer[row[1]:row[2]] * bp.cells + cl[row[1]:row[2]]
        assert np.all(np.diff(key) >= 0)
    first = _grog._first_valid_mask(tgt, kw).numpy().reshape(-1, kw)
    valid = tgt.numpy() >= 0
    assert np.array_equal(first.sum(1), valid.any(1).astype(int))
    for n in range(0, 2000, 37):
        if valid[n].any():
            assert first[n, np.argmax(valid[n])]


@pytest.mark.parametrize("shape,brick,n_outer,sub_cap", [
    ((40, 70), (1, 16, 32), 11, 64),
    ((20, 17, 33), (4, 8, 8), 11, 32),
    ((24, 16, 40), (8, 8, 8), 1, 256),
])
def test_brick_plan6_invariants(shape, brick, n_outer, sub_cap):
    from pygrog_b200.calib._plan6 import BrickPlan6, lane_chunk

    rng = np.random.default_rng(5)
    kw = 3
    tgt, _, w = _toy_plan(shape, 3000, kw, rng, hot=1500)
    idx = torch.from_numpy(rng.integers(0, 11 * 121, size=(3000, kw)).astype(np.int64))
    n_cta = 7
    bp = BrickPlan6(tgt, idx, w, kw, shape, brick, n_outer=n_outer, sub_cap=sub_cap, item_subs=4, n_cta=n_cta)
    t_all = tgt.numpy().reshape(-1)
    i_all = idx.numpy().reshape(-1)
    w_all = w.numpy().reshape(-1)
    r = np.nonzero(t_all >= 0)[0]
    assert bp.n_valid == r.size
    subs = bp.subs.numpy()
    meta = bp.meta.numpy().astype(np.int64)
    uniq = bp.uniq.numpy()
    cl = meta[:, 0] & 0xFFFF
    slot = meta[:, 0] >> 16
    q = meta[:, 1] & 0xFFFF
    k = meta[:, 1] >> 16
    # sub-chunks tile the replica list and the slot list in order
    assert subs[0, 0] == 0 and subs[-1, 1] == bp.n_valid and np.all(subs[1:, 0] == subs[:-1, 1])
    assert subs[0, 2] == 0 and subs[-1, 3] == uniq.size and np.all(subs[1:, 2] == subs[:-1, 3])
    assert np.all(subs[:, 1] - subs[:, 0] <= sub_cap) and np.all(subs[:, 1] > subs[:, 0])
    # per-CTA streams: every sub-chunk exactly once, items contiguous with first/last flags
    sd = bp.sd.numpy()
    si = bp.si.numpy()
    ptr = bp.cta_ptr.numpy()
    assert ptr[0] == 0 and ptr[-1] == len(subs) and len(ptr) == n_cta + 1
    seen = sorted(map(tuple, sd.tolist()))
    assert seen == sorted(map(tuple, subs.tolist()))
    brick_of_sub = {}
    for c in range(n_cta):
        ent = si[ptr[c]:ptr[c + 1]]
        if len(ent) == 0:
            continue
        assert ent[0, 1] & 1 and ent[-1, 1] & 2  # stream starts and ends on item boundaries
        for j in range(len(ent)):
            if j and not ent[j, 1] & 1:
                assert ent[j, 0] == ent[j - 1, 0] and not ent[j - 1, 1] & 2
        for row, e in zip(sd[ptr[c]:ptr[c + 1]], ent):
            brick_of_sub[tuple(row)] = int(e[0])
    work = bp.work.numpy()
    split_bricks = set(bp.split_bricks.numpy().tolist())
    for b, s0, s1, split, c in work:
        assert 1 <= s1 - s0 <= 4 and split == (b in split_bricks)
    nb = int(np.prod(bp.nb))
    occupied = set(work[:, 0].tolist())
    assert set(bp.zero_bricks.numpy().tolist()) == (set(range(nb)) - occupied) | split_bricks
    # split bricks first (cleared before the gridding kernel), the empty ones last
    zb = bp.zero_bricks.numpy().tolist()
    n_split = len(zb) - bp.n_empty_tail
    assert set(zb[:n_split]) == split_bricks and set(zb[n_split:]) == set(range(nb)) - occupied
    assert bp._c.n_empty_tail == bp.n_empty_tail and bp._c.n_zero_bricks == len(zb)
    # LPT keeps the CTAs balanced
    cost = bp.cta_cost
    assert cost.max() <= cost.mean() * 1.5 + (work[:, 2] - work[:, 1]).max() * sub_cap
    gz, gy, gx = bp.grid
    bz, by, bx = bp.brick
    nby, nbx = bp.nb[1], bp.nb[2]
    triples = []
    for s, (r0, r1, u0, u1) in enumerate(subs):
        us = uniq[u0:u1]
        assert np.all(np.diff(us) > 0)  # staged samples ascending and distinct
        assert np.all(slot[r0:r1] < u1 - u0)
        key = (k[r0:r1] * 65536 + q[r0:r1]) * bp.cells + cl[r0:r1]
        assert np.all(np.diff(key) >= 0)  # (outer, inner, cell) order
        b = brick_of_sub[(r0, r1, u0, u1)]
        biz, biy, bix = b // (nby * nbx), (b // nbx) % nby, b % nbx
        c = cl[r0:r1]
        cell = ((biz * bz + c // (by * bx)) * gy + biy * by + (c // bx) % by) * gx + bix * bx + c % bx
        for j in range(r1 - r0):
            triples.append((int(us[slot[r0 + j]]), int(cell[j]), int(q[r0 + j] * n_outer + k[r0 + j]),
                            float(bp.w[r0 + j])))
    exp = sorted(zip((r // kw).tolist(), t_all[r].tolist(), i_all[r].tolist(), w_all[r].tolist()))
    assert sorted(triples) == exp
    # lane-chunk layout: [q, j, l, t] = M[q][l * RPL + t][j]
    M = torch.randn(5, 12, 12, dtype=torch.complex64)
    lc = lane_chunk(M)
    assert lc.shape == (5, 12, 6, 2)
    assert lc[3, 7, 4, 1] == M[3, 4 * 2 + 1, 7]
    lc5 = lane_chunk(torch.randn(2, 5, 5, dtype=torch.complex64))
    assert lc5.shape == (2, 5, 5, 1)


def test_brick_plan6_lane_order_residue_columns():
    from pygrog_b200.calib._plan6 import BrickPlan6

    rng = np.random.default_rng(9)
    shape, kw = (24, 16, 40), 3
    tgt, _, w = _toy_plan(shape, 6000, kw, rng, hot=3000)
    idx = torch.from_numpy(rng.integers(0, 11 * 121, size=(6000, kw)).astype(np.int64))
    a = BrickPlan6(tgt, idx, w, kw, shape, (4, 8, 8), n_outer=11, sub_cap=256, n_cta=3)
    b = BrickPlan6(tgt, idx, w, kw, shape, (4, 8, 8), n_outer=11, sub_cap=256, n_cta=3, lane_order=True)
    assert b.n_valid == a.n_valid and b.n_pad > 0
    assert torch.equal(a.uniq, b.uniq) and torch.equal(a.subs[:, 2:], b.subs[:, 2:])

    def qw_cost(m):
        """Quarter-warps with an active lane, each costing the largest number of
        distinct operators (inner or outer) that share one bank quad residue."""
        cost = 0
        for g0 in range(0, len(m), 8):
            g = m[g0:g0 + 8]
            g = g[g[:, 0] >= 0]
            if len(g):
                for ops in (np.unique(g[:, 1] & 0xFFFF), np.unique(g[:, 1] >> 16)):
                    cost += np.bincount(ops % 8, minlength=8).max()
        return cost

    ca = cb = 0
    wa, wb = a.w.numpy(), b.w.numpy()
    for (r0, r1, u0a, _), (t0, t1, u0b, _) in zip(a.subs.numpy(), b.subs.numpy()):
        ma = a.meta.numpy()[r0:r1].astype(np.int64)
        mb = b.meta.numpy()[t0:t1].astype(np.int64)
        real = mb[:, 0] >= 0
        # whole quarter-warps, fewer than eight padding entries, the same replicas
        assert (t1 - t0) % 8 == 0 and t1 - t0 <= 256 and (t1 - t0) - (r1 - r0) < 8
        # the same replicas: (cell, inner | outer << 16, sample, weight)
        ua_, ub_ = a.uniq.numpy(), b.uniq.numpy()
        sa = ua_[u0a + (ma[:, 0] >> 16)]
        sbm = ub_[u0b + (mb[real, 0] >> 16)]
        ra = sorted(zip((ma[:, 0] & 0xFFFF).tolist(), ma[:, 1].tolist(), sa.tolist(), wa[r0:r1].tolist()))
        rb = sorted(zip((mb[real, 0] & 0xFFFF).tolist(), mb[real, 1].tolist(), sbm.tolist(),
                        wb[t0:t1][real].tolist()))
        assert ra == rb
        assert np.all(wb[t0:t1][~real] == 0)
        ca += qw_cost(ma)
        cb += qw_cost(mb)
    assert cb < 0.85 * ca


def test_brick_plan6_pair_lane_packing():
    from pygrog_b200.calib._plan6 import BrickPlan6

    rng = np.random.default_rng(19)
    shape, kw = (24, 16, 40), 3
    tgt, _, w = _toy_plan(shape, 6000, kw, rng, hot=3000)
    idx = torch.from_numpy(rng.integers(0, 11 * 121, size=(6000, kw)).astype(np.int64))
    a = BrickPlan6(tgt, idx, w, kw, shape, (4, 8, 8), n_outer=11, sub_cap=256, n_cta=3)
    b = BrickPlan6(tgt, idx, w, kw, shape, (4, 8, 8), n_outer=11, sub_cap=256, n_cta=3, lane_order=True,
                   pair_lanes=True, cell_order=True)

    def cost(m):
        """Quarter-warps of four replicas (two lanes each, half-row offset = 4
        bank quads): largest number of distinct operators per class mod 4."""
        tot = 0
        for g0 in range(0, len(m), 4):
            g = m[g0:g0 + 4]
            g = g[g[:, 0] >= 0]
            if len(g):
                for ops in (np.unique(g[:, 1] & 0xFFFF), np.unique(g[:, 1] >> 16)):
                    tot += np.bincount(ops % 4, minlength=4).max()
        return tot

    ca = cb = 0
    for (r0, r1, _, _), (t0, t1, _, _) in zip(a.subs.numpy(), b.subs.numpy()):
        ma = a.meta.numpy()[r0:r1].astype(np.int64)
        mb = b.meta.numpy()[t0:t1].astype(np.int64)
        real = mb[:, 0] >= 0
        assert (t1 - t0) % 4 == 0 and t1 - t0 <= 256 and (t1 - t0) - (r1 - r0) < 4
        assert sorted(zip((ma[:, 0] & 0xFFFF).tolist(), ma[:, 1].tolist())) == \
            sorted(zip((mb[real, 0] & 0xFFFF).tolist(), mb[real, 1].tolist()))
        ca += cost(ma)
        cb += cost(mb)
    assert cb < 0.85 * ca


def test_brick_plan6_cell_order_words():
    from pygrog_b200.calib._plan6 import BrickPlan6

    rng = np.random.default_rng(12)
    shape, kw = (24, 16, 40), 3
    tgt, _, w = _toy_plan(shape, 5000, kw, rng, hot=2500)
    idx = torch.from_numpy(rng.integers(0, 11 * 121, size=(5000, kw)).astype(np.int64))
    seg = 4
    bp = BrickPlan6(tgt, idx, w, kw, shape, (4, 8, 8), n_outer=11, sub_cap=256, n_cta=3, lane_order=True,
                    cell_order=True, seg_len=seg)
    cw = bp.cword.numpy().astype(np.int64)
    meta = bp.meta.numpy().astype(np.int64)
    n_shared = 0
    for r0, r1, _, _ in bp.subs.numpy():
        e = cw[r0:r1]
        pos, cell, head, shared = e & 511, (e >> 9) & 4095, (e >> 21) & 1, (e >> 22) & 1
        assert sorted(pos.tolist()) == list(range(r1 - r0))  # every entry once
        real = meta[r0 + pos, 0] >= 0
        assert np.array_equal(cell[real], meta[r0 + pos[real], 0] & 0xFFFF)  # the replica's cell
        assert np.all(cell[~real] == bp.cells) and np.all(head[~real] == 1) and np.all(shared[~real] == 0)
        key = cell * 512 + pos
        assert np.all(np.diff(key) > 0)  # sorted by (cell, pos)
        # segments: every cell's run cut into ceil(L / seg) parts of near-equal size
        new_cell = np.concatenate([[1], (np.diff(cell) != 0).astype(int)])
        starts = np.flatnonzero(new_cell)
        run_len = np.diff(np.append(starts, len(cell)))
        for s0, L in zip(starts, run_len):
            if cell[s0] == bp.cells:
                continue
            h = np.flatnonzero(head[s0:s0 + L])
            sizes = np.diff(np.append(h, L))
            assert h[0] == 0 and sizes.max() <= seg and sizes.max() - sizes.min() <= 1
            assert len(h) == -(-L // seg)
            assert np.all(shared[s0:s0 + L] == (L > seg))
        n_shared += int(shared.sum())
    assert n_shared > 0  # the hot cells give runs longer than a segment


def test_cell_row_plan_runs_and_straddle_bits():
    """Tensor-core forward plan: (cell, sample) order inside each sub-chunk and
    bit 30 of meta.x set exactly on runs that cross a 16-row m-tile."""
    import torch

    from pygrog_b200.calib._plan6 import BrickPlan6

    rng = np.random.default_rng(3)
    n_src, kw, gs = 3000, 1, (16, 32, 32)
    tgt = torch.as_tensor(rng.integers(0, 16 * 32 * 32 // 64, (n_src, kw)) * 7 % (16 * 32 * 32))
    tgt[::5] = 100  # a hot cell
    idx = torch.as_tensor(rng.integers(0, 11 ** 3, (n_src, kw)))
    w = torch.rand(n_src, kw)
    p = BrickPlan6(tgt, idx, w, kw, gs, brick=(4, 8, 8), n_outer=11, sub_cap=256, n_cta=4, sample_order=True,
                   cell_rows=True)
    meta = p.meta.numpy()
    cell = meta[:, 0] & 0xFFFF
    strad = (meta[:, 0] >> 30) & 1
    assert (meta[:, 0] >= 0).all()
    for b, e, _, _ in p.subs.numpy():
        c = cell[b:e]
        assert (np.diff(c) >= 0).all()
        for v in np.unique(c):
            pos = np.nonzero(c == v)[0]
            crosses = pos[0] // 16 != pos[-1] // 16
            assert (strad[b:e][pos] == crosses).all()
    # same replicas (cell, weight) as a sample-ordered plan
    q = BrickPlan6(tgt, idx, w, kw, gs, brick=(4, 8, 8), n_outer=11, sub_cap=256, n_cta=4, sample_order=True)
    assert p.n_valid == q.n_valid == n_src
    assert sorted(zip(cell.tolist(), p.w.numpy().round(6).tolist())) == \
        sorted(zip((q.meta.numpy()[:, 0] & 0xFFFF).tolist(), q.w.numpy().round(6).tolist()))


def test_cell_row_plan_packs_runs_into_m_tiles():
    """With pack_rows, runs of at most 16 entries never cross a 16-entry
    m-tile; padding entries (meta -1, weight 0) fill the gaps and every
    replica appears once."""
    import torch

    from pygrog_b200.calib._plan6 import BrickPlan6

    rng = np.random.default_rng(4)
    n_src, kw, gs = 6000, 1, (16, 32, 32)
    tgt = torch.as_tensor(rng.integers(0, 2500, (n_src, kw)))  # runs of 1-6 replicas per cell and sub-chunk
    tgt[::97] = 123  # and one long run
    idx = torch.as_tensor(rng.integers(0, 11 ** 3, (n_src, kw)))
    w = torch.rand(n_src, kw) + 0.1
    p = BrickPlan6(tgt, idx, w, kw, gs, brick=(4, 8, 8), n_outer=11, sub_cap=256, n_cta=4, sample_order=True,
                   cell_rows=True, full_subs=True, pack_rows=16)
    meta = p.meta.numpy()
    valid = meta[:, 0] >= 0
    assert valid.sum() == n_src and p.n_pad == (~valid).sum()
    assert (p.w.numpy()[~valid] == 0).all()
    crossing = 0
    for b, e, _, _ in p.subs.numpy():
        assert e - b <= 256
        m = meta[b:e]
        c = np.where(m[:, 0] >= 0, m[:, 0] & 0xFFFF, -1)
        strad = (m[:, 0] >> 30) & 1
        for v in np.unique(c[c >= 0]):
            pos = np.nonzero(c == v)[0]
            assert (np.diff(pos) == 1).all()  # one contiguous run
            crosses = pos[0] // 16 != pos[-1] // 16
            assert (strad[pos] == crosses).all()
            if crosses and pos.size <= 16:
                crossing += 1
    # only runs that met an exhausted padding budget may still cross: far fewer
    # than without packing
    q0 = BrickPlan6(tgt, idx, w, kw, gs, brick=(4, 8, 8), n_outer=11, sub_cap=256, n_cta=4, sample_order=True,
                    cell_rows=True, full_subs=True)
    before = int(((q0.meta.numpy()[:, 0] >> 30) & 1).sum())
    after = int(((meta[valid, 0] >> 30) & 1).sum())
    assert crossing <= 0.25 * p.n_subs and after < 0.5 * before
    q = BrickPlan6(tgt, idx, w, kw, gs, brick=(4, 8, 8), n_outer=11, sub_cap=256, n_cta=4, sample_order=True,
                   cell_rows=True, full_subs=True)
    qm = q.meta.numpy()
    assert sorted(zip((meta[valid, 0] & 0xFFFF).tolist(), p.w.numpy()[valid].round(6).tolist())) == \
        sorted(zip((qm[:, 0] & 0xFFFF).tolist(), q.w.numpy().round(6).tolist()))


def test_tensor_core_timeout_count_raises(monkeypatch):
    """A non-zero tile-wait timeout count becomes a RuntimeError at the check
    points (counter read mocked: no device here); a zero count passes and a
    pending check is consumed once."""
    from pygrog_b200 import _lib

    counts = [2]
    monkeypatch.setattr(_lib, "tc_timeouts", lambda reset=True: counts.pop(0) if counts else 0)
    with pytest.raises(RuntimeError, match="2 tensor-core tile wait"):
        _lib.check_tc_timeouts("degrid")
    _lib.check_tc_timeouts("degrid")  # counter now 0: no error

    g = _grog.GrogInterpolator.__new__(_grog.GrogInterpolator)
    g.device = torch.device("cpu")
    monkeypatch.setattr(torch.cuda, "is_current_stream_capturing", lambda: False)
    monkeypatch.setattr(torch.cuda, "synchronize", lambda device=None: None)
    g.check_errors()  # nothing launched: no read at all
    counts[:] = [1]
    g._tc_pending = True
    with pytest.raises(RuntimeError, match="GrogInterpolator.degrid: 1 tensor-core tile wait"):
        g.check_errors()
    assert g._tc_pending is False
    counts[:] = [5]
    g.check_errors()  # no launch since the last check: the counter is not read
    assert counts == [5]


def test_device_power_path_matches_host_powers_on_near_singular_operators():
    """The device fit's fractional powers (host eigendecomposition logarithm,
    batched matrix exponentials on the tensor's device) equal the host
    path's on the nearly singular unit operators of a 16-coil calibration
    with lamda = 1e-3 (eigenvalue moduli down to ~1e-5), where an iterative
    square-root logarithm loses accuracy."""
    from pygrog_b200.workloads import config2

    w = config2()
    ops = _grappa.train_grappa(torch.as_tensor(w.acr).to(torch.complex128), w.lamda)
    d = _grappa.shift_steps(0.5, 1)[2]
    for G in (ops.x, ops.y):
        P = _grappa.grappa_power_device(G, d)
        assert rel_l2(P.numpy(), _grappa.grappa_power(G, d).numpy()) < 1e-12
        assert rel_l2(P[d.numel() - 1].numpy() @ P[d.numel() - 1].numpy(), G.numpy()) < 1e-10  # G^0.5 G^0.5


def test_chain_operands_realify_the_complex_matrices():
    """The shift chain's realified matrices ([stage][output][input], rows 2c / 2c + 1
    the real / imaginary part of coil c) apply the complex operators, and the
    packed shift index holds (i, j, k) in bytes 0 / 1 / 2."""
    from pygrog_b200.calib import _chain

    rng = np.random.default_rng(8)
    C = 12
    W = rng.standard_normal((4, C, C)) + 1j * rng.standard_normal((4, C, C))
    ph = np.exp(1j * rng.uniform(-np.pi, np.pi, (3, _chain.STEPS, C)))
    Wr, phr = _chain.chain_operands(W, ph, "cpu")
    assert tuple(Wr.shape) == (4, 2 * C, 2 * C) and Wr.dtype == torch.float32
    assert tuple(phr.shape) == (3, _chain.STEPS, C, 2)
    x = rng.standard_normal(C) + 1j * rng.standard_normal(C)
    xr = np.empty(2 * C)
    xr[0::2], xr[1::2] = x.real, x.imag
    for s in range(4):
        y = Wr[s].double().numpy() @ xr
        np.testing.assert_allclose(y[0::2] + 1j * y[1::2], W[s] @ x, rtol=1e-5, atol=1e-5)
    ijk = torch.tensor([[3, 0, 10], [7, 10, 1], [10, 5, 0]])
    packed = _chain.pack_shift_indices(ijk)
    assert packed.dtype == torch.int32
    for r in range(3):
        p = int(packed[r])
        assert (p & 0xFF, (p >> 8) & 0xFF, (p >> 16) & 0xFF) == tuple(int(v) for v in ijk[:, r])
