"""Replica plan of the operator-stationary gridding kernels (``csrc/grog_v6.cu``).

The reference applies ``T[e]`` to every replica of every sample
(``calib/_grog.py:1283-1295``) and then scatters the replicas into the grid
(``operator/_sparse_fft.py:416``).  The fused kernels need the valid
replicas grouped by grid brick and, inside a brick, cut into sub-chunks of
at most ``sub_cap`` replicas along the sample index; inside a sub-chunk the
replicas are ordered by (outer table index, inner table index, cell) so a
slot of lanes can keep the outer factor's rows in registers along a run.
Everything here is integer bookkeeping done once per trajectory on the GPU
with torch sorts; the kernels only read the result.
"""

from __future__ import annotations

import numpy as np
import torch

from .. import _lib


def lane_chunk(table: torch.Tensor) -> torch.Tensor:
    """``(K, C, C)`` row-major operators -> lane-chunk layout ``(K, C, L, RPL)``.

    Entry ``[q, j, l, t] = M[q][l * RPL + t][j]`` with ``RPL = 2`` for even
    ``C`` (else 1) and ``L = C // RPL``: lane ``l`` of a slot reads the RPL
    entries of column ``j`` it needs as one contiguous word.
    """
    K, C, _ = table.shape
    rpl = 2 if C % 2 == 0 else 1
    L = C // rpl
    return table.reshape(K, L, rpl, C).permute(0, 3, 1, 2).contiguous()


class BrickPlan6:
    """Valid replicas in sub-chunk order with per-replica ``(cell, slot, inner, outer)``.

    Arrays (all on the plan's device unless noted):
      ``subs``   int32 (n_subs, 4) ``{rep_begin, rep_end, uniq_begin, uniq_end}``
      ``uniq``   int32 source sample of every staging slot (ascending inside a
                 sub-chunk: neighbouring threads stage neighbouring samples)
      ``meta``   int32 (n_valid, 2) ``{cell | slot << 16, inner | outer << 16}``
      ``w``      float32 replica weight
      ``sd`` / ``si`` / ``cta_ptr``  per-CTA sub-chunk streams: descriptor,
                 ``{brick, flags}`` (1 first of item, 2 last, 4 split brick)
      ``work``   (host) int32 (n_items, 5) ``{brick, sub_begin, sub_end, split, cta}``
      ``cword``  int32, with ``cell_order``: each sub-chunk's replicas in cell
                 order, ``pos | cell << 9 | head << 21 | shared << 22``; a
                 head starts a segment of at most ``seg_len`` replicas of one
                 cell, ``shared`` marks segments of a cell with several
      ``n_pad``  padding entries (``lane_order`` only: meta ``-1``, weight 0,
                 cell order cell = ``cells``) that round every sub-chunk to
                 whole quarter-warps
      ``zero_bricks`` bricks the forward zeroes (split ones, then the
      ``n_empty_tail`` empty ones)
      ``zero_src`` samples with no replica in this plan; ``multi`` whether a
      sample has more than one.
    """

    def __init__(
        self,
        target_idx: torch.Tensor,
        interp_idx: torch.Tensor,
        rep_weight: torch.Tensor,
        kw: int,
        grid_shape,
        brick,
        n_outer: int = 1,
        mask: torch.Tensor | None = None,
        sub_cap: int = 256,
        item_subs: int = 8,
        n_cta: int | None = None,
        lane_order: bool = False,
        cell_order: bool = False,
        seg_len: int = 8,
        pair_lanes: bool = False,
        sample_order: bool = False,
        cell_rows: bool = False,
        full_subs: bool = False,
        pack_rows: int = 0,
    ):
        dev = target_idx.device
        grid_shape = tuple(int(s) for s in grid_shape)
        if len(grid_shape) == 2:
            gz, gy, gx = 1, grid_shape[0], grid_shape[1]
        else:
            gz, gy, gx = grid_shape
        bz, by, bx = (int(b) for b in brick)
        for b in (bz, by, bx):
            if b < 1 or (b & (b - 1)):
                raise ValueError("brick extents must be powers of two")
        self.grid = (gz, gy, gx)
        self.brick = (bz, by, bx)
        self.nb = ((gz + bz - 1) // bz, (gy + by - 1) // by, (gx + bx - 1) // bx)
        self.cells = cells = bz * by * bx
        if cells > 4096:
            raise ValueError("brick too large (max 4096 cells)")
        if not 1 <= sub_cap <= 512:
            raise ValueError("sub_cap must be in 1..512")
        self.sub_cap = int(sub_cap)
        self.n_outer = int(n_outer)
        n_bricks = self.nb[0] * self.nb[1] * self.nb[2]

        tgt = target_idx.reshape(-1)
        self.n_src = n_src = tgt.numel() // kw
        valid = tgt >= 0
        if mask is not None:
            valid = valid & mask.reshape(-1)
        r = torch.nonzero(valid).squeeze(1)
        t = tgt[r]
        z = t // (gy * gx)
        rem = t - z * (gy * gx)
        y = rem // gx
        x = rem - y * gx
        brick_id = ((z // bz) * self.nb[1] + (y // by)) * self.nb[2] + (x // bx)
        cl = ((z % bz) * by + (y % by)) * bx + (x % bx)
        src = r // kw
        e = interp_idx.reshape(-1)[r].to(torch.int64)
        q = e // self.n_outer
        k = e - q * self.n_outer
        w = rep_weight.reshape(-1)[r].to(torch.float32)
        if e.numel() and (int(q.max()) >= 65536 or self.n_outer > 65536):
            raise ValueError("table factors too large for 16-bit indices")

        # (1) sub-chunks: replicas of a brick in sample order, sub_cap at a time
        _, p1 = torch.sort(brick_id * n_src + src, stable=True)
        brick_id, cl, src, q, k, w = (a[p1] for a in (brick_id, cl, src, q, k, w))
        n = int(brick_id.numel())
        cnt = torch.bincount(brick_id, minlength=n_bricks)
        start = torch.cumsum(cnt, 0) - cnt
        pos = torch.arange(n, device=dev) - start[brick_id]
        # with pack_rows, sub-chunks take sub_cap - pack_rows replicas and keep
        # pack_rows entries for the padding that aligns cell runs to m-tiles
        form_cap = self.sub_cap - pack_rows if (cell_rows and pack_rows) else self.sub_cap
        if form_cap < 1:
            raise ValueError("sub_cap must exceed pack_rows")
        nsub_b = (cnt + form_cap - 1) // form_cap
        sub_first = torch.cumsum(nsub_b, 0) - nsub_b
        if full_subs:
            # full sub-chunks first (every warp of the tensor-core kernels gets
            # the same number of m-tiles), the remainder last
            sub_id = sub_first[brick_id] + pos // form_cap
        else:
            # near-equal sub-chunks inside a brick keep consecutive sub-chunks balanced
            sub_id = sub_first[brick_id] + (pos * nsub_b[brick_id]) // torch.clamp(cnt[brick_id], min=1)
        n_subs = int(nsub_b.sum())
        # staging slots: distinct samples of a sub-chunk, ascending
        uk, inv = torch.unique_consecutive(sub_id * n_src + src, return_inverse=True)
        uniq_sub = uk // n_src
        ucnt = torch.bincount(uniq_sub, minlength=n_subs)
        ubeg = torch.cumsum(ucnt, 0) - ucnt
        slot = inv - ubeg[sub_id]

        # (2) order inside a sub-chunk: (outer, inner, cell).  With lane_order
        # (one replica per lane, or per lane pair with pair_lanes) the sub-chunk
        # is laid out in whole quarter-warps whose lanes read inner operators in
        # different bank quads or the same operator, and likewise outer ones
        # (_pack_quarter_warps); the places left free are padding entries
        # (meta -1, weight 0), fewer than one quarter-warp per sub-chunk.
        n_in = int(q.max()) + 1 if n else 1
        pad = torch.zeros(0, dtype=torch.bool, device=dev)
        if lane_order and n:
            # processing order inside a sub-chunk: replicas of one inner operator
            # together, largest such group first, then (inner, outer, cell)
            _, pa = torch.sort((q * self.n_outer + k) * cells + cl, stable=True)
            sub_a, q_a = sub_id[pa], q[pa]
            key_q = sub_a * n_in + q_a
            gsz = torch.bincount(key_q)[key_q]
            _, pb = torch.sort(sub_a * (self.sub_cap + 1) + (self.sub_cap - gsz), stable=True)
            p2 = pa[pb]
            sub_id, cl, slot, q, k, w, src = (a[p2] for a in (sub_id, cl, slot, q, k, w, src))
            per = 4 if pair_lanes else 8  # replicas per quarter-warp
            lane, nq = _pack_quarter_warps(sub_id, q, k, n_subs, per)
            nslot = nq * per
            sbase = torch.cumsum(nslot, 0) - nslot
            total = int(nslot.sum())
            dest = sbase[sub_id] + lane
            pad = torch.ones(total, dtype=torch.bool, device=dev)
            pad[dest] = False

            def spread(v, fill):
                out = torch.full((total,), fill, dtype=v.dtype, device=dev)
                out[dest] = v
                return out

            sub_full = torch.searchsorted(sbase, torch.arange(total, device=dev), right=True) - 1
            meta0 = spread(cl | (slot << 16), -1)
            meta1 = spread(q | (k << 16), 0)
            self.meta = torch.stack([meta0, meta1], dim=1).to(torch.int32).contiguous()
            self.w = spread(w, 0.0).contiguous()
            src = spread(src, -1)
            cl = spread(cl, cells)  # padding: no cell
            sub_id = sub_full
        elif cell_rows and n:
            # tensor-core forward: each sub-chunk in (cell, sample) order, so an
            # m-tile's 16 rows hold runs of one cell that the kernel sums in
            # registers; bit 30 of meta.x marks replicas of a cell whose run
            # crosses an m-tile boundary (those segments are added atomically)
            _, p2 = torch.sort((sub_id * cells + cl) * n_src + src, stable=True)
            sub_id, cl, slot, q, k, w, src = (a[p2] for a in (sub_id, cl, slot, q, k, w, src))
            rc = torch.bincount(sub_id, minlength=n_subs)
            rb = torch.cumsum(rc, 0) - rc
            pos = torch.arange(n, device=dev) - rb[sub_id]
            head = torch.ones(n, dtype=torch.bool, device=dev)
            head[1:] = (cl[1:] != cl[:-1]) | (sub_id[1:] != sub_id[:-1])
            run_id = torch.cumsum(head.to(torch.int64), 0) - 1
            run_len = torch.bincount(run_id)
            run_pos = pos[head]
            rs = run_pos[run_id]
            re = rs + run_len[run_id] - 1
            if pack_rows:
                # next-fit of the runs into m-tiles of pack_rows rows: a run that
                # would cross a boundary starts the next m-tile (padding entries,
                # meta -1, in between) while the sub-chunk's padding budget
                # allows; only runs longer than an m-tile still cross one
                rsub = sub_id[head]
                run_ptr = torch.cumsum(torch.bincount(rsub, minlength=n_subs), 0)
                run_ptr = torch.cat([torch.zeros(1, dtype=torch.int64, device=dev), run_ptr])
                run_start, nslot = _native_pack_rows(run_len, run_ptr, n_subs, pack_rows, self.sub_cap)
                new_pos = run_start[run_id] + (pos - rs)  # nslot: entries per sub-chunk, padding included
                sbase = torch.cumsum(nslot, 0) - nslot
                total = int(nslot.sum())
                dest = sbase[sub_id] + new_pos
                pad = torch.ones(total, dtype=torch.bool, device=dev)
                pad[dest] = False
                rs = run_start[run_id]
                re = rs + run_len[run_id] - 1
                straddle = (rs // pack_rows) != (re // pack_rows)

                def spread(v, fill):
                    out = torch.full((total,), fill, dtype=v.dtype, device=dev)
                    out[dest] = v
                    return out

                meta0 = spread(cl | (slot << 16) | (straddle.to(torch.int64) << 30), -1)
                meta1 = spread(q | (k << 16), 0)
                self.meta = torch.stack([meta0, meta1], dim=1).to(torch.int32).contiguous()
                self.w = spread(w, 0.0).contiguous()
                src = spread(src, -1)
                cl = spread(cl, cells)
                sub_id = torch.searchsorted(sbase, torch.arange(total, device=dev), right=True) - 1
            else:
                straddle = (rs // 16) != (re // 16)
                self.meta = torch.stack([cl | (slot << 16) | (straddle.to(torch.int64) << 30), q | (k << 16)],
                                        dim=1).to(torch.int32).contiguous()
                self.w = w.contiguous()
        elif sample_order:
            # keep step (1)'s sample order: the tensor-core gridder reads each
            # m-tile's staged samples in order (conflict-free) and spreads
            # the cells of a tile
            self.meta = torch.stack([cl | (slot << 16), q | (k << 16)], dim=1).to(torch.int32).contiguous()
            self.w = w.contiguous()
        else:
            key2 = ((sub_id * self.n_outer + k) * n_in + q) * cells + cl
            _, p2 = torch.sort(key2, stable=True)
            sub_id, cl, slot, q, k, w, src = (a[p2] for a in (sub_id, cl, slot, q, k, w, src))
            self.meta = torch.stack([cl | (slot << 16), q | (k << 16)], dim=1).to(torch.int32).contiguous()
            self.w = w.contiguous()
        self.uniq = (uk - uniq_sub * n_src).to(torch.int32).contiguous()
        rcnt = torch.bincount(sub_id, minlength=n_subs)
        rbeg = torch.cumsum(rcnt, 0) - rcnt
        self.subs = torch.stack([rbeg, rbeg + rcnt, ubeg, ubeg + ucnt], dim=1).to(torch.int32).contiguous()
        self.n_pad = int(pad.sum())
        self.n_valid = n
        self.n_subs = n_subs
        self.rep_src = src.to(torch.int32)  # replica -> sample in kernel order, -1 for padding
        # cell order of each sub-chunk (lane-per-replica forward): entries
        # sorted by (cell, pos), pos = the replica's index inside the sub-chunk;
        # a cell's run is cut into near-equal segments of at most seg_len entries, each
        # summed by one thread (bounded serial work in dense k-space), and
        # segments of a cell with several are added to the tile atomically
        self.cword = torch.zeros(0, dtype=torch.int32, device=dev)
        if cell_order and n:
            if self.sub_cap > 512 or cells > 4095:
                raise ValueError("cell order needs sub_cap <= 512 and cells <= 4095")
            if seg_len < 1:
                raise ValueError("seg_len must be >= 1")
            n_ent = sub_id.numel()  # replicas + padding
            pos_in = torch.arange(n_ent, device=dev) - rbeg[sub_id]
            _, pc = torch.sort(sub_id * ((cells + 1) * 512) + cl * 512 + pos_in, stable=True)
            c_s, s_s = cl[pc], sub_id[pc]
            first_c = torch.ones(n_ent, dtype=torch.bool, device=dev)
            first_c[1:] = (c_s[1:] != c_s[:-1]) | (s_s[1:] != s_s[:-1])
            run_id = torch.cumsum(first_c.to(torch.int64), 0) - 1
            run_len = torch.bincount(run_id)
            run_beg = torch.cumsum(run_len, 0) - run_len
            in_run = torch.arange(n_ent, device=dev) - run_beg[run_id]
            # a run of L entries -> ceil(L / seg_len) near-equal segments
            L = run_len[run_id]
            parts = (L + seg_len - 1) // seg_len
            part = in_run * parts // L
            head = (in_run == 0) | (part != (in_run - 1).clamp(min=0) * parts // L)
            shared = parts > 1
            is_pad = c_s >= cells  # padding entries: one-entry segments, no tile update
            head = head | is_pad
            shared = shared & ~is_pad
            self.cword = (pos_in[pc] | (c_s << 9) | (head.to(torch.int64) << 21)
                          | (shared.to(torch.int64) << 22)).to(torch.int32).contiguous()

        # (3) brick items of at most item_subs sub-chunks, assigned largest
        # first to the least loaded CTA; each CTA gets a flat sub-chunk stream
        nit_b = (nsub_b + item_subs - 1) // item_subs
        brick_rep = torch.repeat_interleave(torch.arange(n_bricks, device=dev), nit_b)
        first = torch.cumsum(nit_b, 0) - nit_b
        kk = torch.arange(brick_rep.numel(), device=dev) - first[brick_rep]
        s0 = sub_first[brick_rep] + kk * item_subs
        s1 = torch.minimum(s0 + item_subs, sub_first[brick_rep] + nsub_b[brick_rep])
        split = (nit_b[brick_rep] > 1).to(torch.int64)
        rcum = torch.cat([torch.zeros(1, dtype=torch.int64, device=dev), torch.cumsum(rcnt, 0)])
        reps = (rcum[s1] - rcum[s0]).cpu().numpy()
        n_cta = int(n_cta) if n_cta is not None else _sm_count(dev)
        cta = _lpt_assign(reps + cells // 4, n_cta)
        order = np.lexsort((-reps, cta))  # per CTA, largest item first
        items = torch.stack([brick_rep, s0, s1, split], dim=1).cpu().numpy()[order]
        cta = cta[order]
        self.work = torch.from_numpy(np.concatenate([items, cta[:, None]], 1).astype(np.int32))
        nsub_i = items[:, 2] - items[:, 1]
        ent_item = np.repeat(np.arange(len(items)), nsub_i)
        ent_first = np.cumsum(nsub_i) - nsub_i
        sub_idx = items[ent_item, 1] + (np.arange(ent_item.size) - ent_first[ent_item])
        flags = ((sub_idx == items[ent_item, 1]) * 1 + (sub_idx == items[ent_item, 2] - 1) * 2
                 + items[ent_item, 3] * 4)
        sub_idx_t = torch.from_numpy(sub_idx.astype(np.int64)).to(dev)
        self.sd = self.subs[sub_idx_t].contiguous()
        self.si = torch.from_numpy(np.stack([items[ent_item, 0], flags], 1).astype(np.int32)).to(dev).contiguous()
        per_cta = np.bincount(cta[ent_item], minlength=n_cta) if ent_item.size else np.zeros(n_cta, np.int64)
        self.cta_ptr = torch.from_numpy(np.concatenate([[0], np.cumsum(per_cta)]).astype(np.int32)).to(dev)
        self.n_cta = n_cta
        self.cta_cost = (np.bincount(cta, weights=(reps + cells // 4)[order], minlength=n_cta) if len(cta)
                         else np.zeros(n_cta))
        split_b = nit_b > 1
        self.split_bricks = torch.nonzero(split_b).squeeze(1).to(torch.int32).contiguous()
        # split bricks first (cleared before the gridding kernel: they take
        # reduce-adds), then the empty ones (cleared by the tensor-core
        # forward's CTAs while they grid, or beforehand by the other kernels)
        empty_b = cnt == 0
        self.zero_bricks = torch.cat([torch.nonzero(split_b & ~empty_b), torch.nonzero(empty_b)]).squeeze(1)
        self.zero_bricks = self.zero_bricks.to(torch.int32).contiguous()
        self.n_empty_tail = int(empty_b.sum())
        per_src = torch.bincount(src[src >= 0], minlength=n_src)
        self.multi = bool(int(per_src.max()) > 1) if per_src.numel() else False
        self.zero_src = torch.nonzero(per_src == 0).squeeze(1).to(torch.int32).contiguous()
        self._c = self._struct()

    def _struct(self) -> _lib.V6PlanC:
        gz, gy, gx = self.grid
        bz, by, bx = self.brick
        nbz, nby, nbx = self.nb

        def ptr(t):
            return t.data_ptr() if t.numel() else None

        return _lib.V6PlanC(
            ptr(self.sd), ptr(self.si), self.cta_ptr.data_ptr(), self.n_cta if self.sd.numel() else 0,
            ptr(self.uniq), ptr(self.meta), ptr(self.w), self.sub_cap, gz, gy, gx, bz, by, bx, nbz, nby, nbx,
            ptr(self.zero_bricks), int(self.zero_bricks.numel()), ptr(self.cword), self.n_empty_tail,
        )


def _pack_quarter_warps(sub_id: torch.Tensor, q: torch.Tensor, k: torch.Tensor, n_subs: int, per: int = 8):
    """Position of every replica inside its sub-chunk, packing ``ceil(n / per)``
    quarter-warps of ``per`` replicas first-fit so that the inner operators ``q``
    of a quarter-warp are equal or in different bank-quad classes, and so are the
    outer ones ``k``.  ``per = 8``: one lane per replica, operator q starts in
    quad q mod 8.  ``per = 4``: two lanes per replica reading rows 0..C/2-1 and
    C/2..C-1 (4 quads apart when C = 12, mod 8), classes q mod 4.

    Replicas come grouped by sub-chunk, each group in its processing order.  A
    replica goes to the first quarter-warp with a free lane that (1) already
    reads its inner operator, else (2) has its inner residue free, both with a
    compatible outer residue, else (3) has a compatible inner residue, else (4)
    has the fewest lanes taken (native ``pgb_plan_pack_quarter_warps``, one
    sequential pass per sub-chunk).  Returns ``(lane, quarter-warps per
    sub-chunk)`` on the inputs' device.
    """
    dev = sub_id.device
    cnt = torch.bincount(sub_id, minlength=n_subs)
    ptr = np.concatenate([[0], np.cumsum(_host_i64(cnt))]).astype(np.int64)
    qh, kh = _host_i64(q), _host_i64(k)
    lane = np.zeros(qh.size, dtype=np.int64)
    nq = np.zeros(n_subs, dtype=np.int64)
    if n_subs:
        _lib.call("pgb_plan_pack_quarter_warps", ptr.ctypes.data, qh.ctypes.data, kh.ctypes.data, int(n_subs),
                  int(per), lane.ctypes.data, nq.ctypes.data)
    return torch.from_numpy(lane).to(dev), torch.from_numpy(nq).to(dev)


def _sm_count(dev) -> int:
    if dev.type == "cuda":
        return int(torch.cuda.get_device_properties(dev).multi_processor_count)
    return 148


def _lpt_assign(cost: np.ndarray, n_bins: int) -> np.ndarray:
    """Longest-processing-time-first assignment of items to ``n_bins`` bins
    (largest item first, to the least loaded bin, ties to the lowest bin;
    native ``pgb_plan_lpt``)."""
    c = np.ascontiguousarray(cost, dtype=np.float64)
    out = np.zeros(len(c), dtype=np.int32)
    if len(c):
        _lib.call("pgb_plan_lpt", c.ctypes.data, len(c), int(n_bins), out.ctypes.data)
    return out.astype(np.int64)


def _host_i64(t: torch.Tensor) -> np.ndarray:
    return np.ascontiguousarray(t.detach().to("cpu", torch.int64).numpy())


def _native_pack_rows(run_len: torch.Tensor, run_ptr: torch.Tensor, n_subs: int, rows: int, cap: int):
    """Next-fit packing of each sub-chunk's cell runs into ``rows``-row
    m-tiles (native ``pgb_plan_pack_rows``): a run that would cross an m-tile
    starts the next one while the sub-chunk's ``cap`` entries allow the
    padding.  Returns (start of every run, entries per sub-chunk) on the
    runs' device."""
    rl, rp = _host_i64(run_len), _host_i64(run_ptr)
    start = np.zeros(rl.size, dtype=np.int64)
    nent = np.zeros(max(n_subs, 0), dtype=np.int64)
    _lib.call("pgb_plan_pack_rows", rl.ctypes.data, rp.ctypes.data, int(n_subs), int(rows), int(cap),
              start.ctypes.data, nent.ctypes.data)
    dev = run_len.device
    return torch.from_numpy(start).to(dev), torch.from_numpy(nent).to(dev)
