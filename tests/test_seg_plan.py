"""CPU: the fused merge segments (k_fdmt_seg) emulated exactly as the kernel
indexes shared memory -- every load, merge and store of every tile -- and the
whole pass schedule after the head compared bit for bit with the oracle's
FDMT.  Shared memory starts as NaN, so a written sample that depended on a
value the kernel never loaded would come out NaN (and differ); every shared
index is bounds-checked against the kernel's allocation."""
import ctypes

import numpy as np
import pytest

from cpp_projects_b200 import _capi
from oracle import pyoracle

P = ctypes.c_void_p
TILE_INTS = 8
PASS_INTS = 13


def plan_passes(fmin, fmax, nchan, ncols, max_dt, fuse, seg_levels=0, seg_rows=0, seg_flags=0):
    """(head depth, rows per level, passes): each pass is (params, tiles, ent)."""
    desc = _capi.FdmtDesc(fmin=fmin, fmax=fmax, nchan=nchan, ncols=ncols, max_dt=max_dt,
                          fuse_depth=fuse, seg_levels=seg_levels, seg_rows=seg_rows, seg_flags=seg_flags)
    plan = ctypes.c_void_p()
    _capi.call("bfs_fdmt_plan_create_host", ctypes.byref(desc), ctypes.byref(plan))
    try:
        info = _capi.FdmtInfo()
        _capi.call("bfs_fdmt_plan_info", plan, ctypes.byref(info))
        rows = np.zeros(info.niter + 1, np.int32)
        _capi.call("bfs_fdmt_plan_rows", plan, rows.ctypes.data_as(P), rows.size)
        n = ctypes.c_int(0)
        _capi.call("bfs_fdmt_plan_passes", plan, ctypes.byref(n), None, 0)
        params = np.zeros(max(1, n.value) * PASS_INTS, np.int32)
        _capi.call("bfs_fdmt_plan_passes", plan, ctypes.byref(n), params.ctypes.data_as(P), params.size)
        passes = []
        for i in range(n.value):
            pr = params[i * PASS_INTS:(i + 1) * PASS_INTS].copy()
            nt, ne = int(pr[10]), int(pr[11])
            tiles = np.zeros(max(1, nt) * TILE_INTS, np.int32)
            ent = np.zeros(max(1, ne) * 4, np.int32)
            if nt:
                _capi.call("bfs_fdmt_plan_segment", plan, i, tiles.ctypes.data_as(P), tiles.size,
                           ent.ctypes.data_as(P), ent.size)
            passes.append((pr, tiles.reshape(-1, TILE_INTS)[:nt], ent.reshape(-1, 4)[:ne]))
        return int(info.fuse_depth), rows, passes
    finally:
        _capi.lib().bfs_fdmt_plan_destroy(plan)


def level_planes(fmin, fmax, x, nchan, ncols, max_dt, upto):
    """Planes of levels 0..upto: level 0 by the running-mean recurrence (one
    float32 rounding per operation, 0 before row r), merges from the oracle's
    tables."""
    r0 = pyoracle.fdmt_rows(fmin, fmax, nchan, max_dt)
    r0c = int(r0[0]) // nchan
    lv0 = np.zeros((nchan, r0c, ncols), np.float32)
    v = x.astype(np.float32).copy()
    lv0[:, 0] = v
    for r in range(1, r0c):
        xs = np.zeros_like(v)
        xs[:, r:] = x[:, :-r] if r < ncols else 0
        nv = ((v * np.float32(r)).astype(np.float32) + xs).astype(np.float32) / np.float32(r + 1)
        v = nv.astype(np.float32)
        v[:, :r] = 0
        lv0[:, r] = v
    planes = [lv0.reshape(nchan * r0c, ncols)]
    for lev in range(1, upto + 1):
        a, b, s = pyoracle.fdmt_tables(fmin, fmax, nchan, max_dt, lev)
        planes.append(merge_level(planes[-1], a, b, s))
    return planes


def merge_level(plane, a, b, s):
    ncols = plane.shape[1]
    nxt = plane[a].copy()
    for g in range(len(a)):
        if b[g] >= 0:
            sh = int(s[g])
            if sh < ncols:
                nxt[g, sh:] = (plane[a[g], sh:] + plane[b[g], :ncols - sh]).astype(np.float32)
    return nxt


def emulate_seg(src, pr, tiles, ent, ncols, out_rows, fill=0.0):
    """k_fdmt_seg over every (row tile, time tile) of one fused pass.  Each
    shared buffer (X: levels l0, l0+2, ..; Y: l0+1, ..) is its own array of
    its rows, a row of -0.0 and a guard row, NaN where nothing was stored;
    every index is checked against that buffer alone.  The kernel loads 0 for
    samples outside [0, ncols); fill=NaN shows that no written sample
    depends on them (the t >= shift test keeps them out)."""
    l0, l1, G, TT, nc, pitch, rx, ry, max_ent, max_thr = (int(v) for v in pr[:10])
    r0c = int(pr[12])
    m = l1 - l0 + (1 if r0c else 0)  # kernel levels above the input rows (an input
    assert pitch == 32 * nc and TT % 32 == 0  # segment forms level 0 as its first)
    out = np.full((out_rows, ncols), np.nan, np.float32)
    cols = np.arange(nc * 32)
    ocols = np.arange(TT)
    written = np.zeros(out_rows, np.int64)
    for tile in tiles:
        e0, n = int(tile[0]), [int(v) for v in tile[1:2 + m]]
        assert n[0] <= rx and all(n[i] <= (ry if i & 1 else rx) for i in range(m))
        assert sum(n) <= max_ent
        for tb in range((ncols + TT - 1) // TT):
            t0 = tb * TT
            bufs = []
            for rows in (rx, ry):
                b = np.full((rows + 2) * pitch, np.nan, np.float32)
                b[rows * pitch:(rows + 1) * pitch] = np.float32(-0.0)
                bufs.append(b)
            x, y = bufs
            e = ent[e0:]
            for row, lead, _, dst in e[:n[0]]:
                assert 0 <= row < src.shape[0] and lead % 4 == 0 and dst % 4 == 0
                t = t0 - lead + cols
                ok = (t >= 0) & (t < ncols)
                v = np.full(cols.size, fill, np.float32)
                v[ok] = src[row, t[ok]]
                idx = dst + cols
                assert idx.min() >= 0 and idx.max() < rx * pitch
                x[idx] = v
            e = e[n[0]:]
            fast = t0 >= max_thr
            for lev in range(1, m + 1):
                q = e[:n[lev]]
                rd = x if lev % 2 == 1 else y
                c = ocols if lev == m else cols
                if r0c and lev == 1:
                    # level 0 from the channels: running mean of row r over
                    # x[t-r .. t], one float32 rounding per operation, 0 before r
                    for xo, _, thr, w in q:
                        r, dst = (w >> 20) & 15, w & 0xFFFFF
                        assert r < r0c
                        ia = xo + cols
                        assert (ia - r).min() >= 0 and ia.max() < rd.size
                        v = rd[ia].copy()
                        for k in range(1, r + 1):
                            mm = v if k == 1 else (v * np.float32(k)).astype(np.float32)
                            v = ((mm + rd[ia - k]).astype(np.float32) / np.float32(k + 1)).astype(np.float32)
                        v = np.where(cols >= thr - t0, v, np.float32(0.0))
                        idx = dst + cols
                        assert idx.min() >= 0 and idx.max() < ry * pitch
                        y[idx] = v
                    e = e[n[lev]:]
                    continue
                ia = q[:, 0:1] + c[None, :]
                ib = q[:, 1:2] + c[None, :]
                assert ia.min() >= 0 and ia.max() < rd.size and ib.min() >= 0 and ib.max() < rd.size
                a, b = rd[ia], rd[ib]
                cond = fast | (c[None, :] >= (q[:, 2:3] - t0))
                v = np.where(cond, (a + b).astype(np.float32), a)
                if lev < m:
                    wr, wrows = (y, ry) if lev % 2 == 1 else (x, rx)
                    idx = q[:, 3:4] + c[None, :]
                    assert idx.min() >= 0 and idx.max() < wrows * pitch  # never the -0.0 or guard row
                    wr[idx] = v
                else:
                    for j, row in enumerate(q[:, 3]):
                        tt = t0 + c
                        w = tt < ncols
                        out[row, tt[w]] = v[j, w]
                        written[row] += int(w.sum())
                e = e[n[lev]:]
    assert np.all(written == ncols), "every output row is written once per sample"
    return out


def run_schedule(fmin, fmax, nchan, ncols, max_dt, fuse, seg_levels, seg_rows, seed, with_zeros=False):
    k, rows, passes = plan_passes(fmin, fmax, nchan, ncols, max_dt, fuse, seg_levels, seg_rows)
    x = np.random.default_rng(seed).standard_normal((nchan, ncols)).astype(np.float32)
    if with_zeros:  # signed zeros and tiny values through the level-0 means
        x[:, ::7] = np.float32(-0.0)
        x[::3, 5::11] = np.float32(1e-40)
    niter = rows.size - 1
    planes = level_planes(fmin, fmax, x, nchan, ncols, max_dt, niter)
    cur, lev = planes[k], k
    fused = 0
    for pr, tiles, ent in passes:
        l0, l1 = int(pr[0]), int(pr[1])
        assert l0 == lev and l1 > l0
        if int(pr[12]):  # input segment: reads the channels, forms level 0 itself
            assert l0 == 0 and k == 0 and len(tiles)
            fused += 1
            strict = emulate_seg(x, pr, tiles, ent, ncols, int(rows[l1]), fill=np.nan)
            cur = emulate_seg(x, pr, tiles, ent, ncols, int(rows[l1]))
            assert np.array_equal(cur.view(np.uint32), planes[l1].view(np.uint32)), f"levels 1..{l1}"
            assert np.array_equal(strict.view(np.uint32), cur.view(np.uint32))
        elif len(tiles) == 0:
            assert l1 == l0 + 1
            a, b, s = pyoracle.fdmt_tables(fmin, fmax, nchan, max_dt, l1)
            cur = merge_level(cur, a, b, s)
        else:
            fused += 1
            strict = emulate_seg(cur, pr, tiles, ent, ncols, int(rows[l1]), fill=np.nan)
            cur = emulate_seg(cur, pr, tiles, ent, ncols, int(rows[l1]))
            assert np.array_equal(cur.view(np.uint32), planes[l1].view(np.uint32)), f"levels {l0}..{l1}"
            assert np.array_equal(strict.view(np.uint32), cur.view(np.uint32))
        lev = l1
    assert lev == niter
    want = pyoracle.fdmt_f32(fmin, fmax, x, nchan, ncols, max_dt)
    assert np.array_equal(cur.view(np.uint32), want.view(np.uint32))
    return fused


@pytest.mark.parametrize("case", [
    # (fmin, fmax, nchan, ncols, max_dt, head depth, seg_levels, seg_rows)
    (1200.0, 1600.0, 64, 700, 64, 2, 2, 16),     # several row tiles, ragged last time tile
    (1200.0, 1600.0, 256, 600, 256, 3, 3, 0),    # levels 4..8 as 3 + 2
    (1200.0, 1600.0, 256, 300, 256, 3, 5, 16),   # one 5-level segment
    (1100.0, 1500.0, 128, 513, 100, 0, 4, 0),    # no head: segments from level 0
    (1200.0, 1600.0, 99, 531, 99, 0, 3, 8),      # odd sub-band counts: carried rows
    (1200.0, 1328.0, 100, 1100, 80, 2, 3, 16),   # head of 4 channels, 25 sub-bands after it
])
def test_segment_emulation_matches_oracle(case):
    fmin, fmax, nchan, ncols, max_dt, fuse, seg_levels, seg_rows = case
    fused = run_schedule(fmin, fmax, nchan, ncols, max_dt, fuse, seg_levels, seg_rows, seed=nchan)
    assert fused >= 1


@pytest.mark.parametrize("case", [
    (1200.0, 1600.0, 64, 700, 64, 0, 3, 16),
    (1100.0, 1500.0, 128, 513, 100, 0, 4, 0),
    (1200.0, 1600.0, 99, 531, 99, 0, 2, 8),      # odd channel count: a carried level-1 row
    (1200.0, 1328.0, 64, 1031, 200, 0, 3, 32),   # max delay > channels: 5 level-0 rows per channel
    (1200.0, 1600.0, 128, 900, 128, 0, 3, 28),   # 28 rows per tile (a row tile count not a power of 2)
    (1200.0, 1600.0, 96, 777, 96, 0, 4, 24),     # 24 rows per tile, 4 levels
])
def test_input_segment_emulation_matches_oracle(case):
    """No head: the first segment stages the channels and forms level 0 in
    shared memory (no level-0 plane); signed zeros and subnormals included."""
    fmin, fmax, nchan, ncols, max_dt, fuse, seg_levels, seg_rows = case
    k, rows, passes = plan_passes(fmin, fmax, nchan, ncols, max_dt, fuse, seg_levels, seg_rows)
    assert int(passes[0][0][12]) >= 1, "the first pass is an input segment"
    run_schedule(fmin, fmax, nchan, ncols, max_dt, fuse, seg_levels, seg_rows, seed=nchan + 1, with_zeros=True)


def test_segment_geometry_at_search_shapes():
    """Default schedules at the batched search's channel counts: every fused
    pass fits an SM's shared memory, its tiles write each output row once, and
    every shared index stays inside the allocation (the bounds the kernel
    relies on, checked from the tables alone)."""
    for nchan in (256, 512, 1024, 4096):
        k, rows, passes = plan_passes(1200.0, 1600.0, nchan, 1 << 17, nchan, 3)
        assert k == 3
        assert sum(1 for pr, t, e in passes if len(t)) >= 1
        for pr, tiles, ent in passes:
            if len(tiles) == 0:
                continue
            l0, l1, G, TT, nc, pitch, rx, ry, max_ent = (int(v) for v in pr[:9])
            m = l1 - l0
            smem = ((2 * (rx + 2) + ry + 2) * pitch) * 4 + 3 * max_ent * 16
            assert smem <= 227 * 1024 and nc in (9, 10, 12)
            seen = np.zeros(int(rows[l1]), np.int64)
            for tile in tiles:
                e0, n = int(tile[0]), [int(v) for v in tile[1:2 + m]]
                e = ent[e0:]
                inp = e[:n[0]]
                assert inp[:, 0].min() >= 0 and inp[:, 0].max() < rows[l0]
                e = e[n[0]:]
                for lev in range(1, m + 1):
                    q = e[:n[lev]]
                    span = TT if lev == m else 32 * nc
                    below = rx if lev % 2 == 1 else ry
                    assert q[:, :2].min() >= 0 and q[:, :2].max() + span <= (below + 2) * pitch
                    if lev == m:
                        seen[q[:, 3]] += 1
                    e = e[n[lev]:]
            assert np.all(seen == 1)


@pytest.mark.parametrize("rows_per_tile", [24, 28])
@pytest.mark.parametrize("levels", [3, 4])
def test_input_segment_geometry_at_search_shapes(rows_per_tile, levels):
    """Single-buffered input segments of 24 / 28 rows per tile (autotuner
    candidates) at the batched search's channel counts: the shared memory
    fits an SM (at 28 rows and 3 levels, half of one, so two CTAs share it),
    the channels staged are inside the input, every level-0 row's look-back
    of r samples and its 32 nc positions stay inside buffer X, its
    destination inside buffer Y, every merge inside its buffers, and each
    output row of the pass is written once."""
    for nchan in (256, 512, 1024, 4096):
        k, rows, passes = plan_passes(1200.0, 1600.0, nchan, 1 << 17, nchan, 0, levels, rows_per_tile,
                                      _capi.BFS_SEG_SINGLE_BUFFER)
        pr, tiles, ent = passes[0]
        assert k == 0 and int(pr[12]) >= 1 and len(tiles)   # an input segment
        l0, l1, G, TT, nc, pitch, rx, ry, max_ent = (int(v) for v in pr[:9])
        assert l0 == 0 and G in (rows_per_tile, 16) and nc in (9, 10, 12)
        smem = (((rx + 2) + ry + 2) * pitch) * 4 + max_ent * 16
        assert smem <= 227 * 1024
        if rows_per_tile == 28 and levels == 3:
            assert smem <= 113 * 1024
        m = l1 - l0
        seen = np.zeros(int(rows[l1]), np.int64)
        for tile in tiles:
            e0, n = int(tile[0]), [int(v) for v in tile[1:2 + m + 1]]
            e = ent[e0:]
            inp = e[:n[0]]
            assert inp[:, 0].min() >= 0 and inp[:, 0].max() < nchan
            assert inp[:, 3].min() >= 0 and inp[:, 3].max() + 32 * nc <= (rx + 2) * pitch
            e = e[n[0]:]
            q = e[:n[1]]                                  # level-0 rows from the staged channels
            r = (q[:, 3] >> 20) & 15
            assert (q[:, 0] - r).min() >= 0 and q[:, 0].max() + 32 * nc <= (rx + 2) * pitch
            assert (q[:, 3] & 0xFFFFF).max() + 32 * nc <= (ry + 2) * pitch
            e = e[n[1]:]
            for lev in range(2, m + 2):
                q = e[:n[lev]]
                last = lev == m + 1
                span = TT if last else 32 * nc
                below = ry if lev % 2 == 0 else rx
                assert q[:, :2].min() >= 0 and q[:, :2].max() + span <= (below + 2) * pitch
                if last:
                    seen[q[:, 3]] += 1
                else:
                    above = rx if lev % 2 == 0 else ry
                    assert q[:, 3].max() + span <= (above + 2) * pitch
                e = e[n[lev]:]
        assert np.all(seen == 1), nchan


def test_segment_options_are_checked():
    with pytest.raises(_capi.BfsError):
        plan_passes(1200.0, 1600.0, 64, 500, 64, 2, seg_levels=9)
    with pytest.raises(_capi.BfsError):  # explicit segments are FP32-only
        desc = _capi.FdmtDesc(fmin=1200.0, fmax=1600.0, nchan=64, ncols=500, max_dt=64, fuse_depth=2,
                              precision=1, seg_levels=3)
        plan = ctypes.c_void_p()
        _capi.call("bfs_fdmt_plan_create_host", ctypes.byref(desc), ctypes.byref(plan))
    k, rows, passes = plan_passes(1200.0, 1600.0, 64, 500, 64, 2, seg_levels=1)
    assert all(len(t) == 0 for _, t, _ in passes) and len(passes) == rows.size - 1 - k


def _check_pass_geometry(pr, tiles, ent, rows, nchan, single):
    """The bounds k_fdmt_seg relies on, from one fused pass's tables: shared
    memory within an SM, staged rows inside the input, every shared read and
    write inside its buffer (level-0 rows of an input segment including their
    look-back of r samples), each output row of the pass written once."""
    l0, l1, G, TT, nc, pitch, rx, ry, max_ent = (int(v) for v in pr[:9])
    r0c = int(pr[12])
    xs = (rx + 2) * pitch                       # the X buffer in use (either of two, or the one)
    smem = (((1 if single else 2) * (rx + 2) + ry + 2) * pitch) * 4 + (1 if single else 3) * max_ent * 16
    assert smem <= 227 * 1024 and nc in (9, 10, 12)
    m = l1 - l0 + (1 if r0c > 0 else 0)         # shared-memory levels + the one written to HBM
    seen = np.zeros(int(rows[l1]), np.int64)
    for tile in tiles:
        e0, n = int(tile[0]), [int(v) for v in tile[1:2 + m]]
        e = ent[e0:]
        inp = e[:n[0]]
        assert inp[:, 0].min() >= 0 and inp[:, 0].max() < (nchan if r0c > 0 else rows[l0])
        assert inp[:, 3].min() >= 0 and inp[:, 3].max() + 32 * nc <= xs
        e = e[n[0]:]
        for lev in range(1, m + 1):
            q = e[:n[lev]]
            e = e[n[lev]:]
            if len(q) == 0:
                continue
            below = rx if lev % 2 == 1 else ry
            above = ry if lev % 2 == 1 else rx
            if r0c > 0 and lev == 1:             # level 0 formed from the staged channels
                r = (q[:, 3] >> 20) & 15
                assert r.max() < r0c
                assert (q[:, 0] - r).min() >= 0 and q[:, 0].max() + 32 * nc <= xs
                assert (q[:, 3] & 0xFFFFF).max() + 32 * nc <= (ry + 2) * pitch
                continue
            span = TT if lev == m else 32 * nc
            assert q[:, :2].min() >= 0 and q[:, :2].max() + span <= (below + 2) * pitch
            if lev == m:
                seen[q[:, 3]] += 1
            else:
                assert q[:, 3].min() >= 0 and q[:, 3].max() + span <= (above + 2) * pitch
    assert np.all(seen == 1)


@pytest.mark.parametrize("nchan,max_dt", [(256, 256), (512, 512), (1024, 1024), (4096, 4096), (96, 96),
                                          (300, 150)])
def test_every_tuner_schedule_has_sound_geometry(nchan, max_dt):
    """Every schedule the autotuner may time (input segments of 2-4 levels x
    16 / 24 / 28 / 32 rows x one or two input buffers; heads of depth 2-4 with
    16 / 32 rows), at the search's channel counts and odd ones: the plan is
    either refused or every fused pass keeps the kernel's bounds."""
    built = 0
    for ncols in (5003, 1 << 15):
        for seg in (2, 3, 4):
            cands = [(0, rows, flags) for rows in (16, 24, 28, 32) for flags in (0, 1)]
            cands += [(k, rows, 0) for k in (2, 3, 4) for rows in (16, 32)]
            for fuse, rows_per_tile, flags in cands:
                try:
                    k, rows, passes = plan_passes(1200.0, 1600.0, nchan, ncols, max_dt, fuse, seg, rows_per_tile,
                                                  flags)
                except _capi.BfsError:
                    continue                     # not usable for this shape: the tuner skips it
                for pr, tiles, ent in passes:
                    if len(tiles):
                        _check_pass_geometry(pr, tiles, ent, rows, nchan, flags == 1)
                built += 1
    assert built > 0
