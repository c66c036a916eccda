"""CPU: the fused FDMT head's plan (channel groups, shared-memory row tables,
halos) emulated exactly as the k_fdmt_head kernel indexes it, compared with
the oracle's level-k plane.  This checks the halo/look-back reasoning and
every shared-memory index bound without a GPU."""
import ctypes

import numpy as np
import pytest

from cpp_projects_b200 import _capi
from oracle import pyoracle

GROUP_INTS = 2 + 2 * 9  # HeadGroup: halo, out_row0, rows[9], tab_off[9]


def head_plan(fmin, fmax, nchan, ncols, max_dt, fuse):
    desc = _capi.FdmtDesc(fmin=fmin, fmax=fmax, nchan=nchan, ncols=ncols, max_dt=max_dt,
                          fuse_depth=fuse)
    plan = ctypes.c_void_p()
    _capi.call("bfs_fdmt_plan_create_host", ctypes.byref(desc), ctypes.byref(plan))
    params = np.zeros(9, np.int32)
    P = ctypes.c_void_p
    _capi.call("bfs_fdmt_plan_head", plan, params.ctypes.data_as(P), None, 0, None, 0)
    ng, nt = int(params[7]), int(params[8])
    groups = np.zeros(max(ng, 1) * GROUP_INTS, np.int32)
    tab = np.zeros(max(nt, 1) * 4, np.int32)
    _capi.call("bfs_fdmt_plan_head", plan, params.ctypes.data_as(P), groups.ctypes.data_as(P),
               groups.size, tab.ctypes.data_as(P), tab.size)
    rows = np.zeros(64, np.int32)
    _capi.call("bfs_fdmt_plan_rows", plan, rows.ctypes.data_as(P), 64)
    _capi.lib().bfs_fdmt_plan_destroy(plan)
    return params, groups.reshape(-1, GROUP_INTS)[:ng], tab.reshape(-1, 4)[:nt], rows


def level0_column(x, c, t, r0c, ncols):
    """The kernel's level-0 values of channel c at sample t (all rows)."""
    out = np.zeros(r0c, np.float32)
    if t < 0:
        return out
    v = np.float32(x[c, t]) if t < ncols else np.float32(0)
    out[0] = v
    for r in range(1, r0c):
        if t >= r:
            xv = np.float32(x[c, t - r]) if t - r < ncols else np.float32(0)
            v = np.float32(np.float32(np.float32(v * np.float32(r)) + xv) / np.float32(r + 1))
            out[r] = v
    return out


def level0_staged(xs, u, t, r0c):
    """level0_column as the kernel computes it from the staged input window."""
    out = np.zeros(r0c, np.float32)
    v = np.float32(xs[u])
    out[0] = v
    for r in range(1, r0c):
        if t >= r:
            xv = np.float32(xs[u - r]) if u >= r else np.float32(0)
            v = np.float32(np.float32(np.float32(v * np.float32(r)) + xv) / np.float32(r + 1))
            out[r] = v
    return out


def emulate_head(x, params, groups, tab, r0c, ncols, rows_k):
    depth, G, tile, W, rows_a, rows_b = (int(v) for v in params[:6])
    out = np.full((rows_k, ncols), np.nan, np.float32)
    ntiles = (ncols + tile - 1) // tile
    for gi, g in enumerate(groups):
        halo, out_row0 = int(g[0]), int(g[1])
        rows = g[2:11]
        toff = g[11:20]
        for tb in range(ntiles):
            u = np.arange(W)
            t = tb * tile - halo + u
            a = np.zeros((rows_a, W), np.float32)
            b = np.zeros((rows_b, W), np.float32)
            assert G * r0c <= rows_a
            assert G <= rows_b  # buffer B stages the group's input rows
            for c in range(G):
                # the kernel reads x[t - r] from the staged window: 0 before it
                xs = np.zeros(W, np.float32)
                ok = (t >= 0) & (t < ncols)
                xs[ok] = x[gi * G + c, t[ok]]
                for ui in range(W):
                    a[c * r0c:(c + 1) * r0c, ui] = level0_staged(xs, ui, int(t[ui]), r0c)
            # the staged entries as the kernel forms them: byte offsets of the
            # tail row and of the head row minus its shift, the first local
            # column that adds the head row, the destination offset
            t0 = tb * tile - halo
            neg0 = max(0, -t0)
            src, dst = a.reshape(-1), b.reshape(-1)
            for lev in range(1, depth + 1):
                e = tab[int(toff[lev]): int(toff[lev]) + int(rows[lev])]
                res = np.zeros((int(rows[lev]), W), np.float32)
                for j, (ea, eb, es, _) in enumerate(e):
                    fx, fy, fz = ea * W * 4, (eb * W - es) * 4, es + neg0
                    fw = j * W * 4 if lev < depth else j
                    ia = fx // 4 + u
                    assert ia.min() >= 0 and ia.max() < src.size
                    v = src[ia].copy()
                    ok = u >= fz
                    assert np.array_equal(ok, (t >= es) & (u >= es))
                    ib = fy // 4 + u[ok]
                    if ib.size:
                        assert ib.min() >= eb * W and ib.max() < (eb + 1) * W <= src.size
                        v[ok] = (v[ok] + src[ib]).astype(np.float32)
                    if lev < depth:
                        idst = fw // 4 + u
                        assert idst.min() >= 0 and idst.max() < dst.size
                        dst[idst] = v
                    res[j] = v
                if lev < depth:
                    src, dst = dst, src
                else:
                    wr = (u >= halo) & (u < halo + tile) & (t < ncols)
                    out[out_row0: out_row0 + res.shape[0]][:, t[wr]] = res[:, wr]
    return out


def oracle_level_plane(fmin, fmax, x, nchan, ncols, max_dt, level):
    """Level-`level` plane from the oracle's tables (level 0 via the recurrence)."""
    r0 = pyoracle.fdmt_rows(fmin, fmax, nchan, max_dt)
    r0c = int(r0[0]) // nchan
    plane = np.zeros((int(r0[0]), ncols), np.float32)
    for c in range(nchan):
        for t in range(ncols):
            plane[c * r0c:(c + 1) * r0c, t] = level0_column(x, c, t, r0c, ncols)
    for lev in range(1, level + 1):
        a, b, s = pyoracle.fdmt_tables(fmin, fmax, nchan, max_dt, lev)
        nxt = np.zeros((len(a), ncols), np.float32)
        for g in range(len(a)):
            nxt[g] = plane[a[g]]
            if b[g] >= 0:
                sh = int(s[g])
                nxt[g, sh:] = (plane[a[g], sh:] + plane[b[g], : ncols - sh]).astype(np.float32)
        plane = nxt
    return plane, r0c


@pytest.mark.parametrize("case,fuse", [
    ((1200.0, 1600.0, 64, 600, 64), -1),
    ((1200.0, 1600.0, 64, 300, 64), 2),
    ((1100.0, 1500.0, 32, 513, 40), 3),
    ((1200.0, 1328.0, 16, 300, 16), 4),
])
def test_head_emulation_matches_oracle(case, fuse):
    fmin, fmax, nchan, ncols, max_dt = case
    params, groups, tab, rows = head_plan(*case, fuse)
    depth = int(params[0])
    assert depth >= 1
    assert int(params[3]) % 32 == 0 and int(params[3]) <= 1024
    x = np.random.default_rng(depth).standard_normal((nchan, ncols)).astype(np.float32)
    want, r0c = oracle_level_plane(fmin, fmax, x, nchan, ncols, max_dt, depth)
    got = emulate_head(x, params, groups, tab, r0c, ncols, int(rows[depth]))
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


def test_head_autotune_keeps_two_ctas_per_sm():
    for nchan in (256, 512, 1024, 4096):
        params, groups, tab, rows = head_plan(1200.0, 1600.0, nchan, 65536, nchan, -1)
        assert int(params[0]) >= 3, nchan
        assert int(params[6]) <= 113 * 1024
    # odd channel counts cannot be grouped: no fused head
    params, *_ = head_plan(1200.0, 1600.0, 99, 1000, 99, -1)
    assert int(params[0]) == 0
