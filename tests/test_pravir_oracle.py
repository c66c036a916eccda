"""CPU checks of the Pravir plan kind (the reference's second FDMT variant,
MyVSLib_C++/FDMT_PRAVIR/): the oracle's restatement is bit-identical to the
reference's own FDMTCPU built from its sources; the product's host plan has
exactly the oracle's tables and delay grids; shapes the reference rejects are
rejected; the FP64 adjoint is the transpose (dot-product test)."""
import ctypes

import numpy as np
import pytest

from cpp_projects_b200 import _capi
from oracle import pyoracle

# (fmin, fmax, nchans, nsamps, dt_max, dt_step, dt_min)
CASES = [
    (1200.0, 1600.0, 64, 1000, 64, 1, 0),
    (1200.0, 1600.0, 100, 777, 80, 1, 0),     # odd sub-band counts (copies)
    (1100.0, 1500.0, 48, 600, 50, 2, 4),      # dt_step 2, dt_min 4
    (1200.0, 1600.0, 512, 4096, 512, 1, 0),   # config-0 band and delays
    (1200.0, 1328.0, 37, 999, 40, 1, 0),
    (1200.0, 1600.0, 3, 64, 5, 1, 0),
]


@pytest.mark.parametrize("case", CASES)
def test_oracle_matches_reference_fdmtcpu(case):
    if pyoracle.ref_pravir_lib() is None:
        pytest.skip("reference FDMTCPU not built (oracle/_ref)")
    fmin, fmax, nch, ns, dtm, st, dmin = case
    x = np.random.default_rng(nch).standard_normal((nch, ns)).astype(np.float32)
    want = pyoracle.ref_pravir_cpu(fmin, fmax, x, nch, ns, dtm, st, dmin, threads=4)
    got = pyoracle.pravir_fdmt(fmin, fmax, x, nch, ns, dtm, st, dmin)
    assert want is not None and got.shape == want.shape
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    grid = np.zeros(want.shape[0], np.int64)
    r = pyoracle.ref_pravir_lib()
    r.ref_pravir_dt_grid(fmin, fmax, nch, ns, 1.0, dtm, st, dmin, grid.ctypes.data_as(ctypes.c_void_p), grid.size)
    assert list(grid) == list(range(dmin, dtm + 1, st))[: len(grid)]


def _host_plan(case):
    fmin, fmax, nch, ns, dtm, st, dmin = case
    d = _capi.FdmtDesc(fmin=fmin, fmax=fmax, nchan=nch, ncols=ns, max_dt=dtm,
                       plan_kind=_capi.BFS_PLAN_PRAVIR, dt_step=st, dt_min=dmin)
    p = ctypes.c_void_p()
    _capi.call("bfs_fdmt_plan_create_host", ctypes.byref(d), ctypes.byref(p))
    return p


@pytest.mark.parametrize("case", CASES)
def test_product_plan_tables_match_oracle(case):
    fmin, fmax, nch, ns, dtm, st, dmin = case
    orows = pyoracle.pravir_rows(*case)
    p = _host_plan(case)
    P = ctypes.c_void_p
    try:
        rows = np.zeros(64, np.int32)
        _capi.call("bfs_fdmt_plan_rows", p, rows.ctypes.data_as(P), 64)
        np.testing.assert_array_equal(rows[: len(orows)], orows)
        info = _capi.FdmtInfo()
        _capi.call("bfs_fdmt_plan_info", p, ctypes.byref(info))
        assert info.out_rows == orows[-1] and info.fuse_depth == 0
        for lev in range(1, len(orows)):
            _, _, a, b, s = pyoracle.pravir_level(*case, lev)
            n = len(a)
            ga = np.zeros(n, np.int32); gb = np.zeros(n, np.int32); gs = np.zeros(n, np.int32)
            _capi.call("bfs_fdmt_plan_tables", p, lev, ga.ctypes.data_as(P), gb.ctypes.data_as(P),
                       gs.ctypes.data_as(P), n)
            np.testing.assert_array_equal(ga, a)
            np.testing.assert_array_equal(gb, b)
            np.testing.assert_array_equal(gs, s)
        cum0, dt0, *_ = pyoracle.pravir_level(*case, 0)
        _, dtn, *_ = pyoracle.pravir_level(*case, len(orows) - 1)
        out_dt = np.zeros(orows[-1], np.int32)
        cum = np.zeros(nch + 1, np.int32)
        l0 = np.zeros(max(orows[0], nch + 1), np.int32)
        _capi.call("bfs_fdmt_plan_delays", p, out_dt.ctypes.data_as(P), out_dt.size, cum.ctypes.data_as(P),
                   l0.ctypes.data_as(P), l0.size)
        np.testing.assert_array_equal(out_dt, dtn)
        np.testing.assert_array_equal(cum, cum0[: nch + 1])
        np.testing.assert_array_equal(l0[: orows[0]], dt0)
    finally:
        _capi.lib().bfs_fdmt_plan_destroy(p)


def test_rejections_follow_the_reference():
    # offsets reaching nsamps: the reference throws, the product returns BFS_ERR_ARG
    bad = (1100.0, 1500.0, 4096, 1000, 4096, 1, 0)
    with pytest.raises(ValueError):
        pyoracle.pravir_rows(*bad)
    if pyoracle.ref_pravir_lib() is not None:
        assert pyoracle.ref_pravir_lib().ref_pravir_rows(1100.0, 1500.0, 4096, 1000, 1.0, 4096, 1, 0) == -1
    with pytest.raises(_capi.BfsError) as e:
        _host_plan(bad)
    assert e.value.status == _capi.BFS_ERR_ARG
    d = _capi.FdmtDesc(fmin=1200.0, fmax=1600.0, nchan=64, ncols=1000, max_dt=64,
                       plan_kind=_capi.BFS_PLAN_PRAVIR, fuse_depth=2)
    with pytest.raises(_capi.BfsError):
        _capi.call("bfs_fdmt_plan_create_host", ctypes.byref(d), ctypes.byref(ctypes.c_void_p()))


@pytest.mark.parametrize("case", CASES[:3])
def test_pravir_adjoint_is_the_transpose(case):
    fmin, fmax, nch, ns, dtm, st, dmin = case
    rng = np.random.default_rng(3)
    x = rng.standard_normal((nch, ns))
    y = pyoracle.pravir_fdmt(fmin, fmax, x, nch, ns, dtm, st, dmin, dtype=np.float64)
    g = rng.standard_normal(y.shape)
    gx = pyoracle.pravir_adjoint(fmin, fmax, g, nch, ns, dtm, st, dmin, dtype=np.float64)
    a, b = (y * g).sum(), (x * gx).sum()
    assert abs(a - b) <= 1e-10 * abs(a)
