"""CPU tests: the oracle is pinned to the reference's own CFdmtCpu, and the
product's plan builder (C++, through the C ABI, host-only plan) reproduces the
reference's row tables exactly."""
import ctypes

import numpy as np
import pytest

from cpp_projects_b200 import _capi, synth
from oracle import pyoracle

# (fmin, fmax, nchan, ncols, max_dt): the workloads' band and channel counts plus odd counts
CASES = [
    (1200.0, 1600.0, 64, 1024, 64),
    (1200.0, 1600.0, 512, 4096, 512),
    (1100.0, 1500.0, 100, 2048, 77),
    (1200.0, 1600.0, 48, 2000, 48),
    (1200.0, 1328.0, 1024, 2048, 1024),
    (1100.0, 1500.0, 4096, 256, 4096),
    (1200.0, 1600.0, 3, 64, 5),
    (1200.0, 1600.0, 2, 64, 3),
]


def _host_plan(fmin, fmax, nchan, ncols, max_dt):
    desc = _capi.FdmtDesc(fmin=fmin, fmax=fmax, nchan=nchan, ncols=ncols, max_dt=max_dt)
    plan = ctypes.c_void_p()
    _capi.call("bfs_fdmt_plan_create_host", ctypes.byref(desc), ctypes.byref(plan))
    return plan


@pytest.mark.parametrize("case", CASES)
def test_product_plan_tables_match_oracle(case):
    fmin, fmax, nchan, ncols, max_dt = case
    plan = _host_plan(*case)
    try:
        rows = np.zeros(64, np.int32)
        orows = pyoracle.fdmt_rows(fmin, fmax, nchan, max_dt)
        _capi.call("bfs_fdmt_plan_rows", plan, rows.ctypes.data_as(ctypes.c_void_p), 64)
        np.testing.assert_array_equal(rows[: len(orows)], orows)
        for level in range(1, len(orows)):
            n = int(orows[level])
            a = np.zeros(n, np.int32); b = np.zeros(n, np.int32); s = np.zeros(n, np.int32)
            P = ctypes.c_void_p
            _capi.call("bfs_fdmt_plan_tables", plan, level, a.ctypes.data_as(P),
                       b.ctypes.data_as(P), s.ctypes.data_as(P), n)
            oa, ob, os_ = pyoracle.fdmt_tables(fmin, fmax, nchan, max_dt, level)
            np.testing.assert_array_equal(a, oa)
            np.testing.assert_array_equal(b, ob)
            np.testing.assert_array_equal(s, os_)
    finally:
        _capi.lib().bfs_fdmt_plan_destroy(plan)


def test_512_channel_plan_row_counts():
    # level totals of the 512-channel 1200-1600 MHz plan, maxDT 512 (the
    # figures the algorithmic-byte count of this shape is built from)
    rows = pyoracle.fdmt_rows(1200.0, 1600.0, 512, 512)
    assert list(rows) == [1536, 887, 700, 608, 557, 537, 524, 517, 514, 512]


@pytest.mark.parametrize("case", CASES[:5])
def test_oracle_bit_exact_vs_reference_cfdmtcpu(case):
    if pyoracle.ref_lib() is None:
        pytest.skip("reference CFdmtCpu not built (oracle/_ref)")
    fmin, fmax, nchan, ncols, max_dt = case
    x = np.random.default_rng(7).standard_normal((nchan, ncols)).astype(np.float32)
    ours = pyoracle.fdmt_f32(fmin, fmax, x, nchan, ncols, max_dt)
    ref = pyoracle.ref_fdmt_cpu(fmin, fmax, x, nchan, ncols, max_dt, threads=1)
    assert np.array_equal(ours.view(np.uint32), ref.view(np.uint32))
    ones = pyoracle.fdmt_f32(fmin, fmax, None, nchan, ncols, max_dt, b_ones=True)
    ref1 = pyoracle.ref_fdmt_cpu(fmin, fmax, None, nchan, ncols, max_dt, b_ones=True, threads=1)
    assert np.array_equal(ones, ref1)


def test_oracle_f32_close_to_f64():
    fmin, fmax, nchan, ncols, max_dt = CASES[1]
    x = np.random.default_rng(3).standard_normal((nchan, ncols)).astype(np.float32)
    a = pyoracle.fdmt_f32(fmin, fmax, x, nchan, ncols, max_dt)
    b = pyoracle.fdmt_f64(fmin, fmax, x.astype(np.float64), nchan, ncols, max_dt)
    scale = np.abs(b).max()
    assert np.abs(a - b).max() / scale < 1e-5


def test_pulse_lands_on_its_delay_row():
    beam = synth.Beam(64, 2048, 1200.0, 1600.0, 64, 5, [synth.Pulse(500, 40.0, 3, 5.0)])
    x = synth.filterbank(beam)
    out = pyoracle.fdmt_f32(beam.fmin, beam.fmax, x, beam.nchan, beam.nsamp, beam.max_dt)
    r, t = np.unravel_index(np.argmax(out), out.shape)
    assert abs(r - 40) <= 2 and 537 <= t <= 545
