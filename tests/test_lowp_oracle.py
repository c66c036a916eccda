"""CPU checks of the reduced-precision FDMT's oracle: the 16-bit rounding it
emulates is the IEEE binary16 / bfloat16 round-to-nearest-even of numpy and
torch, the emulation with no stored level is the FP32 FDMT, and the error
of the 16-bit planes against the FP64 FDMT is within the stated bounds."""
import ctypes

import numpy as np
import pytest
import torch

from cpp_projects_b200 import _capi
from oracle import pyoracle


def _values():
    rng = np.random.default_rng(0)
    parts = [rng.standard_normal(50000).astype(np.float32) * s
             for s in (1e-8, 1e-6, 6e-5, 1.0, 100.0, 3e4, 7e4)]
    bits = rng.integers(0, 2**32, 100000, dtype=np.uint64).astype(np.uint32).view(np.float32)
    edge = np.array([65504, 65519.99, 65520, -65520, 6.1035156e-05, 5.96e-8, 2.9802322e-08,
                     0.0, -0.0, 1.0009765625, 1.00048828125], np.float32)
    return np.concatenate(parts + [bits[np.isfinite(bits)], edge])


def test_round16_is_ieee_half_and_bfloat16():
    x = _values()
    with np.errstate(over="ignore"):
        want16 = x.astype(np.float16).astype(np.float32)
    assert np.array_equal(pyoracle.round16(x, pyoracle.PREC_F16).view(np.uint32), want16.view(np.uint32))
    wantb = torch.from_numpy(x).to(torch.bfloat16).float().numpy()
    assert np.array_equal(pyoracle.round16(x, pyoracle.PREC_BF16).view(np.uint32), wantb.view(np.uint32))


def test_lowp_without_stored_levels_is_fp32():
    fmin, fmax, nchan, ncols, mdt = 1200.0, 1600.0, 64, 700, 64
    x = np.random.default_rng(1).standard_normal((nchan, ncols)).astype(np.float32)
    niter = pyoracle.fdmt_rows(fmin, fmax, nchan, mdt).size - 1
    a = pyoracle.fdmt_lowp(fmin, fmax, x, nchan, ncols, mdt, pyoracle.PREC_F16, niter)
    assert np.array_equal(a, pyoracle.fdmt_f32(fmin, fmax, x, nchan, ncols, mdt))


@pytest.mark.parametrize("prec,bound_max,bound_rms", [(1, 2e-3, 1.5e-3), (2, 1.5e-2, 1.2e-2)])
def test_lowp_error_against_fp64(prec, bound_max, bound_rms):
    # N(0,1) with a per-channel bandpass gain in [0.5, 2]: error relative to
    # the output's max |value| and to its RMS
    fmin, fmax, nchan, ncols, mdt = 1100.0, 1500.0, 512, 4096, 512
    rng = np.random.default_rng(3)
    g = np.exp(rng.uniform(np.log(0.5), np.log(2.0), nchan)).astype(np.float32)[:, None]
    x = rng.standard_normal((nchan, ncols)).astype(np.float32) * g
    y64 = pyoracle.fdmt_f64(fmin, fmax, x, nchan, ncols, mdt)
    for kstore in (0, 4):
        y = pyoracle.fdmt_lowp(fmin, fmax, x, nchan, ncols, mdt, prec, kstore)
        e = y - y64
        assert np.abs(e).max() / np.abs(y64).max() < bound_max
        assert np.sqrt((e ** 2).mean() / (y64 ** 2).mean()) < bound_rms


def test_host_plan_accepts_16bit_and_counts_its_bytes():
    fmin, fmax, nchan, ncols, mdt = 1100.0, 1500.0, 4096, 256, 4096
    rows = pyoracle.fdmt_rows(fmin, fmax, nchan, mdt).astype(np.float64)
    info = {}
    for prec in (0, 1, 2):
        d = _capi.FdmtDesc(fmin=fmin, fmax=fmax, nchan=nchan, ncols=ncols, max_dt=mdt, precision=prec,
                           fuse_depth=0)
        p = ctypes.c_void_p()
        _capi.call("bfs_fdmt_plan_create_host", ctypes.byref(d), ctypes.byref(p))
        inf = _capi.FdmtInfo()
        _capi.call("bfs_fdmt_plan_info", p, ctypes.byref(inf))
        _capi.lib().bfs_fdmt_plan_destroy(p)
        info[prec] = inf.alg_bytes
    n = rows.size - 1
    b32 = ncols * (4 * nchan + 4 * rows[0] + 12 * rows[1:].sum())
    b16 = ncols * (4 * nchan + 2 * rows[0] + 6 * rows[1:n].sum() + 8 * rows[n])
    assert info[0] == pytest.approx(b32) and info[1] == pytest.approx(b16) and info[2] == pytest.approx(b16)
    # per chan-sample at 4096 x T, 1100-1500 MHz, FDMT only (the search adds
    # 2 reads of the FP32 output, 8 B): 177.9 B (FP32), 92.95 B (16-bit)
    assert info[0] / (nchan * ncols) == pytest.approx(177.9, abs=0.05)
    assert info[1] / (nchan * ncols) == pytest.approx(92.95, abs=0.05)
    d = _capi.FdmtDesc(fmin=fmin, fmax=fmax, nchan=nchan, ncols=ncols, max_dt=mdt, precision=3)
    with pytest.raises(_capi.BfsError):
        _capi.call("bfs_fdmt_plan_create_host", ctypes.byref(d), ctypes.byref(ctypes.c_void_p()))
