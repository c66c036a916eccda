"""GPU parity at the shapes the batched search runs: the FDMT at 4096
channels (max delay 4096) under every kind of schedule the autotuner can
pick, bit for bit against the oracle in FP32 and against the oracle's exact
emulation of the 16-bit stores; one beam of each channel count of the
multi-beam workload (256, 512, 1024, 4096) searched end to end by the plain
per-beam pipeline and by the batched runner, each compared with the oracle's
search on the same DM-time plane -- candidate count, delegate records bit for
bit and group sizes; and the FP16 / BF16 forms' candidate recall against FP32
on a slice of the reduced-precision workload, with its bound written here."""
import functools

import numpy as np
import pytest
import torch

from cpp_projects_b200 import CFdmtGpu, search, synth
from cpp_projects_b200.pipeline import BatchedSearch, BeamShape, SearchPipeline
from oracle import pyoracle

pytestmark = pytest.mark.gpu

BAND = (1200.0, 1600.0)


def _bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


@functools.lru_cache(maxsize=4)
def _x4096(ncols):
    return np.random.default_rng(ncols).standard_normal((4096, ncols)).astype(np.float32)


@functools.lru_cache(maxsize=4)
def _want4096(ncols):
    return pyoracle.fdmt_f32(*BAND, _x4096(ncols), 4096, ncols, 4096)


# (fuse_depth, head_tile, seg_levels, seg_rows, seg_threads, seg_flags): the
# tuned choice, one pass per level, fused segments of 2 / 3 / 4 levels with
# 16, 24, 28 or 32 rows per tile, with and without a head (without: the first
# segment forms level 0 from the channels), the wide head tile, CTAs of 256 /
# 512 / 1024 threads, one input buffer per CTA
SCHEDULES = [(-2, 0, 0, 0, 0, 0), (3, 256, 1, 0, 0, 0), (3, 512, 3, 32, 0, 0), (3, 256, 4, 16, 0, 0),
             (0, 0, 3, 16, 0, 0), (4, 256, 2, 16, 0, 0), (2, 256, 3, 32, 0, 0), (0, 0, 4, 32, 1024, 0),
             (0, 0, 3, 32, 256, 1), (3, 256, 3, 16, 512, 1), (0, 0, 3, 28, 0, 1), (0, 0, 4, 24, 0, 1),
             (0, 0, 3, 28, 0, 0)]


@pytest.mark.parametrize("ncols", [8192, 5003])
@pytest.mark.parametrize("sched", SCHEDULES)
def test_fdmt_4096_channels_bit_exact(cuda, ncols, sched):
    fuse, tile, seg, rows, threads, flags = sched
    f = CFdmtGpu(*BAND, 4096, ncols, 4096, fuse_depth=fuse, head_tile=tile, seg_levels=seg, seg_rows=rows,
                 seg_threads=threads, seg_flags=flags)
    d_out = torch.full((4096, ncols), float("nan"), device=cuda)
    f.process_image(torch.from_numpy(_x4096(ncols)).to(cuda), d_out, False)
    assert np.array_equal(_bits(d_out.cpu().numpy()), _bits(_want4096(ncols)))


@pytest.mark.parametrize("prec", [1, 2])
@pytest.mark.parametrize("fuse", [-2, 3])
def test_fdmt_4096_channels_16bit_planes_bit_exact(cuda, prec, fuse):
    ncols = 4096
    x = _x4096(ncols)
    f = CFdmtGpu(*BAND, 4096, ncols, 4096, fuse_depth=fuse, precision=prec)
    d_out = torch.full((4096, ncols), float("nan"), device=cuda)
    f.process_image(torch.from_numpy(x).to(cuda), d_out, False)
    want = pyoracle.fdmt_lowp(*BAND, x, 4096, ncols, 4096, prec, f.info.fuse_depth)
    assert np.array_equal(_bits(d_out.cpu().numpy()), _bits(want))


# ---- end-to-end search, one beam per channel class --------------------------
THR, MODE, PARAM, METRICS = 7.0, 0, 5, (16, 8, 1 << 30)
CLASS_BEAMS = [(256, 20011), (512, 16384), (1024, 12289), (4096, 8192)]


def _class_beams():
    out = []
    for i, (nchan, nsamp) in enumerate(CLASS_BEAMS):
        rng = np.random.default_rng(40 + i)
        pulses = [synth.Pulse(int(rng.integers(500, nsamp - nchan - 100)), float(rng.uniform(0.2, 0.8) * nchan),
                              int(rng.integers(1, 17)), float(rng.uniform(0.6, 1.2)))
                  for _ in range(2)]
        out.append(synth.Beam(nchan, nsamp, *BAND, nchan, 500 + i, pulses))
    return out


def _normalise(y, stats):
    """The product's per-row normalisation, (x - mean) / std in float32 with
    one rounding per operation, 0 for a row of zero spread."""
    r = y.shape[0]
    m, s = stats[:r, None], stats[r:, None]
    with np.errstate(divide="ignore", invalid="ignore"):
        z = ((y - m).astype(np.float32) / s).astype(np.float32)
    z[np.broadcast_to(s == 0, z.shape)] = 0.0
    return z


def _oracle_search(y, stats):
    """Candidates, delegate records (in delegate order) and each delegate's
    group size from the oracle's boxcar and clustering on plane y normalised
    with `stats`."""
    c = pyoracle.boxcar(_normalise(y, stats), THR, MODE, PARAM, cap=1 << 24)
    perm, offs, dl = pyoracle.cluster(c, METRICS)
    pos = np.empty(len(perm), np.int64)
    pos[perm] = np.arange(len(perm))
    g = np.searchsorted(offs, pos[dl], side="right") - 1
    return len(c), c[dl], (offs[g + 1] - offs[g]).astype(np.int64)


def test_search_per_class_plain_and_batched_vs_oracle(cuda):
    beams = _class_beams()
    xs = [synth.filterbank(b) for b in beams]
    inputs = [torch.from_numpy(x).to(cuda) for x in xs]
    shapes = [BeamShape(b.nchan, b.nsamp, b.fmin, b.fmax, b.max_dt) for b in beams]
    plain = SearchPipeline(shapes, thr=THR, param=PARAM, metrics=METRICS, capacity=1 << 24, device=cuda,
                           fuse_depth=-2).run(inputs)
    batch = BatchedSearch(shapes, thr=THR, param=PARAM, metrics=METRICS, capacity=1 << 24)
    batched = batch.run(inputs)
    for b, x, got_p, got_b in zip(beams, xs, plain, batched):
        y = pyoracle.fdmt_f32(b.fmin, b.fmax, x, b.nchan, b.nsamp, b.max_dt)
        yd = torch.from_numpy(y).to(cuda)
        st = search.row_stats(yd).cpu().numpy()   # the row statistics both runners compute
        _, m, s = pyoracle.norm_rows(y)           # FP64 sums in another order: within 1 ulp
        assert np.abs(st[:b.max_dt].view(np.int32) - m.view(np.int32)).max() <= 1
        assert np.abs(st[b.max_dt:].view(np.int32) - s.view(np.int32)).max() <= 1
        n, dlg, sizes = _oracle_search(y, st)
        assert n > 0 and len(dlg) >= 1, b.nchan
        for got in (got_p, got_b):
            assert got.n_candidates == n, b.nchan
            assert np.array_equal(got.delegates.view(np.uint32).reshape(-1), dlg.view(np.uint32).reshape(-1))
            assert np.array_equal(got.group_sizes, sizes)


# ---- reduced precision: candidate recall against FP32 ------------------------
def _recall_beam():
    """A 16384-sample slice of the reduced-precision workload: 4096 channels,
    1100-1500 MHz, max delay 4096, the same bandpass gain model, 3 pulses."""
    full = synth.config3()
    rng = np.random.default_rng(33)
    pulses = []
    for _ in range(3):
        span = float(rng.uniform(0.1, 0.6) * 4095)
        width = int(rng.integers(1, 65))
        pulses.append(synth.Pulse(int(rng.integers(0, 16384 - int(span) - width)), span, width,
                                  float(rng.uniform(1.0, 3.0))))
    return synth.Beam(4096, 16384, full.fmin, full.fmax, 4096, 333, pulses, full.gain)


def test_16bit_planes_candidate_recall_against_fp32(cuda):
    beam = _recall_beam()
    x = torch.from_numpy(synth.filterbank(beam)).to(cuda)
    shape = [BeamShape(beam.nchan, beam.nsamp, beam.fmin, beam.fmax, beam.max_dt)]
    keys, found, ndel = {}, {}, {}
    for prec in (0, 1, 2):
        pipe = SearchPipeline(shape, thr=THR, param=PARAM, metrics=METRICS, capacity=1 << 26, device=cuda,
                              fuse_depth=-2, precision=prec)
        plane = pipe.plane[: beam.max_dt * beam.nsamp].view(beam.max_dt, beam.nsamp)
        pipe.plans[0].process_image_ws(x, plane, False, pipe.workspace)
        st = search.row_stats(plane)
        c, n = search.boxcar_gather(plane, THR, MODE, PARAM, stats=st, out=pipe.cands)
        c = search.cands_to_numpy(c)
        keys[prec] = set((c["mt"].astype(np.int64) << 32 | c["mdt"].astype(np.int64) << 8
                          | c["mwidth"].astype(np.int64)).tolist())
        # every injected pulse is detected at its delay and arrival sample
        found[prec] = [bool(((np.abs(c["mdt"] - p.span) <= 8)
                             & (np.abs(c["mt"] - (p.t0 + p.span)) <= 16 + p.width)).any())
                       for p in beam.pulses]
        ndel[prec] = len(pipe.run([x])[0].delegates)
    n32 = len(keys[0])
    assert n32 > 1000
    # recall bounds (measured at the full workload size: 99.99 % FP16, 99.93 % BF16)
    for prec, bound in ((1, 0.998), (2, 0.99)):
        assert len(keys[prec] & keys[0]) / n32 >= bound, prec
    assert all(all(f) for f in found.values()), found
    assert ndel[1] == ndel[0] and ndel[2] == ndel[0], ndel
