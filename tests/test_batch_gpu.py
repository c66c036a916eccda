"""The batched runner (one CUDA graph for every beam's FDMT + statistics +
boxcar, one sort and one clustering for all beams) returns, beam by beam,
exactly what the plain per-beam pipeline returns: same candidate counts, same
delegates (bit-identical records) and same group sizes."""
import numpy as np
import pytest
import torch

from cpp_projects_b200 import synth
from cpp_projects_b200.pipeline import BatchedSearch, BeamShape, SearchPipeline, device_filterbank

pytestmark = pytest.mark.gpu


def _beams():
    rng = np.random.default_rng(8)
    out = []
    for i, (nchan, nsamp) in enumerate([(256, 20000), (512, 16384), (256, 33333), (1024, 20001),
                                         (512, 30000), (256, 17000)]):
        pulses = [synth.Pulse(int(rng.integers(1000, nsamp - 2000)), float(0.5 * nchan), 4, 2.5)]
        out.append(synth.Beam(nchan, nsamp, 1200.0, 1600.0, nchan, 100 + i, pulses))
    return out


@pytest.mark.parametrize("use_graph", [True, False])
def test_batched_equals_plain_per_beam(cuda, use_graph):
    beams = _beams()
    shapes = [BeamShape(b.nchan, b.nsamp, b.fmin, b.fmax, b.max_dt) for b in beams]
    inputs = [device_filterbank(b.nchan, b.nsamp, b.fmin, b.fmax, b.seed, b.pulses, cuda) for b in beams]
    plain = SearchPipeline(shapes, thr=6.0, capacity=1 << 22, device=cuda, fuse_depth=0)
    want = plain.run(inputs)
    batch = BatchedSearch(shapes, thr=6.0, capacity=1 << 22, use_graph=use_graph)
    for rep in range(3):  # eager run, then capture, then replay
        got = batch.run(inputs)
        for w, g in zip(want, got):
            assert g.n_candidates == w.n_candidates
            assert np.array_equal(g.delegates.view(np.uint32).reshape(-1), w.delegates.view(np.uint32).reshape(-1))
            assert np.array_equal(g.group_sizes, w.group_sizes)
    assert sum(r.n_candidates for r in want) > 0


def test_host_input_form_equals_device_form(cuda):
    beams = _beams()
    shapes = [BeamShape(b.nchan, b.nsamp, b.fmin, b.fmax, b.max_dt) for b in beams]
    inputs = [device_filterbank(b.nchan, b.nsamp, b.fmin, b.fmax, b.seed, b.pulses, cuda) for b in beams]
    host = [x.cpu().pin_memory() for x in inputs]
    batch = BatchedSearch(shapes, thr=6.0, capacity=1 << 22)
    want = batch.run(inputs)
    dev = [torch.full_like(x, float("nan")) for x in inputs]
    for rep in range(3):  # eager run, then capture, then replay
        got = batch.run_host(host, dev)
        for w, g in zip(want, got):
            assert g.n_candidates == w.n_candidates
            assert np.array_equal(g.delegates.view(np.uint32).reshape(-1), w.delegates.view(np.uint32).reshape(-1))
            assert np.array_equal(g.group_sizes, w.group_sizes)
    assert all(torch.equal(d, x) for d, x in zip(dev, inputs))



def test_explicit_schedules_equal_autotuned(cuda):
    """Plans built from saved schedules (what a profiled run replays) run the
    autotuner's kernels: same passes, same results."""
    from cpp_projects_b200.pipeline import tuned_schedule
    beams = _beams()[:3]
    shapes = [BeamShape(b.nchan, b.nsamp, b.fmin, b.fmax, b.max_dt) for b in beams]
    inputs = [device_filterbank(b.nchan, b.nsamp, b.fmin, b.fmax, b.seed, b.pulses, cuda) for b in beams]
    auto = SearchPipeline(shapes, thr=6.0, capacity=1 << 22, device=cuda, fuse_depth=-2)
    scheds = [tuned_schedule(s) for s in shapes]
    fixed = SearchPipeline(shapes, thr=6.0, capacity=1 << 22, device=cuda, schedules=scheds)
    for a, f in zip(auto.plans, fixed.plans):
        assert a.passes() == f.passes() and a.info.fuse_depth == f.info.fuse_depth
    want = auto.run(inputs)
    got = BatchedSearch(shapes, thr=6.0, capacity=1 << 22, schedules=scheds).run(inputs)
    for w, g in zip(want, got):
        assert g.n_candidates == w.n_candidates
        assert np.array_equal(g.delegates.view(np.uint32).reshape(-1), w.delegates.view(np.uint32).reshape(-1))
    with pytest.raises(ValueError):
        SearchPipeline(shapes, device=cuda, schedules=scheds[:1])


def test_submit_collect_equals_run(cuda):
    """The asynchronous form (submit run i + 1 before collecting run i, two
    candidate buffers) returns for every run exactly what bfs_batch_run
    returns, with inputs alternating between two sets; a third run in flight
    and a synchronous run while runs are in flight are refused."""
    from cpp_projects_b200 import BfsError
    beams = _beams()
    shapes = [BeamShape(b.nchan, b.nsamp, b.fmin, b.fmax, b.max_dt) for b in beams]
    ins = [[device_filterbank(b.nchan, b.nsamp, b.fmin, b.fmax, b.seed + 50 * k, b.pulses, cuda) for b in beams]
           for k in range(2)]
    batch = BatchedSearch(shapes, thr=6.0, capacity=1 << 22)
    want = [batch.run(ins[0]), batch.run(ins[1])]
    order = [0, 1, 0, 1, 0]
    batch.submit(ins[order[0]])
    for i, k in enumerate(order):
        if i + 1 < len(order):
            batch.submit(ins[order[i + 1]])
        got = batch.collect()
        for w, g in zip(want[k], got):
            assert g.n_candidates == w.n_candidates, (i, k)
            assert np.array_equal(g.delegates.view(np.uint32).reshape(-1), w.delegates.view(np.uint32).reshape(-1))
            assert np.array_equal(g.group_sizes, w.group_sizes)
    batch.submit(ins[0])
    batch.submit(ins[1])
    with pytest.raises(BfsError):
        batch.submit(ins[0])
    with pytest.raises(BfsError):
        batch.run(ins[0])
    for k in (0, 1):
        got = batch.collect()
        assert [g.n_candidates for g in got] == [w.n_candidates for w in want[k]]
    with pytest.raises(BfsError):
        batch.collect()


def test_destroy_with_a_run_in_flight(cuda):
    """A batch destroyed with a submitted run never collected waits for that
    run's kernels before freeing their buffers; the device stays usable."""
    beams = _beams()[:2]
    shapes = [BeamShape(b.nchan, b.nsamp, b.fmin, b.fmax, b.max_dt) for b in beams]
    ins = [device_filterbank(b.nchan, b.nsamp, b.fmin, b.fmax, b.seed, b.pulses, cuda) for b in beams]
    batch = BatchedSearch(shapes, thr=6.0, capacity=1 << 22)
    want = batch.run(ins)
    batch.submit(ins)
    del batch
    torch.cuda.synchronize()
    again = BatchedSearch(shapes, thr=6.0, capacity=1 << 22).run(ins)
    assert [g.n_candidates for g in again] == [w.n_candidates for w in want]
