"""FDMT + normalise + boxcar + cluster over many beams (host orchestration).

The per-beam chain is the reference's search path
(MyVSLib_C++/CDMT/Chunk_gpu.cu:347-425 and Clusterization.cu:17-166): FDMT
of the beam's filterbank, per-delay-row normalisation statistics, boxcar
detection with compaction (normalisation fused into the boxcar's load),
then three-pass clustering and delegates.  ``SearchPipeline`` runs it beam
after beam on one stream with plans sharing a single FDMT workspace and a
single DM-time plane, so device memory is sized by the largest beam, not by
the batch.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np
import torch

from . import search
from .cluster import complete_clusterization
from .fdmt import CFdmtGpu


def fdmt_launches(plan: CFdmtGpu) -> int:
    """Kernels one FDMT launches: level 0 (or the fused head over the first
    ``depth`` levels), then one per merge pass (a plain level or a fused
    segment of several levels)."""
    return 1 + plan.info.hbm_passes


# An FDMT schedule: (fuse_depth, head_tile, seg_levels, seg_rows, seg_threads,
# seg_flags), the fields of bfs_fdmt_desc that fix the kernels a plan runs.
SCHEDULE_FIELDS = ("fuse_depth", "head_tile", "seg_levels", "seg_rows", "seg_threads", "seg_flags")


def tuned_schedule(shape: "BeamShape") -> tuple:
    """The autotuner's schedule for `shape` on the current device (its cached
    choice once a plan of that shape was created with fuse_depth -2)."""
    from . import _capi
    from .fdmt import autotune_desc
    d = _capi.FdmtDesc(fmin=shape.fmin, fmax=shape.fmax, nchan=shape.nchan, ncols=shape.nsamp,
                       max_dt=shape.max_dt, fuse_depth=_capi.BFS_FUSE_AUTOTUNE)
    t, _ = autotune_desc(d)
    return tuple(int(getattr(t, f)) for f in SCHEDULE_FIELDS)


def _schedule_kwargs(schedules, i: int, fuse_depth: int) -> dict:
    if schedules is None:
        return {"fuse_depth": fuse_depth}
    return dict(zip(SCHEDULE_FIELDS, (int(v) for v in schedules[i])))


@dataclass
class BeamShape:
    nchan: int
    nsamp: int
    fmin: float
    fmax: float
    max_dt: int


@dataclass
class BeamResult:
    n_candidates: int
    delegates: np.ndarray      # Cand records of the delegates, sorted by (mt, group)
    group_sizes: np.ndarray    # size of each delegate's own group


class SearchPipeline:
    def __init__(self, shapes: list[BeamShape], widths_mode: int = 0, param: int = 5,
                 thr: float = 7.0, metrics=(16, 8, 1 << 30), capacity: int = 1 << 26,
                 device: torch.device | str = "cuda:0", fuse_depth: int = -1, precision: int = 0,
                 schedules: list | None = None):
        """`schedules`: one SCHEDULE_FIELDS tuple per beam, used instead of
        `fuse_depth` (e.g. the schedules an earlier run's autotuner chose)."""
        self.device = torch.device(device)
        self.shapes = list(shapes)
        if schedules is not None and len(schedules) != len(self.shapes):
            raise ValueError("one schedule per beam")
        self.widths_mode, self.param, self.thr = widths_mode, param, float(thr)
        self.metrics = tuple(int(m) for m in metrics)
        self.plans = [CFdmtGpu(s.fmin, s.fmax, s.nchan, s.nsamp, s.max_dt, external_ws=True, precision=precision,
                               **_schedule_kwargs(schedules, i, fuse_depth))
                      for i, s in enumerate(self.shapes)]
        ws = max(p.workspace_size() for p in self.plans)
        self.workspace = torch.empty(ws, dtype=torch.uint8, device=self.device)
        plane = max(s.max_dt * s.nsamp for s in self.shapes)
        self.plane = torch.empty(plane, dtype=torch.float32, device=self.device)
        self.stats = torch.empty(2 * max(s.max_dt for s in self.shapes), dtype=torch.float32,
                                 device=self.device)
        self.cands = torch.empty((capacity, 4), dtype=torch.int32, device=self.device)
        self.launches = 0  # kernels of this library launched so far (CUB's not counted)

    @property
    def chan_samples(self) -> int:
        return sum(s.nchan * s.nsamp for s in self.shapes)

    def fdmt_alg_bytes(self) -> float:
        """Level-by-level bytes of the reference's algorithm, summed over beams."""
        return sum(p.alg_bytes for p in self.plans)

    def fdmt_sched_bytes(self) -> list[float]:
        """Per beam: the DRAM bytes its FDMT schedule cannot avoid (input read,
        every plane that reaches HBM written and read once, output written)."""
        return [p.sched_bytes for p in self.plans]

    def search_alg_bytes(self) -> float:
        """Row-statistics read + boxcar read of each DM-time plane."""
        return sum(2.0 * 4 * s.max_dt * s.nsamp for s in self.shapes)

    def run_beam(self, i: int, d_in: torch.Tensor, fdmt_events=None) -> BeamResult:
        s = self.shapes[i]
        plane = self.plane[: s.max_dt * s.nsamp].view(s.max_dt, s.nsamp)
        if fdmt_events is not None:
            fdmt_events[0].record()
        self.plans[i].process_image_ws(d_in, plane, False, self.workspace)
        if fdmt_events is not None:
            fdmt_events[1].record()
        stats = self.stats[: 2 * s.max_dt]
        search.launch_row_stats(plane, stats)
        cands, n = search.boxcar_gather(plane, self.thr, self.widths_mode, self.param,
                                        stats=stats, out=self.cands)
        # FDMT, row statistics, boxcar, canonical sort (keys + gather),
        # clustering (3 passes x keys/flags/scatter, offsets, delegates, delegate keys)
        self.launches += fdmt_launches(self.plans[i]) + 2 + (2 if n >= 2 else 0) + (12 if n else 0)
        if n == 0:
            return BeamResult(0, np.zeros(0, search.CAND_DTYPE), np.zeros(0, np.int64))
        cl = complete_clusterization(cands, self.metrics)
        return BeamResult(n, cl.delegate_records(), cl.delegate_group_sizes())

    def run(self, inputs: list[torch.Tensor], fdmt_timing: list | None = None) -> list[BeamResult]:
        out = []
        for i, x in enumerate(inputs):
            ev = None
            if fdmt_timing is not None:
                ev = (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
                fdmt_timing.append(ev)
            out.append(self.run_beam(i, x, ev))
        return out


class BatchedSearch:
    """All beams in one native batch (include/bfs.h bfs_batch_*): autotuned
    FDMT plans, every beam's FDMT + row statistics + boxcar captured in one
    CUDA graph, then one sort and one clustering for all beams."""

    def __init__(self, shapes: list[BeamShape], widths_mode: int = 0, param: int = 5,
                 thr: float = 7.0, metrics=(16, 8, 1 << 30), capacity: int = 1 << 26,
                 fuse_depth: int = -2, use_graph: bool = True, precision: int = 0,
                 schedules: list | None = None):
        """`schedules`: as for SearchPipeline."""
        import ctypes
        from . import _capi
        self._capi = _capi
        self.shapes = list(shapes)
        if schedules is not None and len(schedules) != len(self.shapes):
            raise ValueError("one schedule per beam")
        descs = (_capi.FdmtDesc * len(shapes))()
        for i, (d, sh) in enumerate(zip(descs, shapes)):
            d.fmin, d.fmax, d.nchan, d.ncols, d.max_dt = sh.fmin, sh.fmax, sh.nchan, sh.nsamp, sh.max_dt
            for f, v in _schedule_kwargs(schedules, i, fuse_depth).items():
                setattr(d, f, v)
            d.precision = precision
        bd = _capi.BatchDesc(nbeams=len(shapes), beams=descs, widths_mode=widths_mode, param=param,
                             thr=thr, capacity=capacity, use_graph=1 if use_graph else 0)
        for i, m in enumerate(metrics):
            bd.metrics[i] = int(m)
        self._descs = descs
        self._h = ctypes.c_void_p()
        _capi.call("bfs_batch_create", ctypes.byref(bd), ctypes.byref(self._h))
        self._ptrs = (ctypes.c_void_p * len(shapes))()

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                self._capi.lib().bfs_batch_destroy(h)
            except Exception:
                pass
            self._h = None

    @property
    def chan_samples(self) -> int:
        return sum(s.nchan * s.nsamp for s in self.shapes)

    def launches_per_run(self, n_candidates: int) -> int:
        """Kernels of this library one run launches (CUB's not counted): per
        beam the FDMT, row statistics and boxcar; then the tagged sort (keys
        + gather), clustering (3 passes x keys/flags/scatter, offsets,
        delegate lanes/tree, delegate keys) and the per-beam split (inverse
        permutation, delegate info, permutation, beam bounds)."""
        import ctypes
        k = 0
        for d in self._descs:
            info = self._capi.FdmtInfo()
            p = ctypes.c_void_p()
            dd = self._capi.FdmtDesc.from_buffer_copy(d)
            if dd.fuse_depth == self._capi.BFS_FUSE_AUTOTUNE:  # the batch's plans: cached choice
                from .fdmt import autotune_desc
                dd, _ = autotune_desc(dd)
            self._capi.call("bfs_fdmt_plan_create_host", ctypes.byref(dd), ctypes.byref(p))
            self._capi.call("bfs_fdmt_plan_info", p, ctypes.byref(info))
            self._capi.lib().bfs_fdmt_plan_destroy(p)
            k += 1 + info.hbm_passes + 2
        return k + ((2 + 12 + 4) if n_candidates else 0)

    def run(self, inputs: list[torch.Tensor], stream=None) -> list[BeamResult]:
        from ._tensors import dev_ptr, stream_handle
        for i, x in enumerate(inputs):
            self._ptrs[i] = dev_ptr(x, torch.float32, "input")
        self._capi.call("bfs_batch_run", self._h, self._ptrs, stream_handle(stream))
        return self._results()

    def submit(self, inputs: list[torch.Tensor], stream=None) -> None:
        """Start one run (FDMT + statistics + boxcar of every beam) without
        waiting; at most two runs in flight.  The tensors must stay unchanged
        until the run is collected."""
        from ._tensors import dev_ptr, stream_handle
        if len(inputs) != len(self.shapes):
            raise ValueError("one input per beam")
        ptrs = (ctypes.c_void_p * len(inputs))()
        for i, (x, sh) in enumerate(zip(inputs, self.shapes)):
            if x.numel() != sh.nchan * sh.nsamp:
                raise ValueError(f"beam {i}: input must hold {sh.nchan}x{sh.nsamp} floats")
            ptrs[i] = dev_ptr(x, torch.float32, f"inputs[{i}]")
        self._capi.call("bfs_batch_submit", self._h, ptrs, stream_handle(stream))

    def collect(self, stream=None) -> list[BeamResult]:
        """Finish the oldest submitted run (sort, clustering, delegates)."""
        from ._tensors import stream_handle
        self._capi.call("bfs_batch_collect", self._h, stream_handle(stream))
        return self._results()

    def run_host(self, host_inputs: list[torch.Tensor], dev_inputs: list[torch.Tensor],
                 stream=None) -> list[BeamResult]:
        """Search beams whose inputs are in pinned host memory: each beam is
        copied into its device buffer while the beams before it are searched."""
        import ctypes
        from ._tensors import dev_ptr, stream_handle
        n = len(self.shapes)
        hp = (ctypes.c_void_p * n)()
        dp = (ctypes.c_void_p * n)()
        for i, (h, d) in enumerate(zip(host_inputs, dev_inputs)):
            if h.device.type != "cpu" or not h.is_pinned() or not h.is_contiguous() or h.dtype != torch.float32:
                raise ValueError(f"beam {i}: host input must be a contiguous pinned float32 CPU tensor")
            if h.numel() != self.shapes[i].nchan * self.shapes[i].nsamp or d.numel() != h.numel():
                raise ValueError(f"beam {i}: input has the wrong size")
            hp[i] = h.data_ptr()
            dp[i] = dev_ptr(d, torch.float32, "device input")
        self._capi.call("bfs_batch_run_host", self._h, hp, dp, stream_handle(stream))
        return self._results()

    def _results(self) -> list[BeamResult]:
        import ctypes
        out = []
        for b in range(len(self.shapes)):
            nd, nc = ctypes.c_int(0), ctypes.c_uint32(0)
            self._capi.call("bfs_batch_beam_results", self._h, b, None, None, 0, ctypes.byref(nd),
                            ctypes.byref(nc))
            rec = np.zeros(nd.value, search.CAND_DTYPE)
            sizes = np.zeros(nd.value, np.int32)
            if nd.value:
                self._capi.call("bfs_batch_beam_results", self._h, b,
                                rec.ctypes.data_as(ctypes.c_void_p), sizes.ctypes.data_as(ctypes.c_void_p),
                                nd.value, ctypes.byref(nd), ctypes.byref(nc))
            out.append(BeamResult(int(nc.value), rec, sizes.astype(np.int64)))
        return out


def device_filterbank(nchan: int, nsamp: int, fmin: float, fmax: float, seed: int, pulses,
                      device, out: torch.Tensor | None = None, gain=None, rfi=()) -> torch.Tensor:
    """Seeded N(0,1) filterbank generated on the device with the same gain
    and pulse model as synth.filterbank (the noise stream differs from numpy's)."""
    from .synth import track
    g = torch.Generator(device=device).manual_seed(int(seed))
    x = out if out is not None else torch.empty((nchan, nsamp), dtype=torch.float32, device=device)
    x.normal_(generator=g)
    if gain is not None:
        x *= torch.as_tensor(np.asarray(gain, np.float32), device=device)[:, None]
    if len(rfi):
        t = torch.arange(nsamp, dtype=torch.float64, device=device)
        for c, f, ph, a in rfi:
            x[c] += (a * torch.sin(2 * np.pi * f * t + ph)).float()
    for p in pulses:
        tt = torch.from_numpy(track(nchan, fmin, fmax, p.t0, p.span)).to(device)
        cols = tt[:, None] + torch.arange(int(p.width), device=device)[None, :]
        rows = torch.arange(nchan, device=device)[:, None].expand_as(cols)
        ok = (cols >= 0) & (cols < nsamp)
        x.index_put_((rows[ok], cols[ok]), torch.tensor(float(p.amp), device=device), accumulate=True)
    return x
