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

from dataclasses import dataclass

import numpy as np
import torch

from . import search
from .cluster import complete_clusterization
from .fdmt import CFdmtGpu


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
    delegates: np.ndarray      # Cand records of the delegates, sorted by mt
    group_sizes: np.ndarray


class SearchPipeline:
    def __init__(self, shapes: list[BeamShape], widths_mode: int = 0, param: int = 5,
                 thr: float = 7.0, metrics=(16, 8, 1 << 30), capacity: int = 1 << 26,
                 device: torch.device | str = "cuda:0", fuse_depth: int = -1):
        self.device = torch.device(device)
        self.shapes = list(shapes)
        self.widths_mode, self.param, self.thr = widths_mode, param, float(thr)
        self.metrics = tuple(int(m) for m in metrics)
        self.plans = [CFdmtGpu(s.fmin, s.fmax, s.nchan, s.nsamp, s.max_dt, fuse_depth=fuse_depth,
                               external_ws=True) for s in self.shapes]
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
        return sum(p.alg_bytes for p in self.plans)

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
        # init + one per level, row statistics, boxcar, canonical sort (keys + gather),
        # clustering (3 passes x keys/flags/scatter, offsets, delegates, delegate keys)
        self.launches += 1 + self.plans[i].m_iNumIter + 2 + (2 if n >= 2 else 0) + (12 if n else 0)
        if n == 0:
            return BeamResult(0, np.zeros(0, search.CAND_DTYPE), np.zeros(0, np.int64))
        cl = complete_clusterization(cands, self.metrics)
        return BeamResult(n, cl.delegate_records(), cl.group_sizes())

    def run(self, inputs: list[torch.Tensor], fdmt_timing: list | None = None) -> list[BeamResult]:
        out = []
        for i, x in enumerate(inputs):
            ev = None
            if fdmt_timing is not None:
                ev = (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
                fdmt_timing.append(ev)
            out.append(self.run_beam(i, x, ev))
        return out


def device_filterbank(nchan: int, nsamp: int, fmin: float, fmax: float, seed: int, pulses,
                      device, out: torch.Tensor | None = None) -> torch.Tensor:
    """Seeded N(0,1) filterbank generated on the device with the same pulse
    model as synth.filterbank (the noise stream differs from numpy's)."""
    from .synth import track
    g = torch.Generator(device=device).manual_seed(int(seed))
    x = out if out is not None else torch.empty((nchan, nsamp), dtype=torch.float32, device=device)
    x.normal_(generator=g)
    for p in pulses:
        tt = torch.from_numpy(track(nchan, fmin, fmax, p.t0, p.span)).to(device)
        cols = tt[:, None] + torch.arange(int(p.width), device=device)[None, :]
        rows = torch.arange(nchan, device=device)[:, None].expand_as(cols)
        ok = (cols >= 0) & (cols < nsamp)
        x.index_put_((rows[ok], cols[ok]), torch.tensor(float(p.amp), device=device), accumulate=True)
    return x
