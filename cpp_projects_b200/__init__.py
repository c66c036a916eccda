"""B200-native FRB / pulsar search core.

Host-side mirror (Python) of the reference's C++ entry points on the search
hot path, calling hand-written sm_100a CUDA through the C ABI in
``include/bfs.h``:

* :class:`CFdmtGpu` — FDMT (``CFdmtGpu::process_image``)
* :class:`FDMTGPU` — the reference's second FDMT variant (``FDMT::execute``,
  Pravir plan)
* :mod:`.search` — boxcar detection (``clusterization::gather_candidates_*``),
  per-row normalisation
* :mod:`.cluster` — ``clusterization::complete_clusterization`` /
  ``clusterization_main``, ``select_delegates``
* :mod:`.preproc` — ``statistical_preprocessing::calc_fdmt_inputs``,
  ``fdmt_normalization``
* :mod:`.chunk` — ``CChunk_gpu`` coherent-dedispersion stage
* :mod:`.guppi` — GUPPI RAW headers, chunk reads, streaming reader
* :mod:`.session` — ``CSession_guppi_gpu`` (``CSessionB::launch``): a GUPPI
  file through the chunk stage and the candidate search
* :mod:`.pipeline` — per-beam and batched (CUDA-graph) search
* :mod:`.autograd` — differentiable FDMT + boxcar S/N
"""
from ._capi import BfsError, lib  # noqa: F401
from .fdmt import FDMTGPU, CFdmtGpu  # noqa: F401

__all__ = ["CFdmtGpu", "FDMTGPU", "BfsError", "lib"]
