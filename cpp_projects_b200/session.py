"""The GUPPI session driver: host mirror of the reference's
``CSession_guppi_gpu`` (MyVSLib_C++/CDMT/Session_guppi_gpu.cuh:9-39) and its
``CSessionB::launch`` (MyVSLib_C++/CDMT/SessionB.cpp:106-300).

``launch`` derives the chunk geometry from the first block's header and the
pulse length (``guppi.session_plan``: len_sft, overlap, chunk length, number
of coherent DMs, SessionB.cpp:144-206), creates one ``CChunk_gpu``, and runs
every chunk of every block through it: the streaming reader fills pinned
host buffers on a background thread and copies each chunk to the device on
the caller's stream (the current one by default); ``CChunk_gpu.process_raw`` turns the int8 chunk into
normalised FDMT planes (the reference's ``unpack_chunk`` + ``process``,
SessionB.cpp:255-267) and ``CChunk_gpu.search`` writes the delegate log.

As in the reference, every chunk writes the same log file (the chunk's
``candidates.log``; the output path is stored but not used), the images
handed back are those of the last chunk, and the return value is msamp.
Unlike the reference, the clusters of every chunk are kept in
``results`` as ``(block, chunk, Clusters | None)``.
"""
from __future__ import annotations

import torch

from . import guppi
from .chunk import CChunk_gpu


class CSession_guppi_gpu:
    def __init__(self, strGuppiPath, strOutPutPath, t_p: float, d_min: float, d_max: float,
                 sigma_bound: float, length_sum_wnd: int, nbin: int, nfft: int, device=None):
        self.m_strInpPath = str(strGuppiPath)
        self.m_strOutPutPath = str(strOutPutPath)
        self.m_pulse_length = float(t_p)
        self.m_d_min = float(d_min)
        self.m_d_max = float(d_max)
        self.m_sigma_bound = float(sigma_bound)
        self.m_length_sum_wnd = int(length_sum_wnd)
        self.m_nbin = int(nbin)
        self.m_nfft = int(nfft)
        self.device = torch.device(device) if device is not None else None
        self.results: list = []

    def plan(self, f: guppi.GuppiFile | None = None) -> dict:
        """The session's chunk geometry from the first block's header."""
        f = f if f is not None else guppi.GuppiFile(self.m_strInpPath)
        return guppi.session_plan(f.header(0), self.m_pulse_length, self.m_d_min, self.m_d_max,
                                  self.m_nbin, self.m_nfft)

    # createChunk (Session_guppi_gpu.cu:89-116): one chunk for the whole session
    def createChunk(self, p: dict, header: dict) -> CChunk_gpu:
        return CChunk_gpu(p["fmin"], p["fmax"], header["npol"], header["nchan"], p["len_sft"], 0, 0,
                          p["d_max"], p["d_min"], p["ncoherent"], self.m_sigma_bound,
                          self.m_length_sum_wnd, self.m_nbin, self.m_nfft, p["noverlap"], p["tsamp"])

    def open_reader(self, f: guppi.GuppiFile, p: dict, device, stream):
        return guppi.GuppiReader(f, p["len_chunk"], p["noverlap"], nbuffers=2, device=device, ndevice=2,
                                 stream=stream)

    def launch(self, pvecImg: list | None = None, logfile: str | None = "candidates.log",
               stream=None) -> int:
        """Runs the whole file; returns msamp.  pvecImg (a list) receives one
        max_dt x msamp image per coherent DM of the last chunk.  logfile=None
        skips the log."""
        device = self.device if self.device is not None else torch.device("cuda", torch.cuda.current_device())
        f = guppi.GuppiFile(self.m_strInpPath)
        h = f.header(0)
        p = self.plan(f)
        ch = self.createChunk(p, h)
        if len(ch.m_coh_dm_Vector) == 0:
            raise ValueError(f"DM range {p['d_min']}..{p['d_max']} holds no coherent DM")
        self.results = []
        planes = None
        with torch.cuda.stream(stream):      # None: the current stream
            spec = ch.complex_buffer(device)
            reader = self.open_reader(f, p, device, stream)
            try:
                for block, chunk, d_raw in reader:
                    ch.set_blockid(block)
                    ch.set_chunkid(chunk)
                    planes = ch.process_raw(d_raw, spec, stream=stream)
                    self.results.append((block, chunk, ch.search(planes, logfile, 0.0)))
            finally:
                reader.close()
            if pvecImg is not None and planes is not None:
                pvecImg[:] = list(planes.cpu().numpy())
        return ch.get_msamp()
