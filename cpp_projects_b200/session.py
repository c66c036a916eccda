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
Unlike the reference, every chunk's delegates are kept on the host in
``results`` as ``(block, chunk, delegates, group_sizes)``: the delegate Cand
records sorted by mt and the sizes of their groups in the log's pairing
(empty arrays when no candidate passed); the device buffers of a chunk are
released before the next one.
"""
from __future__ import annotations

import numpy as np
import torch

from . import guppi
from .chunk import CChunk_gpu
from .search import CAND_DTYPE


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
                    cl = ch.search(planes, logfile, 0.0)
                    if cl is None:
                        self.results.append((block, chunk, np.zeros(0, CAND_DTYPE), np.zeros(0, np.int64)))
                    else:
                        self.results.append((block, chunk, cl.delegate_records(), cl.group_sizes()))
            finally:
                reader.close()
            if pvecImg is not None and planes is not None:
                pvecImg[:] = list(planes.cpu().numpy())
        return ch.get_msamp()


def main(argv=None) -> int:
    """Command line in the manner of the reference's driver (the GUPPI GPU
    branch of my_hcdmt_inwork/main.cpp): a GUPPI file through the session,
    the delegate log and the last chunk's images (``images.npy``, one
    max_dt x msamp plane per coherent DM) written to the output folder.
    ``--plan-only`` prints the chunk geometry and exits (no GPU needed)."""
    import argparse
    import json
    from pathlib import Path

    ap = argparse.ArgumentParser(prog="python -m cpp_projects_b200.session")
    ap.add_argument("guppi")
    ap.add_argument("outdir")
    ap.add_argument("--t-p", type=float, required=True, help="pulse length, s")
    ap.add_argument("--d-min", type=float, default=0.0)
    ap.add_argument("--d-max", type=float, required=True)
    ap.add_argument("--sigma", type=float, default=6.0, help="detection threshold (S/N)")
    ap.add_argument("--length-sum-wnd", type=int, default=1)
    ap.add_argument("--nbin", type=int, default=1 << 20)
    ap.add_argument("--nfft", type=int, default=1)
    ap.add_argument("--plan-only", action="store_true")
    a = ap.parse_args(argv)
    s = CSession_guppi_gpu(a.guppi, a.outdir, a.t_p, a.d_min, a.d_max, a.sigma, a.length_sum_wnd,
                           a.nbin, a.nfft)
    p = s.plan()
    if a.plan_only:
        print(json.dumps(p))
        return 0
    out = Path(a.outdir)
    out.mkdir(parents=True, exist_ok=True)
    imgs: list = []
    msamp = s.launch(imgs, logfile=str(out / "candidates.log"))
    if imgs:
        np.save(out / "images.npy", np.stack(imgs))
    ndel = sum(len(d) for _, _, d, _ in s.results)
    print(json.dumps({**p, "msamp": msamp, "chunks": len(s.results), "delegates": ndel}))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
