"""Candidate output formats (host mirror of the reference's COutChunkHeader
and CFragment, MyVSLib_C++/OutChunkHeader.cpp:89-227, Fragment.h:3-28,
CDMT/ChunkB.cpp:255-275).

* :class:`COutChunkHeader` — one detection per chunk; :func:`write_report`
  writes the reference's text report byte for byte, and
  :func:`read_outputlogfile_line` parses one line back as the reference does.
* :class:`CFragment` / :func:`cut_quadratic_fragment` — the square cut-out of
  a DM-time plane around a detection (cut on the GPU), saved as ``.npy``
  with a ``.json`` sidecar for vetting.
"""
from __future__ import annotations

import ctypes
import json
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np
import torch

from . import _capi
from ._tensors import dev_ptr, stream_handle


@dataclass
class COutChunkHeader:
    m_nrows: int = 0
    m_ncols: int = 0
    m_nSucessRow: int = 0
    m_nSucessCol: int = 0
    m_wnd_width: int = 0
    m_SNR: float = 0.0
    m_coherentDedisp: float = 0.0
    m_numBlock: int = 0
    m_numChunk: int = 0

    def createOutStr(self) -> str:
        """The reference's line (block and chunk counted from 1; float32 values)."""
        return ("Block=  %d,Chunk=  %d,Rows=  %d,Cols=  %d, SucRow=  %d,SucCol=  %d, SNR=  %.4f, "
                "CohDisp=  %.4f, windWidth=  %d" % (
                    self.m_numBlock + 1, self.m_numChunk + 1, self.m_nrows, self.m_ncols, self.m_nSucessRow,
                    self.m_nSucessCol, float(np.float32(self.m_SNR)), float(np.float32(self.m_coherentDedisp)),
                    self.m_wnd_width))


def write_report(path, headers: list[COutChunkHeader], pulse_length: float) -> None:
    """COutChunkHeader::writeReport: one line per header plus the pulse length."""
    with open(path, "wb") as f:
        for h in headers:
            f.write((h.createOutStr() + ", Length of pulse= %.10e\n" % float(np.float32(pulse_length))).encode())


def _num(line: str, key: str, off: int, conv):
    p = line.find(key)
    if p < 0:
        raise ValueError(f"{key} missing")
    s = line[p + off:]
    # atoi / atof on the text after the key: the longest numeric prefix
    j = 0
    while j < len(s) and s[j] in " \t":
        j += 1
    k = j
    while k < len(s) and (s[k].isdigit() or s[k] in "+-.eE"):
        k += 1
    txt = s[j:k]
    while txt:
        try:
            return conv(txt)
        except ValueError:
            txt = txt[:-1]
    return conv(0)


def read_outputlogfile_line(path, num_line: int) -> dict | None:
    """COutChunkHeader::read_outputlogfile_line: fields of line `num_line`
    (block and chunk as written, i.e. counted from 1); None if a key is
    missing."""
    lines = Path(path).read_text().splitlines(keepends=True)
    if num_line >= len(lines):
        return None
    line = lines[num_line]
    try:
        return {"numBlock": _num(line, "Block=", 8, int), "numChunk": _num(line, "Chunk=", 8, int),
                "nrows": _num(line, "Rows=", 7, int), "ncols": _num(line, "Cols=", 7, int),
                "sucRow": _num(line, "SucRow=", 9, int), "sucCol": _num(line, "SucCol=", 9, int),
                "snr": float(np.float32(_num(line, "SNR=", 6, float))),
                "cohDisp": float(np.float32(_num(line, "CohDisp=", 10, float))),
                "width": _num(line, "windWidth=", 12, int)}
    except ValueError:
        return None


@dataclass
class CFragment:
    m_nBeginRow: int = 0
    m_nBeginCol: int = 0
    m_dim: int = 0
    m_vctData: np.ndarray = field(default_factory=lambda: np.zeros(1, np.float32))
    m_width: int = 0
    m_snr: float = 0.0
    m_cohDisp: float = 0.0

    def save_npy(self, path) -> Path:
        """The fragment as a dim x dim float32 .npy plus a .json sidecar."""
        path = Path(path).with_suffix(".npy")
        np.save(path, self.m_vctData.reshape(self.m_dim, self.m_dim))
        path.with_suffix(".json").write_text(json.dumps({
            "begin_row": self.m_nBeginRow, "begin_col": self.m_nBeginCol, "dim": self.m_dim,
            "width": self.m_width, "snr": self.m_snr, "coherent_dm": self.m_cohDisp}))
        return path


def cut_quadratic_fragment(plane: torch.Tensor, target_row: int, target_col: int, width: int = 0,
                           snr: float = 0.0, coh_dm: float = 0.0, stream=None) -> CFragment:
    """The square fragment of a (rows x cols) CUDA plane holding the target
    (CChunkB::cutQuadraticFragment's rule), cut on the device."""
    rows, cols = plane.shape
    rb, cb, d = ctypes.c_int(0), ctypes.c_int(0), ctypes.c_int(0)
    _capi.call("bfs_cut_fragment", None, rows, cols, int(target_row), int(target_col), None,
               ctypes.byref(rb), ctypes.byref(cb), ctypes.byref(d), None)
    out = torch.empty((d.value, d.value), dtype=torch.float32, device=plane.device)
    _capi.call("bfs_cut_fragment", dev_ptr(plane, torch.float32, "plane"), rows, cols, int(target_row),
               int(target_col), dev_ptr(out), ctypes.byref(rb), ctypes.byref(cb), ctypes.byref(d),
               stream_handle(stream))
    return CFragment(rb.value, cb.value, d.value, out.cpu().numpy().reshape(-1), int(width), float(snr),
                     float(coh_dm))
