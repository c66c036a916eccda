"""GUPPI RAW input (host mirror of the reference's CSession_guppi file
handling, MyVSLib_C++/CDMT/Session_guppi.cpp and TelescopeHeader.cpp) over
the C ABI: block headers, per-channel strided chunk reads with overlap, and
a streaming reader that overlaps file reads, host-to-device copies and the
caller's kernels (pinned double buffers, a background reader thread).

Chunks come back as ``[nchan][len_chunk][npol]`` int8 in ascending
frequency, the layout ``CChunk_gpu.unpack`` takes.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _capi
from ._tensors import dev_ptr, stream_handle

TELESCOPES = {0: "GBT", 1: "PARKES"}


def _header_dict(h: _capi.GuppiHeader) -> dict:
    return {k: getattr(h, k) for k, _ in h._fields_ if k != "reserved"}


def parse_header(text: bytes) -> dict:
    """Parse one header (bytes of the header and whatever follows it)."""
    h = _capi.GuppiHeader()
    buf = ctypes.create_string_buffer(text, len(text))
    _capi.call("bfs_guppi_parse_header", buf, len(text), ctypes.byref(h))
    return _header_dict(h)


def session_plan(header: dict, t_p: float, d_min: float, d_max: float, nbin: int, nfft: int) -> dict:
    """Chunk geometry of a session (CSessionB::launch, SessionB.cpp:144-160,
    184-206, 384-401) from a block header as ``GuppiFile.header`` or
    ``parse_header`` return it: len_sft, noverlap, len_chunk, ncoherent,
    optimal_overlap, fmin, fmax, tsamp, d_min, d_max."""
    h = _capi.GuppiHeader()
    for k, _ in h._fields_:
        if k != "reserved":
            setattr(h, k, header[k])
    out = _capi.GuppiSession()
    _capi.call("bfs_guppi_session_plan", ctypes.byref(h), float(t_p), float(d_min), float(d_max),
               int(nbin), int(nfft), ctypes.byref(out))
    return {k: getattr(out, k) for k, _ in out._fields_ if k != "reserved"}


class GuppiFile:
    def __init__(self, path: str):
        self.path = str(path)
        self._h = ctypes.c_void_p()
        _capi.call("bfs_guppi_open", self.path.encode(), ctypes.byref(self._h))
        n = ctypes.c_int(0)
        _capi.call("bfs_guppi_blocks", self._h, ctypes.byref(n))
        self.nblocks = int(n.value)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                _capi.lib().bfs_guppi_close(h)
            except Exception:
                pass
            self._h = None

    def header(self, block: int = 0) -> dict:
        h = _capi.GuppiHeader()
        _capi.call("bfs_guppi_block_header", self._h, int(block), ctypes.byref(h))
        return _header_dict(h)

    def chunk_count(self, block: int, len_chunk: int, noverlap: int) -> int:
        n = ctypes.c_int64(0)
        _capi.call("bfs_guppi_chunk_count", self._h, int(block), int(len_chunk), int(noverlap), ctypes.byref(n))
        return int(n.value)

    def read_chunk(self, block: int, chunk: int, len_chunk: int, noverlap: int) -> np.ndarray:
        h = self.header(block)
        out = np.empty((h["nchan"], len_chunk, h["npol"]), np.int8)
        _capi.call("bfs_guppi_read_chunk", self._h, int(block), int(chunk), int(len_chunk), int(noverlap),
                   out.ctypes.data_as(ctypes.c_void_p), out.nbytes)
        return out


class GuppiReader:
    """Iterates (block, chunk, data) over every chunk of every block; with
    ``device`` the data is a CUDA int8 tensor filled by an asynchronous copy
    on ``stream`` (one of ``ndevice`` rotating device buffers), else a numpy
    view of the host buffer (valid until the next step)."""

    def __init__(self, f: GuppiFile, len_chunk: int, noverlap: int, nbuffers: int = 2, device=None,
                 ndevice: int = 2, stream=None):
        self.f = f
        h = f.header(0)
        self.shape = (h["nchan"], int(len_chunk), h["npol"])
        self.device = torch.device(device) if device is not None else None
        self.stream = stream
        self._r = ctypes.c_void_p()
        _capi.call("bfs_guppi_reader_create", f._h, int(len_chunk), int(noverlap), int(nbuffers),
                   1 if self.device is not None else 0, ctypes.byref(self._r))
        self._dev = ([torch.empty(self.shape, dtype=torch.int8, device=self.device) for _ in range(ndevice)]
                     if self.device is not None else [])
        self._k = 0

    def close(self):
        r = getattr(self, "_r", None)
        if r is not None and r.value:
            _capi.lib().bfs_guppi_reader_destroy(r)
            self._r = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __iter__(self):
        return self

    def __next__(self):
        block, chunk = ctypes.c_int(0), ctypes.c_int64(0)
        host = ctypes.c_void_p()
        dst = None
        if self._dev:
            dst = self._dev[self._k % len(self._dev)]
            self._k += 1
        _capi.call("bfs_guppi_reader_next", self._r, dev_ptr(dst, torch.int8) if dst is not None else None,
                   stream_handle(self.stream) if dst is not None else None, ctypes.byref(host),
                   ctypes.byref(block), ctypes.byref(chunk))
        if block.value < 0:
            raise StopIteration
        if dst is not None:
            return int(block.value), int(chunk.value), dst
        n = int(np.prod(self.shape))
        arr = np.ctypeslib.as_array(ctypes.cast(host, ctypes.POINTER(ctypes.c_int8)), shape=(n,))
        return int(block.value), int(chunk.value), arr.reshape(self.shape)
