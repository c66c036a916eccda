"""Coherent-dedispersion chunk stage (host mirror of the reference's
``CChunk_gpu`` / ``CChunk_fly_gpu`` and ``CSession_guppi_gpu::unpack_chunk``;
MyVSLib_C++/CDMT/Chunk_gpu.cu:134-460, Chunk_fly_gpu.cu:94-163,
Session_guppi_gpu.cu:53-60).

``CChunk_gpu(Fmin, Fmax, npol, nchan, len_sft, Block_id, Chunk_id, d_max,
d_min, ncoherent, sigma_bound, length_sum_wnd, nbin, nfft, noverlap, tsamp)``
keeps the reference constructor's argument list; ``max_dt`` (FDMT output
rows, the reference uses ``len_sft``) is an extra keyword.  ``process`` takes
the unpacked complex chunk (overwritten by the forward FFT, as in the
reference) and returns the stacked normalised DM-time planes.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _capi
from ._tensors import dev_ptr, stream_handle


def coherent_dms(d_min: float, d_max: float, ncoherent: int) -> np.ndarray:
    """The coherent-DM grid of CChunkB's constructor (ChunkB.cpp:171-176)."""
    fn = _capi.lib().bfs_chunk_coherent_dms
    n = fn(ctypes.c_double(d_min), ctypes.c_double(d_max), int(ncoherent), None, 0)
    buf = np.zeros(max(n, 0), np.float64)
    if n > 0:
        fn(ctypes.c_double(d_min), ctypes.c_double(d_max), int(ncoherent), buf.ctypes.data_as(ctypes.c_void_p),
           buf.size)
    return buf


class CChunk_gpu:
    def __init__(self, Fmin, Fmax, npol, nchan, len_sft, Block_id, Chunk_id, d_max, d_min,
                 ncoherent, sigma_bound, length_sum_wnd, nbin, nfft, noverlap, tsamp,
                 max_dt: int = 0, dms=None):
        self.m_Fmin, self.m_Fmax = float(Fmin), float(Fmax)
        self.m_npol, self.m_nchan, self.m_len_sft = int(npol), int(nchan), int(len_sft)
        self.m_Block_id, self.m_Chunk_id = int(Block_id), int(Chunk_id)
        self.m_sigma_bound, self.m_length_sum_wnd = float(sigma_bound), int(length_sum_wnd)
        self.m_nbin, self.m_nfft, self.m_noverlap = int(nbin), int(nfft), int(noverlap)
        self.m_tsamp = float(tsamp)
        self.m_coh_dm_Vector = (np.asarray(dms, np.float64) if dms is not None
                                else coherent_dms(d_min, d_max, ncoherent))
        desc = _capi.ChunkDesc(fmin=self.m_Fmin, fmax=self.m_Fmax, npol=self.m_npol,
                               nchan=self.m_nchan, len_sft=self.m_len_sft, nbin=self.m_nbin,
                               nfft=self.m_nfft, noverlap=self.m_noverlap, tsamp=self.m_tsamp,
                               max_dt=int(max_dt))
        self._h = ctypes.c_void_p()
        _capi.call("bfs_chunk_create", ctypes.byref(desc), ctypes.byref(self._h))
        info = np.zeros(8, np.int64)
        _capi.call("bfs_chunk_info", self._h, info.ctypes.data_as(ctypes.c_void_p), 8)
        (self.mbin, self.noverlap_per_channel, self.mbin_adjusted, self.msamp, self.rows,
         self.len_chunk, self.cplx_len, self.max_dt) = (int(v) for v in info)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                _capi.lib().bfs_chunk_destroy(h)
            except Exception:
                pass
            self._h = None

    # geometry accessors named as in CChunkB (ChunkB.h:77-98)
    def get_mbin(self): return self.mbin
    def get_noverlap_per_channel(self): return self.noverlap_per_channel
    def get_mbin_adjusted(self): return self.mbin_adjusted
    def get_msamp(self): return self.msamp
    def set_blockid(self, nC): self.m_Block_id = int(nC)
    def set_chunkid(self, nC): self.m_Chunk_id = int(nC)

    def complex_buffer(self, device) -> torch.Tensor:
        return torch.empty((self.cplx_len, 2), dtype=torch.float32, device=device)

    # --- stages -------------------------------------------------------------
    def unpack(self, d_raw: torch.Tensor, d_cplx: torch.Tensor, stream=None) -> None:
        """GUPPI int8 [nchan][len_chunk][npol] -> complex [npol/2][nfft][nchan][nbin]."""
        if d_raw.numel() != self.m_nchan * self.len_chunk * self.m_npol:
            raise ValueError("raw chunk has the wrong size")
        _capi.call("bfs_chunk_unpack", self._h, dev_ptr(d_raw, torch.int8, "d_raw"),
                   dev_ptr(d_cplx, torch.float32, "d_cplx"), stream_handle(stream))

    def forward_fft(self, d_cplx, stream=None):
        _capi.call("bfs_chunk_forward_fft", self._h, dev_ptr(d_cplx, torch.float32), stream_handle(stream))

    def unpack_fft(self, d_raw: torch.Tensor, d_spec: torch.Tensor, stream=None) -> None:
        """unpack + forward FFT in one step: the spectra of every segment of the
        GUPPI int8 chunk (for nbin = 2^20 a fused four-step transform that reads
        the int8 samples directly; other sizes unpack and call cuFFT)."""
        if d_raw.numel() != self.m_nchan * self.len_chunk * self.m_npol:
            raise ValueError("raw chunk has the wrong size")
        _capi.call("bfs_chunk_unpack_fft", self._h, dev_ptr(d_raw, torch.int8, "d_raw"),
                   dev_ptr(d_spec, torch.float32, "d_spec"), stream_handle(stream))

    def voltages(self, d_spec, dm: float, d_volt, stream=None):
        _capi.call("bfs_chunk_voltages", self._h, dev_ptr(d_spec, torch.float32), ctypes.c_double(dm),
                   dev_ptr(d_volt, torch.float32), stream_handle(stream))

    def detect(self, d_volt, dm: float, d_plane, stream=None):
        _capi.call("bfs_chunk_detect", self._h, dev_ptr(d_volt, torch.float32), ctypes.c_double(dm),
                   dev_ptr(d_plane, torch.float32), stream_handle(stream))

    def detect_spectrum(self, d_spec, dm: float, d_plane, stream=None):
        """voltages + detect in one call (the voltages are not stored where
        the own sub-band transform applies)."""
        _capi.call("bfs_chunk_detect_spectrum", self._h, dev_ptr(d_spec, torch.float32), ctypes.c_double(dm),
                   dev_ptr(d_plane, torch.float32), stream_handle(stream))

    def process(self, pcmparrRawSignalCur: torch.Tensor, stream=None) -> torch.Tensor:
        """CChunkB::process: returns (ndm, max_dt, msamp) normalised FDMT planes."""
        dms = np.ascontiguousarray(self.m_coh_dm_Vector, np.float64)
        out = torch.empty((len(dms), self.max_dt, self.msamp), dtype=torch.float32,
                          device=pcmparrRawSignalCur.device)
        _capi.call("bfs_chunk_process", self._h, dev_ptr(pcmparrRawSignalCur, torch.float32),
                   dms.ctypes.data_as(ctypes.c_void_p), len(dms), dev_ptr(out), stream_handle(stream))
        return out

    def process_spectrum(self, d_spec: torch.Tensor, stream=None) -> torch.Tensor:
        """The per-DM part of process on spectra from unpack_fft / forward_fft
        (d_spec is not modified): (ndm, max_dt, msamp) planes."""
        dms = np.ascontiguousarray(self.m_coh_dm_Vector, np.float64)
        out = torch.empty((len(dms), self.max_dt, self.msamp), dtype=torch.float32, device=d_spec.device)
        _capi.call("bfs_chunk_process_spectrum", self._h, dev_ptr(d_spec, torch.float32),
                   dms.ctypes.data_as(ctypes.c_void_p), len(dms), dev_ptr(out), stream_handle(stream))
        return out

    def process_raw(self, d_raw: torch.Tensor, d_spec: torch.Tensor, stream=None) -> torch.Tensor:
        """unpack_fft + the per-DM part of process: (ndm, max_dt, msamp) planes
        straight from the int8 chunk; d_spec receives the spectra."""
        if d_raw.numel() != self.m_nchan * self.len_chunk * self.m_npol:
            raise ValueError("raw chunk has the wrong size")
        dms = np.ascontiguousarray(self.m_coh_dm_Vector, np.float64)
        out = torch.empty((len(dms), self.max_dt, self.msamp), dtype=torch.float32, device=d_raw.device)
        _capi.call("bfs_chunk_process_raw", self._h, dev_ptr(d_raw, torch.int8, "d_raw"),
                   dev_ptr(d_spec, torch.float32, "d_spec"), dms.ctypes.data_as(ctypes.c_void_p), len(dms),
                   dev_ptr(out), stream_handle(stream))
        return out

    def search(self, planes: torch.Tensor, logfile: str | None = "candidates.log",
               t_chunkBegin: float = 0.0):
        """The candidate step at the end of the reference's process
        (Chunk_gpu.cu:403-425): every width 1..4, threshold sigma_bound,
        metrics {2, 1, 2}, delegate log with delt_bin = tsamp * len_sft."""
        from .cluster import clusterization_main
        rows = planes.shape[0] * planes.shape[1]
        return clusterization_main(planes.reshape(rows, -1), rows, planes.shape[2],
                                   self.m_sigma_bound, 4, (2, 1, 2), logfile or "candidates.log",
                                   self.m_tsamp * self.m_len_sft, t_chunkBegin,
                                   bwrite=logfile is not None)
