"""FDMT host interface mirroring the reference's ``CFdmtGpu`` class.

Reference: ``CFdmtGpu(Fmin, Fmax, nchan, cols, imaxDt)`` and
``process_image(d_in, d_out, b_ones)`` (MyVSLib_C++/FDMT/FdmtGpu.cuh:12-53).
Inputs and outputs are caller-owned device buffers (here: CUDA torch tensors,
float32, contiguous): ``d_in`` is ``nchan x cols`` with row 0 the lowest
frequency channel, ``d_out`` is ``imaxDt x cols``.  The work is enqueued on
the current torch stream.  Unlike the reference (which prints to stderr and
returns), errors raise :class:`BfsError`.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _capi
from ._tensors import dev_ptr, stream_handle


def autotune(Fmin: float, Fmax: float, nchan: int, cols: int, imaxDt: int) -> tuple[int, int, float]:
    """Time the fused-head depths, tile widths and merge-segment lengths for
    this shape on the current device (cached per shape): returns
    (fuse_depth, head_tile, ms)."""
    desc = _capi.FdmtDesc(fmin=float(Fmin), fmax=float(Fmax), nchan=int(nchan), ncols=int(cols),
                          max_dt=int(imaxDt))
    depth, tile, ms = ctypes.c_int(0), ctypes.c_int(0), ctypes.c_float(0)
    _capi.call("bfs_fdmt_autotune", ctypes.byref(desc), ctypes.byref(depth), ctypes.byref(tile),
               ctypes.byref(ms))
    return depth.value, tile.value, ms.value


def autotune_desc(desc: "_capi.FdmtDesc") -> tuple["_capi.FdmtDesc", float]:
    """The tuned description (fuse_depth, head_tile, seg_levels, seg_rows
    filled in) of `desc` on the current device, and its time in ms."""
    out = _capi.FdmtDesc()
    ms = ctypes.c_float(0)
    _capi.call("bfs_fdmt_autotune_desc", ctypes.byref(desc), ctypes.byref(out), ctypes.byref(ms))
    return out, ms.value


class CFdmtGpu:
    def __init__(self, Fmin: float, Fmax: float, nchan: int, cols: int, imaxDt: int,
                 fuse_depth: int = -1, external_ws: bool = False, head_tile: int = 0,
                 precision: int = 0, seg_levels: int = 0, seg_rows: int = 0, seg_threads: int = 0,
                 seg_flags: int = 0):
        self.m_Fmin = float(Fmin)
        self.m_Fmax = float(Fmax)
        self.m_nchan = int(nchan)
        self.m_cols = int(cols)
        self.m_imaxDt = int(imaxDt)
        self.precision = int(precision)
        desc = _capi.FdmtDesc(fmin=self.m_Fmin, fmax=self.m_Fmax, nchan=self.m_nchan,
                              ncols=self.m_cols, max_dt=self.m_imaxDt, plan_kind=0,
                              precision=int(precision), fuse_depth=int(fuse_depth),
                              flags=_capi.BFS_FDMT_EXTERNAL_WS if external_ws else 0,
                              head_tile=int(head_tile), seg_levels=int(seg_levels),
                              seg_rows=int(seg_rows), seg_threads=int(seg_threads),
                              seg_flags=int(seg_flags))
        self._plan = ctypes.c_void_p()
        _capi.call("bfs_fdmt_plan_create", ctypes.byref(desc), ctypes.byref(self._plan))
        info = _capi.FdmtInfo()
        _capi.call("bfs_fdmt_plan_info", self._plan, ctypes.byref(info))
        self.info = info
        self.m_iNumIter = info.niter

    def __del__(self):
        p = getattr(self, "_plan", None)
        if p is not None and p.value:
            try:
                _capi.lib().bfs_fdmt_plan_destroy(p)
            except Exception:
                pass
            self._plan = None

    # --- reference API ---------------------------------------------------
    def process_image(self, d_in: torch.Tensor | None, d_out: torch.Tensor, b_ones: bool = False,
                      stream: torch.cuda.Stream | None = None) -> None:
        if d_out.numel() != self.m_imaxDt * self.m_cols:
            raise ValueError(f"d_out must hold {self.m_imaxDt}x{self.m_cols} floats")
        pin = None
        if not b_ones:
            if d_in is None or d_in.numel() != self.m_nchan * self.m_cols:
                raise ValueError(f"d_in must hold {self.m_nchan}x{self.m_cols} floats")
            pin = dev_ptr(d_in, torch.float32, "d_in")
        _capi.call("bfs_fdmt_execute", self._plan, pin, dev_ptr(d_out, torch.float32, "d_out"),
                   1 if b_ones else 0, stream_handle(stream))

    def workspace_size(self) -> int:
        n = ctypes.c_size_t(0)
        _capi.call("bfs_fdmt_workspace_size", self._plan, ctypes.byref(n))
        return int(n.value)

    def process_image_ws(self, d_in: torch.Tensor | None, d_out: torch.Tensor, b_ones: bool,
                         workspace: torch.Tensor, stream: torch.cuda.Stream | None = None) -> None:
        """process_image with caller-provided scratch (a uint8 CUDA tensor of at
        least workspace_size() bytes, 256-byte aligned)."""
        pin = None if b_ones else dev_ptr(d_in, torch.float32, "d_in")
        _capi.call("bfs_fdmt_execute_ws", self._plan, pin, dev_ptr(d_out, torch.float32, "d_out"),
                   1 if b_ones else 0, dev_ptr(workspace, None, "workspace"),
                   ctypes.c_size_t(workspace.numel() * workspace.element_size()),
                   stream_handle(stream))

    # --- adjoint -------------------------------------------------------------
    def adjoint(self, d_grad_out: torch.Tensor, d_grad_in: torch.Tensor | None = None,
                stream: torch.cuda.Stream | None = None) -> torch.Tensor:
        """d_grad_in (nchan x cols) = F^T d_grad_out (imaxDt x cols)."""
        if d_grad_out.numel() != self.m_imaxDt * self.m_cols:
            raise ValueError(f"d_grad_out must hold {self.m_imaxDt}x{self.m_cols} floats")
        if d_grad_in is None:
            d_grad_in = torch.empty((self.m_nchan, self.m_cols), dtype=torch.float32,
                                    device=d_grad_out.device)
        if d_grad_in.numel() != self.m_nchan * self.m_cols:
            raise ValueError(f"d_grad_in must hold {self.m_nchan}x{self.m_cols} floats")
        _capi.call("bfs_fdmt_adjoint", self._plan, dev_ptr(d_grad_out, torch.float32, "d_grad_out"),
                   dev_ptr(d_grad_in, torch.float32, "d_grad_in"), stream_handle(stream))
        return d_grad_in

    def adjoint_workspace_size(self) -> int:
        n = ctypes.c_size_t(0)
        _capi.call("bfs_fdmt_adjoint_workspace_size", self._plan, ctypes.byref(n))
        return int(n.value)

    def adjoint_ws(self, d_grad_out: torch.Tensor, d_grad_in: torch.Tensor, workspace: torch.Tensor,
                   stream: torch.cuda.Stream | None = None) -> None:
        _capi.call("bfs_fdmt_adjoint_ws", self._plan, dev_ptr(d_grad_out, torch.float32, "d_grad_out"),
                   dev_ptr(d_grad_in, torch.float32, "d_grad_in"), dev_ptr(workspace, None, "workspace"),
                   ctypes.c_size_t(workspace.numel() * workspace.element_size()), stream_handle(stream))

    # --- plan introspection ------------------------------------------------
    def passes(self) -> list[list[int]]:
        """[l0, l1, r0c] of every merge pass after the head: a plain level
        (l1 = l0 + 1) or a fused segment of levels l0+1..l1; r0c > 0 marks an
        input segment (it reads the channels and forms level 0 itself)."""
        n = ctypes.c_int(0)
        _capi.call("bfs_fdmt_plan_passes", self._plan, ctypes.byref(n), None, 0)
        p = np.zeros(max(1, n.value) * 13, np.int32)
        _capi.call("bfs_fdmt_plan_passes", self._plan, ctypes.byref(n), p.ctypes.data_as(ctypes.c_void_p), p.size)
        return [[int(p[13 * i]), int(p[13 * i + 1]), int(p[13 * i + 12])] for i in range(n.value)]

    @property
    def sched_bytes(self) -> float:
        """DRAM bytes of one call that this plan's schedule cannot avoid."""
        return float(self.info.sched_bytes)

    def rows_per_level(self) -> np.ndarray:
        rows = np.zeros(self.m_iNumIter + 1, np.int32)
        _capi.call("bfs_fdmt_plan_rows", self._plan, rows.ctypes.data_as(ctypes.c_void_p),
                   rows.size)
        return rows

    def tables(self, level: int):
        n = int(self.rows_per_level()[level])
        a = np.zeros(n, np.int32); b = np.zeros(n, np.int32); s = np.zeros(n, np.int32)
        P = ctypes.c_void_p
        _capi.call("bfs_fdmt_plan_tables", self._plan, level, a.ctypes.data_as(P),
                   b.ctypes.data_as(P), s.ctypes.data_as(P), n)
        return a, b, s

    @property
    def alg_bytes(self) -> float:
        """Level-by-level algorithmic bytes of one call (input read, level-0
        plane write, each level's tail + head read and output write)."""
        return float(self.info.alg_bytes)

    def __call__(self, d_in: torch.Tensor, b_ones: bool = False) -> torch.Tensor:
        out = torch.empty((self.m_imaxDt, self.m_cols), dtype=torch.float32, device=d_in.device)
        self.process_image(d_in, out, b_ones)
        return out


# Dispersion constant of the reference's DM grid (TEMPO2 / Manchester & Taylor
# 1972, L/FDMT_PRAVIR/fdmtUtils.hpp:7-11), MHz^2 pc^-1 cm^3 s.
K_DISP_MT = np.float32(4.1493774e3)


class FDMTGPU:
    """The reference's second FDMT variant (``FDMT`` / ``FDMTGPU``,
    MyVSLib_C++/FDMT_PRAVIR/fdmt_base.hpp:37-84, fdmt_gpu.cuh) on the
    library's kernels: delay grids ``dt_min .. dt_max`` step ``dt_step``,
    window-mean level 0, rounded mid-band mappings (``BFS_PLAN_PRAVIR``).
    ``execute`` takes device tensors and raises ``ValueError`` on a size
    mismatch (the reference throws ``std::invalid_argument``)."""

    def __init__(self, f_min: float, f_max: float, nchans: int, nsamps: int, tsamp: float,
                 dt_max: int, dt_step: int = 1, dt_min: int = 0, external_ws: bool = False):
        self.m_f_min, self.m_f_max = float(f_min), float(f_max)
        self.m_nchans, self.m_nsamps = int(nchans), int(nsamps)
        self.m_tsamp = float(tsamp)
        self.m_dt_max, self.m_dt_step, self.m_dt_min = int(dt_max), int(dt_step), int(dt_min)
        desc = _capi.FdmtDesc(fmin=self.m_f_min, fmax=self.m_f_max, nchan=self.m_nchans,
                              ncols=self.m_nsamps, max_dt=self.m_dt_max, plan_kind=_capi.BFS_PLAN_PRAVIR,
                              fuse_depth=0, dt_min=self.m_dt_min, dt_step=self.m_dt_step,
                              tsamp=self.m_tsamp,
                              flags=_capi.BFS_FDMT_EXTERNAL_WS if external_ws else 0)
        self._plan = ctypes.c_void_p()
        _capi.call("bfs_fdmt_plan_create", ctypes.byref(desc), ctypes.byref(self._plan))
        self.info = _capi.FdmtInfo()
        _capi.call("bfs_fdmt_plan_info", self._plan, ctypes.byref(self.info))

    def __del__(self):
        p = getattr(self, "_plan", None)
        if p is not None and p.value:
            try:
                _capi.lib().bfs_fdmt_plan_destroy(p)
            except Exception:
                pass
            self._plan = None

    # --- the reference's getters --------------------------------------------
    def get_df(self) -> float:
        return float(np.float32(np.float32(self.m_f_max) - np.float32(self.m_f_min)) / np.float32(self.m_nchans))

    def get_correction(self) -> float:
        return float(np.float32(self.get_df()) / np.float32(2))

    def get_niters(self) -> int:
        return int(self.info.niter)

    def get_dt_grid_final(self) -> list[int]:
        n = int(self.info.out_rows)
        dt = np.zeros(n, np.int32)
        _capi.call("bfs_fdmt_plan_delays", self._plan, dt.ctypes.data_as(ctypes.c_void_p), n, None, None, 0)
        return [int(v) for v in dt]

    def get_dm_grid_final(self) -> list[float]:
        """dt * tsamp / (K (f_min^-2 - f_max^-2)) in float32
        (L/FDMT_PRAVIR/fdmt_base.cpp:64-74)."""
        f32 = np.float32
        conv = f32(K_DISP_MT * (np.power(f32(self.m_f_min), f32(-2.0)) - np.power(f32(self.m_f_max), f32(-2.0))))
        step = f32(f32(self.m_tsamp) / conv)
        return [float(f32(f32(dt) * step)) for dt in self.get_dt_grid_final()]

    @property
    def out_rows(self) -> int:
        return int(self.info.out_rows)

    @property
    def alg_bytes(self) -> float:
        return float(self.info.alg_bytes)

    # --- transform --------------------------------------------------------------
    def execute(self, waterfall: torch.Tensor, waterfall_size: int, dmt: torch.Tensor, dmt_size: int,
                stream: torch.cuda.Stream | None = None) -> None:
        if waterfall_size != self.m_nchans * self.m_nsamps or waterfall.numel() != waterfall_size:
            raise ValueError("Invalid size of waterfall")
        if dmt_size != self.out_rows * self.m_nsamps or dmt.numel() != dmt_size:
            raise ValueError("Invalid size of dmt")
        _capi.call("bfs_fdmt_execute", self._plan, dev_ptr(waterfall, torch.float32, "waterfall"),
                   dev_ptr(dmt, torch.float32, "dmt"), 0, stream_handle(stream))

    def __call__(self, waterfall: torch.Tensor) -> torch.Tensor:
        out = torch.empty((self.out_rows, self.m_nsamps), dtype=torch.float32, device=waterfall.device)
        self.execute(waterfall, waterfall.numel(), out, out.numel())
        return out

    def adjoint(self, d_grad_out: torch.Tensor, d_grad_in: torch.Tensor | None = None,
                stream: torch.cuda.Stream | None = None) -> torch.Tensor:
        if d_grad_in is None:
            d_grad_in = torch.empty((self.m_nchans, self.m_nsamps), dtype=torch.float32,
                                    device=d_grad_out.device)
        _capi.call("bfs_fdmt_adjoint", self._plan, dev_ptr(d_grad_out, torch.float32, "d_grad_out"),
                   dev_ptr(d_grad_in, torch.float32, "d_grad_in"), stream_handle(stream))
        return d_grad_in

