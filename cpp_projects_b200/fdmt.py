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
    """Time the fused-head depths and tile widths for this shape on the
    current device (cached per shape): returns (fuse_depth, head_tile, ms)."""
    desc = _capi.FdmtDesc(fmin=float(Fmin), fmax=float(Fmax), nchan=int(nchan), ncols=int(cols),
                          max_dt=int(imaxDt))
    depth, tile, ms = ctypes.c_int(0), ctypes.c_int(0), ctypes.c_float(0)
    _capi.call("bfs_fdmt_autotune", ctypes.byref(desc), ctypes.byref(depth), ctypes.byref(tile),
               ctypes.byref(ms))
    return depth.value, tile.value, ms.value


class CFdmtGpu:
    def __init__(self, Fmin: float, Fmax: float, nchan: int, cols: int, imaxDt: int,
                 fuse_depth: int = -1, external_ws: bool = False, head_tile: int = 0,
                 precision: int = 0):
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
                              head_tile=int(head_tile))
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
