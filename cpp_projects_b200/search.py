"""Boxcar detection and DM-time plane normalisation (host mirror).

Mirrors the reference's ``clusterization`` gather entry points
(MyVSLib_C++/Clusterization/Clusterization.cuh):

* :func:`gather_candidates_in_dynamicalArray` — widths 1, 2, 4 .. 2^Q,
  ``mwidth = log2 w`` (Clusterization.cu:56-89);
* :func:`gather_candidates_in_heap_with_plan` — widths 1..W, ``mwidth = w``
  (Clusterization.cu:169-202).

Candidates come back as an ``(n, 4)`` int32 CUDA tensor whose rows are the
reference's 16-byte ``Cand`` records (``mt, mdt, mwidth`` and the float bits of
``msnr``), sorted in the canonical (mdt, mt, width) order.  The reference
returns a freshly ``cudaMalloc``'d array and a host count; here the tensor
owns the memory.  ``thr`` may be a Python float or a 1-element CUDA tensor
(the reference passes a reference bound to device memory).
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _capi
from ._tensors import dev_ptr, opt_ptr, stream_handle

CAND_DTYPE = np.dtype([("mt", "<i4"), ("mdt", "<i4"), ("mwidth", "<i4"), ("msnr", "<f4")])
DEFAULT_CAPACITY = 1 << 20


def cands_to_numpy(c: torch.Tensor) -> np.ndarray:
    """(n, 4) int32 tensor of Cand records -> numpy structured array."""
    a = np.ascontiguousarray(c.detach().cpu().numpy().astype(np.int32, copy=False))
    return a.view(CAND_DTYPE).reshape(-1)


def cands_from_numpy(a: np.ndarray, device) -> torch.Tensor:
    a = np.ascontiguousarray(a, CAND_DTYPE)
    return torch.from_numpy(a.view(np.int32).reshape(-1, 4).copy()).to(device)


def row_stats(plane: torch.Tensor, stream=None) -> torch.Tensor:
    rows, cols = plane.shape
    st = torch.empty(2 * rows, dtype=torch.float32, device=plane.device)
    _capi.call("bfs_row_stats", dev_ptr(plane, torch.float32, "plane"), rows, cols,
               dev_ptr(st), stream_handle(stream))
    return st


def launch_row_stats(plane: torch.Tensor, stats: torch.Tensor, stream=None) -> None:
    rows, cols = plane.shape
    _capi.call("bfs_row_stats", dev_ptr(plane, torch.float32, "plane"), rows, cols,
               dev_ptr(stats, torch.float32, "stats"), stream_handle(stream))


def norm_rows(plane: torch.Tensor, out: torch.Tensor | None = None, stream=None):
    """Per-delay-row (x - mean_r) / std_r; returns (normalised plane, stats)."""
    rows, cols = plane.shape
    out = torch.empty_like(plane) if out is None else out
    st = torch.empty(2 * rows, dtype=torch.float32, device=plane.device)
    _capi.call("bfs_norm_rows", dev_ptr(plane, torch.float32, "plane"),
               dev_ptr(out, torch.float32, "out"), rows, cols, dev_ptr(st), stream_handle(stream))
    return out, st


def boxcar_gather(plane: torch.Tensor, thr, widths_mode: int, param: int,
                  stats: torch.Tensor | None = None, snr_fast: bool = False,
                  capacity: int = DEFAULT_CAPACITY, out: torch.Tensor | None = None,
                  stream=None):
    """Returns (candidates (n,4) int32, total count found).  Raises BfsError
    (BFS_ERR_OVERFLOW) when more than ``capacity`` were found."""
    rows, cols = plane.shape
    if out is None:
        out = torch.empty((max(capacity, 1), 4), dtype=torch.int32, device=plane.device)
    capacity = out.shape[0]
    d_thr = None
    thr_host = 0.0
    if isinstance(thr, torch.Tensor):
        d_thr = dev_ptr(thr, torch.float32, "thr")
    else:
        thr_host = float(thr)
    count = ctypes.c_uint32(0)
    st = _capi.lib().bfs_boxcar_gather(
        dev_ptr(plane, torch.float32, "plane"), rows, cols, opt_ptr(stats, torch.float32, "stats"),
        ctypes.c_float(thr_host), d_thr, int(widths_mode), int(param), 1 if snr_fast else 0,
        dev_ptr(out, torch.int32, "out"), ctypes.c_uint32(capacity), ctypes.byref(count),
        stream_handle(stream))
    _capi.check(st)
    return out[: count.value], int(count.value)


# --- reference names ---------------------------------------------------------
def gather_candidates_in_dynamicalArray(d_arr_fdmt: torch.Tensor, Rows: int, Cols: int,
                                        val_thresh, QUantPower2_Wnd: int, **kw):
    plane = d_arr_fdmt.view(Rows, Cols)
    return boxcar_gather(plane, val_thresh, _capi.BFS_WIDTHS_POW2, QUantPower2_Wnd, **kw)


def gather_candidates_in_heap_with_plan(d_fdmt: torch.Tensor, Rows: int, Cols: int,
                                        d_VAlTresh, WndWidth: int, **kw):
    plane = d_fdmt.view(Rows, Cols)
    return boxcar_gather(plane, d_VAlTresh, _capi.BFS_WIDTHS_ALL, WndWidth, **kw)


# ---- S/N at cells and its gradient --------------------------------------------
def _cells_tensor(cells, rows: int, cols: int, device) -> torch.Tensor:
    c = torch.as_tensor(cells, dtype=torch.int32).reshape(-1, 3)
    ch = c.cpu()
    if len(ch) and not (bool((ch[:, 0] >= 0).all()) and bool((ch[:, 0] < rows).all())
                        and bool((ch[:, 1] >= 0).all()) and bool((ch[:, 2] >= 1).all())
                        and bool((ch[:, 1] + ch[:, 2] <= cols).all())):
        raise ValueError("cells must be {row, start, width} inside the plane")
    return c.to(device).contiguous()


def snr_cells(plane: torch.Tensor, stats: torch.Tensor, cells, stream=None) -> torch.Tensor:
    """Boxcar S/N at cells (n x {row, start, width}) of the plane normalised
    by ``stats`` (means, stds); the same value the boxcar search reports."""
    rows, cols = plane.shape
    c = _cells_tensor(cells, rows, cols, plane.device)
    out = torch.empty(c.shape[0], dtype=torch.float32, device=plane.device)
    _capi.call("bfs_boxcar_snr_cells", dev_ptr(plane, torch.float32, "plane"), rows, cols,
               dev_ptr(stats, torch.float32, "stats"), dev_ptr(c), int(c.shape[0]), dev_ptr(out),
               stream_handle(stream))
    return out


def snr_cells_adjoint(plane: torch.Tensor, stats: torch.Tensor, cells, snr: torch.Tensor,
                      gsnr: torch.Tensor, out: torch.Tensor | None = None, stream=None) -> torch.Tensor:
    """Gradient of sum_k gsnr[k] * S_k with respect to the plane (the row
    statistics' dependence on the plane included)."""
    rows, cols = plane.shape
    c = _cells_tensor(cells, rows, cols, plane.device)
    out = torch.empty_like(plane) if out is None else out
    _capi.call("bfs_boxcar_snr_cells_adjoint", dev_ptr(plane, torch.float32, "plane"), rows, cols,
               dev_ptr(stats, torch.float32, "stats"), dev_ptr(c), int(c.shape[0]),
               dev_ptr(snr, torch.float32, "snr"), dev_ptr(gsnr.contiguous(), torch.float32, "gsnr"),
               dev_ptr(out, torch.float32, "out"), stream_handle(stream))
    return out

