"""Differentiable FDMT + boxcar S/N (torch.autograd.Function bindings).

The forward passes run the library's FDMT and the boxcar S/N at chosen
cells; the backward passes run the hand-written adjoints (bfs_fdmt_adjoint,
bfs_boxcar_snr_cells_adjoint).  No reference counterpart: the reference has
no gradients.  Typical use — optimise per-channel weights ``w`` (bandpass /
RFI mask) for the S/N of known pulses::

    y = fdmt(w[:, None] * x, plan)          # x: nchan x T filterbank
    loss = -boxcar_snr(y, cells).sum()      # cells: n x {row, start, width}
    loss.backward()                          # w.grad, via the adjoints
"""
from __future__ import annotations

import torch

from . import search
from .fdmt import CFdmtGpu


class FdmtFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x: torch.Tensor, plan: CFdmtGpu) -> torch.Tensor:
        x = x.contiguous()
        y = torch.empty((plan.m_imaxDt, plan.m_cols), dtype=torch.float32, device=x.device)
        plan.process_image(x, y, False)
        ctx.plan = plan
        return y

    @staticmethod
    def backward(ctx, gy: torch.Tensor):
        return ctx.plan.adjoint(gy.contiguous()), None


class BoxcarSnrFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, y: torch.Tensor, cells: torch.Tensor) -> torch.Tensor:
        y = y.contiguous()
        stats = search.row_stats(y)
        snr = search.snr_cells(y, stats, cells)
        ctx.save_for_backward(y, stats, snr)
        ctx.cells = cells
        return snr

    @staticmethod
    def backward(ctx, gsnr: torch.Tensor):
        y, stats, snr = ctx.saved_tensors
        return search.snr_cells_adjoint(y, stats, ctx.cells, snr, gsnr.contiguous()), None


def fdmt(x: torch.Tensor, plan: CFdmtGpu) -> torch.Tensor:
    """FDMT of a (nchan x T) float32 CUDA tensor, differentiable in x."""
    return FdmtFunction.apply(x, plan)


def boxcar_snr(y: torch.Tensor, cells) -> torch.Tensor:
    """Boxcar S/N at cells (n x {row, start, width}) of the row-normalised
    plane y, differentiable in y (row means and stds included)."""
    return BoxcarSnrFunction.apply(y, torch.as_tensor(cells, dtype=torch.int32))
