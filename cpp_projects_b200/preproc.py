"""Statistical preprocessing of the FDMT input (host mirror of the
reference's ``statistical_preprocessing::calc_fdmt_inputs``,
MyVSLib_C++/CDMT/Statistical_preprocessing.cu:15-88, and ``fdmt_normalization``,
MyVSLib_C++/CDMT/Chunk_gpu.cu:842-852)."""
from __future__ import annotations

import torch

from . import _capi
from ._tensors import dev_ptr, stream_handle


def calc_fdmt_inputs(d_parr_inp: torch.Tensor, NRows: int, NCols: int, d_buff: torch.Tensor,
                     d_parrNormInput: torch.Tensor, stream=None) -> None:
    """In place: zero rows whose variance is > 4 sigma off the mean variance
    (mask 0), normalise the rest to (x - mean)/std (mask 1).  d_buff holds
    4 + 2*NRows floats: [row mean][row variance][mean][std][var mean][var std]."""
    if d_buff.numel() < 4 + 2 * NRows:
        raise ValueError("d_buff needs 4 + 2*NRows floats")
    _capi.call("bfs_preproc_calc_fdmt_inputs", dev_ptr(d_parr_inp, torch.float32, "d_parr_inp"),
               NRows, NCols, dev_ptr(d_buff, torch.float32, "d_buff"),
               dev_ptr(d_parrNormInput, torch.float32, "d_parrNormInput"), stream_handle(stream))


def fdmt_normalization(d_arr: torch.Tensor, d_norm: torch.Tensor, len_: int,
                       d_pOutArray: torch.Tensor, stream=None) -> None:
    _capi.call("bfs_fdmt_normalize", dev_ptr(d_arr, torch.float32), dev_ptr(d_norm, torch.float32),
               int(len_), dev_ptr(d_pOutArray, torch.float32), stream_handle(stream))
