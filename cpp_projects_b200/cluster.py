"""Candidate clustering and delegate logs (host mirror of the reference's
``clusterization::complete_clusterization`` / ``clusterization_main`` and
``select_delegates``; MyVSLib_C++/Clusterization/Clusterization.cu:17-166,
select_delegates.cu:63-177)."""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _capi
from ._tensors import dev_ptr, stream_handle
from .search import CAND_DTYPE, cands_to_numpy, gather_candidates_in_heap_with_plan


class Clusters:
    """Result of :func:`complete_clusterization` (device tensors)."""

    def __init__(self, cands, perm, offsets, delegates, ngroups):
        self.cands = cands            # (n, 4) int32 Cand records
        self.perm = perm              # (n,) members in group order
        self.offsets = offsets        # (ngroups + 1,) group starts
        self.delegates = delegates    # (ngroups,) delegate index per group, sorted by (mt, group)
        self.ngroups = ngroups

    def delegate_records(self) -> np.ndarray:
        """Delegate Cand records (gathered on the device; only they cross PCIe)."""
        if self.ngroups == 0:
            return np.zeros(0, CAND_DTYPE)
        return cands_to_numpy(self.cands.index_select(0, self.delegates.long()))

    def group_sizes(self) -> np.ndarray:
        """Sizes in group order (the order of ``offsets``)."""
        o = self.offsets.cpu().numpy()
        return np.diff(o)

    def delegate_group_sizes(self) -> np.ndarray:
        """Size of each delegate's own group, in delegate order (computed on
        the device: position of the delegate in ``perm`` -> its group)."""
        if self.ngroups == 0:
            return np.zeros(0, np.int64)
        n = int(self.perm.shape[0])
        inv = torch.empty(n, dtype=torch.int64, device=self.perm.device)
        inv[self.perm.long()] = torch.arange(n, device=self.perm.device)
        pos = inv[self.delegates.long()]
        offs = self.offsets.long()
        g = torch.searchsorted(offs, pos, right=True) - 1
        return (offs[g + 1] - offs[g]).cpu().numpy()


def complete_clusterization(cands: torch.Tensor, metrics, stream=None) -> Clusters:
    n = int(cands.shape[0])
    dev = cands.device
    perm = torch.empty(max(n, 1), dtype=torch.int32, device=dev)
    offsets = torch.empty(n + 1, dtype=torch.int32, device=dev)
    delegates = torch.empty(max(n, 1), dtype=torch.int32, device=dev)
    m = (ctypes.c_int * 3)(*[int(v) for v in metrics])
    ng = ctypes.c_uint32(0)
    if n > 0:
        _capi.call("bfs_cluster", dev_ptr(cands, torch.int32, "cands"), ctypes.c_uint32(n), m,
                   dev_ptr(perm), dev_ptr(offsets), dev_ptr(delegates), ctypes.byref(ng),
                   stream_handle(stream))
    g = int(ng.value)
    return Clusters(cands, perm[:n], offsets[: g + 1] if n else offsets[:1].zero_(),
                    delegates[:g], g)


def select_delegates(cands, perm, offsets, stream=None) -> torch.Tensor:
    """Per-group argmax of msnr; perm and offsets as ``clusterization_main``
    returns them (one perm entry per candidate, ngroups + 1 offsets)."""
    ng = int(offsets.shape[0]) - 1
    if ng < 0:
        raise ValueError("offsets needs at least one entry")
    if perm.shape[0] != cands.shape[0]:
        raise ValueError(f"perm has {perm.shape[0]} entries for {cands.shape[0]} candidates")
    out = torch.empty(max(ng, 1), dtype=torch.int32, device=cands.device)
    _capi.call("bfs_select_delegates", dev_ptr(cands, torch.int32), dev_ptr(perm, torch.int32),
               ctypes.c_uint32(int(cands.shape[0])), dev_ptr(offsets, torch.int32),
               ctypes.c_uint32(ng), dev_ptr(out), stream_handle(stream))
    return out[:ng]


# --- text formats -------------------------------------------------------------
def _fmt_g(v: float) -> str:
    """C++ ostream default formatting (6 significant digits, %g-like)."""
    return f"{v:.6g}"


def write_log(cl: Clusters, filename: str, delt_bin: float, t_chunkBegin: float,
              num_from_delegate_group: bool = False) -> None:
    """Delegate log in the reference's layout (select_delegates.cu:127-177):
    columns N, t bin, t sec, dedisp, width, SNR, num, each setw(10).
    The reference pairs the i-th delegate (sorted by mt) with the i-th group's
    size in group order; that quirk is kept unless num_from_delegate_group."""
    drec = cl.delegate_records()
    sizes = cl.delegate_group_sizes() if num_from_delegate_group else cl.group_sizes()
    with open(filename, "w") as f:
        f.write("".join(s.rjust(10) for s in ("N", "t, bin", "t, sec", "dedisp", "width", "SNR",
                                                "num")) + "\n")
        for i in range(cl.ngroups):
            r = drec[i]
            num = sizes[i]
            t_sec = np.float32(t_chunkBegin) + np.float32(r["mt"]) * np.float32(delt_bin)
            cols = [str(i + 1), str(int(r["mt"])), _fmt_g(float(t_sec)), str(int(r["mdt"])),
                    str(int(r["mwidth"])), _fmt_g(float(r["msnr"])), str(int(num))]
            f.write("".join(s.rjust(10) for s in cols) + "\n")


def writeCandHostArrayToCSV(cands: np.ndarray, filename: str) -> None:
    """CSV ``mt,mdt,mwidth,msnr`` (Clusterization.cu:338-358)."""
    with open(filename, "w") as f:
        f.write("mt,mdt,mwidth,msnr\n")
        for r in cands:
            f.write(f"{int(r['mt'])},{int(r['mdt'])},{int(r['mwidth'])},{_fmt_g(float(r['msnr']))}\n")


def clusterization_main(d_fdmt: torch.Tensor, Rows: int, Cols: int, d_VAlTresh, WndWidth: int,
                        metrics, filename: str, delt_bin: float, t_chunkBegin: float,
                        bwrite: bool = True):
    """Gather with every width 1..WndWidth, cluster, and write the delegate log.
    Returns the Clusters, or None when no candidate passed (the reference
    returns false there)."""
    cands, n = gather_candidates_in_heap_with_plan(d_fdmt, Rows, Cols, d_VAlTresh, WndWidth)
    if n == 0:
        return None
    cl = complete_clusterization(cands, metrics)
    if bwrite:
        write_log(cl, filename, delt_bin, t_chunkBegin)
    return cl
