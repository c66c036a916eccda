"""ORACLE — test infrastructure only.

ctypes wrapper over ``oracle/liboracle.so`` (the C restatement in
``fdmt_oracle.c`` / ``search_oracle.c``) and, when it has been built,
``oracle/_ref/libref_fdmt.so`` (the reference's own ``CFdmtCpu`` compiled from
its sources by ``oracle/Makefile``).  Only tests/, ``__graft_entry__.smoke()``
and bench.py's CPU-baseline leg may use this module, and only as the checker.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
_P = ctypes.c_void_p
_F = ctypes.c_float

CAND_DTYPE = np.dtype([("mt", "<i4"), ("mdt", "<i4"), ("mwidth", "<i4"), ("msnr", "<f4")])

_lib = None
_ref = None
_ref_gpu = None


def reference_dir() -> Path:
    """The reference checkout the oracle's recipe builds from:
    BFS_REFERENCE_DIR, else oracle/Makefile's default (it may be absent)."""
    env = os.environ.get("BFS_REFERENCE_DIR")
    if env:
        return Path(env)
    r = subprocess.run(["make", "-s", "-C", str(HERE), "print-ref"], capture_output=True, text=True)
    return Path(r.stdout.strip()) if r.returncode == 0 and r.stdout.strip() else Path("/nonexistent")


def build() -> None:
    """Compile the oracle (and the reference shim when the sources exist)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True, capture_output=True)


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        path = HERE / "liboracle.so"
        if not path.exists():
            build()
        _lib = ctypes.CDLL(str(path))
        _lib.orc_boxcar.restype = ctypes.c_int64
        _lib.orc_boxcar.argtypes = [_P, ctypes.c_int, ctypes.c_int, _F, ctypes.c_int,
                                    ctypes.c_int, _P, ctypes.c_int64]
        _lib.orc_boxcar_mt.restype = ctypes.c_int64
        _lib.orc_boxcar_mt.argtypes = _lib.orc_boxcar.argtypes
        for n in ("orc_fdmt_rows", "orc_fdmt_tables", "orc_fdmt_run_f32", "orc_fdmt_run_f64"):
            getattr(_lib, n).restype = ctypes.c_int
    return _lib


def ref_lib() -> ctypes.CDLL | None:
    """The reference's CFdmtCpu (oracle/_ref), or None when it was not built."""
    global _ref
    if _ref is None:
        path = HERE / "_ref" / "libref_fdmt.so"
        if not path.exists():
            return None
        _ref = ctypes.CDLL(str(path))
    return _ref


_ref_report = None


def _report_lib():
    global _ref_report
    if _ref_report is None:
        p = HERE / "_ref" / "libref_report.so"
        if not p.exists():
            return None
        _ref_report = ctypes.CDLL(str(p))
        _ref_report.ref_write_report.argtypes = [ctypes.c_char_p, ctypes.c_int, _P, _P, _P, _F]
        _ref_report.ref_read_report_line.restype = ctypes.c_int
        _ref_report.ref_read_report_line.argtypes = [ctypes.c_char_p, ctypes.c_int, _P, _P]
    return _ref_report


def ref_write_report(path, records, pulse_length) -> bool:
    """The reference's COutChunkHeader::writeReport; records are tuples
    (nrows, ncols, suc_row, suc_col, width, snr, cohdisp, block, chunk)."""
    lib_ = _report_lib()
    if lib_ is None:
        return False
    ints = np.zeros((max(len(records), 1), 9), np.int32)
    snr = np.zeros(max(len(records), 1), np.float32)
    coh = np.zeros(max(len(records), 1), np.float32)
    for i, r in enumerate(records):
        ints[i, :5] = r[:5]
        snr[i], coh[i] = r[5], r[6]
        ints[i, 5], ints[i, 6] = r[7], r[8]
    lib_.ref_write_report(str(path).encode(), len(records), _ptr(ints), _ptr(snr), _ptr(coh), pulse_length)
    return True


def ref_read_report_line(path, line) -> dict | None:
    lib_ = _report_lib()
    if lib_ is None:
        return None
    ints = np.zeros(7, np.int32)
    fl = np.zeros(2, np.float32)
    if not lib_.ref_read_report_line(str(path).encode(), int(line), _ptr(ints), _ptr(fl)):
        return {"ok": False}
    return {"ok": True, "numBlock": int(ints[0]), "numChunk": int(ints[1]), "nrows": int(ints[2]),
            "ncols": int(ints[3]), "sucRow": int(ints[4]), "sucCol": int(ints[5]), "width": int(ints[6]),
            "cohDisp": float(fl[0]), "snr": float(fl[1])}


def cut_quadratic_fragment(plane: np.ndarray, target_row: int, target_col: int):
    """Restates CChunkB::cutQuadraticFragment (MyVSLib_C++/CDMT/ChunkB.cpp:
    255-275) on the flat row-major plane; positions past its end read 0
    (the reference's memcpy would read outside the array there)."""
    rows, cols = plane.shape
    flat = np.ascontiguousarray(plane, np.float32).reshape(-1)
    if rows < cols:
        d, cb, rb = rows, (target_col // rows) * rows, 0
        start = cb
    else:
        part = target_row // rows
        d, cb, rb = cols, 0, part
        start = part * cols
    out = np.zeros((d, d), np.float32)
    for i in range(d):
        a = i * cols + start
        n = max(0, min(d, flat.size - a))
        out[i, :n] = flat[a:a + n]
    return out, rb, cb


_ref_guppi = None


def ref_guppi_header(path, offset: int = 0) -> dict | None:
    """The reference's CTelescopeHeader::readGuppiHeader on the block starting
    at `offset` (None if oracle/_ref was not built; {'ok': False} if it
    rejects the header)."""
    global _ref_guppi
    if _ref_guppi is None:
        p = HERE / "_ref" / "libref_guppi.so"
        if not p.exists():
            return None
        _ref_guppi = ctypes.CDLL(str(p))
        _ref_guppi.ref_guppi_read_header.restype = ctypes.c_int
    i = [ctypes.c_int(0) for _ in range(5)]
    f = [ctypes.c_float(0) for _ in range(4)]
    blk = ctypes.c_longlong(0)
    pos = ctypes.c_long(0)
    ok = _ref_guppi.ref_guppi_read_header(
        str(path).encode(), ctypes.c_long(offset), ctypes.byref(i[0]), ctypes.byref(f[0]), ctypes.byref(i[1]),
        ctypes.byref(i[2]), ctypes.byref(f[1]), ctypes.byref(i[3]), ctypes.byref(f[2]), ctypes.byref(blk),
        ctypes.byref(i[4]), ctypes.byref(f[3]), ctypes.byref(pos))
    return {"ok": ok == 1, "nbits": i[0].value, "chan_bw": f[0].value, "npol": i[1].value,
            "directio": i[2].value, "obsfreq": f[1].value, "nchan": i[3].value, "obsbw": f[2].value,
            "blocsize": blk.value, "telescope": i[4].value, "tbin": f[3].value, "data_pos": pos.value}


_ref_pravir = None


def ref_pravir_lib() -> ctypes.CDLL | None:
    """The reference's own FDMTCPU (Pravir plan, oracle/_ref), or None."""
    global _ref_pravir
    if _ref_pravir is None:
        path = HERE / "_ref" / "libref_pravir.so"
        if not path.exists():
            return None
        l = ctypes.CDLL(str(path))
        L = ctypes.c_long
        l.ref_pravir_rows.restype = L
        l.ref_pravir_rows.argtypes = [_F, _F, L, L, _F, L, L, L]
        l.ref_pravir_dt_grid.restype = L
        l.ref_pravir_dt_grid.argtypes = [_F, _F, L, L, _F, L, L, L, _P, L]
        l.ref_pravir_execute.restype = ctypes.c_int
        l.ref_pravir_execute.argtypes = [_F, _F, L, L, _F, L, L, L, _P, _P, L, ctypes.c_int]
        _ref_pravir = l
    return _ref_pravir


def ref_gpu_lib() -> ctypes.CDLL | None:
    """The reference's own GPU classes (oracle/_ref/libref_gpu.so), or None."""
    global _ref_gpu
    if _ref_gpu is None:
        path = HERE / "_ref" / "libref_gpu.so"
        if not path.exists():
            return None
        l = ctypes.CDLL(str(path))
        l.ref_fdmt_gpu_create.restype = ctypes.c_void_p
        l.ref_fdmt_gpu_create.argtypes = [_F, _F, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        l.ref_fdmt_gpu_destroy.argtypes = [_P]
        l.ref_fdmt_gpu_process.argtypes = [_P, _P, _P, ctypes.c_int]
        for n in ("ref_gather_heap", "ref_gather_dynamic"):
            getattr(l, n).restype = ctypes.c_uint
            getattr(l, n).argtypes = [_P, ctypes.c_int, ctypes.c_int, _P, ctypes.c_int, _P, ctypes.c_uint]
        l.ref_cluster_heap.restype = ctypes.c_uint
        l.ref_cluster_heap.argtypes = [_P, ctypes.c_int, ctypes.c_int, _P, ctypes.c_int, _P,
                                       ctypes.c_char_p, _F, _F]
        l.ref_search_dynamic.restype = ctypes.c_uint
        l.ref_search_dynamic.argtypes = [_P, ctypes.c_int, ctypes.c_int, _P, ctypes.c_int, _P,
                                         ctypes.c_char_p, _F, _F]
        _ref_gpu = l
    return _ref_gpu


class RefFdmtGpu:
    """The reference's CFdmtGpu (device pointers as ints; default stream)."""

    def __init__(self, fmin, fmax, nchan, cols, max_dt):
        self.l = ref_gpu_lib()
        self.h = self.l.ref_fdmt_gpu_create(_F(fmin), _F(fmax), nchan, cols, max_dt)

    def process_image(self, d_in: int, d_out: int, b_ones=False) -> int:
        return self.l.ref_fdmt_gpu_process(self.h, _P(d_in), _P(d_out), 1 if b_ones else 0)

    def __del__(self):
        if getattr(self, "h", None):
            self.l.ref_fdmt_gpu_destroy(self.h)
            self.h = None


def ref_gpu_gather(d_plane: int, rows: int, cols: int, d_thr: int, mode: int, param: int,
                   cap: int = 1 << 22) -> np.ndarray:
    """The reference's gather (mode 0: dynamic, widths 2^q; 1: heap, widths 1..W)."""
    l = ref_gpu_lib()
    out = np.zeros(cap, CAND_DTYPE)
    fn = l.ref_gather_dynamic if mode == 0 else l.ref_gather_heap
    n = fn(_P(d_plane), rows, cols, _P(d_thr), param, _ptr(out), cap)
    return out[: min(n, cap)].copy()


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(_P)


# ---- FDMT -------------------------------------------------------------------
def fdmt_rows(fmin, fmax, nchan, max_dt) -> np.ndarray:
    rows = np.zeros(64, np.int32)
    n = lib().orc_fdmt_rows(_F(fmin), _F(fmax), nchan, max_dt, _ptr(rows), rows.size)
    if n < 0:
        raise ValueError("bad FDMT parameters")
    return rows[: n + 1].copy()


def fdmt_tables(fmin, fmax, nchan, max_dt, level):
    n = int(fdmt_rows(fmin, fmax, nchan, max_dt)[level])
    a = np.zeros(n, np.int32); b = np.zeros(n, np.int32); s = np.zeros(n, np.int32)
    lib().orc_fdmt_tables(_F(fmin), _F(fmax), nchan, max_dt, level, _ptr(a), _ptr(b), _ptr(s), n)
    return a, b, s


def fdmt_f32(fmin, fmax, x: np.ndarray | None, nchan, ncols, max_dt, b_ones=False) -> np.ndarray:
    out = np.zeros((max_dt, ncols), np.float32)
    xin = np.zeros(1, np.float32) if b_ones else np.ascontiguousarray(x, np.float32)
    rc = lib().orc_fdmt_run_f32(_F(fmin), _F(fmax), nchan, ncols, max_dt, _ptr(xin), _ptr(out),
                                1 if b_ones else 0)
    if rc != 0:
        raise ValueError(f"oracle FDMT failed ({rc})")
    return out


def fdmt_f64(fmin, fmax, x: np.ndarray | None, nchan, ncols, max_dt, b_ones=False) -> np.ndarray:
    out = np.zeros((max_dt, ncols), np.float64)
    xin = np.zeros(1, np.float64) if b_ones else np.ascontiguousarray(x, np.float64)
    rc = lib().orc_fdmt_run_f64(_F(fmin), _F(fmax), nchan, ncols, max_dt, _ptr(xin), _ptr(out),
                                1 if b_ones else 0)
    if rc != 0:
        raise ValueError(f"oracle FDMT failed ({rc})")
    return out


PREC_F16, PREC_BF16 = 1, 2


def fdmt_lowp(fmin, fmax, x: np.ndarray | None, nchan, ncols, max_dt, prec: int, kstore: int,
              b_ones=False) -> np.ndarray:
    """The FP32 FDMT whose planes of levels kstore..niter-1 are rounded to
    FP16 (prec 1) or BF16 (prec 2) with the per-row power-of-two scale."""
    out = np.zeros((max_dt, ncols), np.float32)
    xin = np.zeros(1, np.float32) if b_ones else np.ascontiguousarray(x, np.float32)
    rc = lib().orc_fdmt_run_lowp(_F(fmin), _F(fmax), nchan, ncols, max_dt, _ptr(xin), _ptr(out),
                                 1 if b_ones else 0, int(prec), int(kstore))
    if rc != 0:
        raise ValueError(f"oracle FDMT failed ({rc})")
    return out


def round16(x: np.ndarray, prec: int) -> np.ndarray:
    x = np.ascontiguousarray(x, np.float32)
    out = np.empty_like(x)
    lib().orc_round16(_ptr(x), _ptr(out), ctypes.c_int64(x.size), int(prec))
    return out


def fdmt_adjoint_f32(fmin, fmax, gy: np.ndarray, nchan, ncols, max_dt) -> np.ndarray:
    """F^T gy in FP32, summed in the product's order."""
    gx = np.zeros((nchan, ncols), np.float32)
    g = np.ascontiguousarray(gy, np.float32)
    if lib().orc_fdmt_adjoint_f32(_F(fmin), _F(fmax), nchan, ncols, max_dt, _ptr(g), _ptr(gx)) != 0:
        raise ValueError("oracle adjoint failed")
    return gx


def fdmt_adjoint_f64(fmin, fmax, gy: np.ndarray, nchan, ncols, max_dt) -> np.ndarray:
    gx = np.zeros((nchan, ncols), np.float64)
    g = np.ascontiguousarray(gy, np.float64)
    if lib().orc_fdmt_adjoint_f64(_F(fmin), _F(fmax), nchan, ncols, max_dt, _ptr(g), _ptr(gx)) != 0:
        raise ValueError("oracle adjoint failed")
    return gx


def snr_cells_f64(y: np.ndarray, cells: np.ndarray):
    """S/N at cells {row, start, width} of the plane y with FP64 row mean and
    population std; returns (snr, dsnr_dy) where dsnr_dy[k] is the gradient
    of S_k with respect to row cells[k, 0] (a length-ncols vector)."""
    y = np.asarray(y, np.float64)
    n = y.shape[1]
    snr = np.zeros(len(cells))
    grads = []
    for k, (d, t, w) in enumerate(np.asarray(cells, np.int64)):
        row = y[d]
        m = row.mean()
        sd = np.sqrt(((row - m) ** 2).mean())
        z = (row - m) / sd
        snr[k] = z[t:t + w].sum() / np.sqrt(w)
        win = np.zeros(n)
        win[t:t + w] = 1.0
        grads.append((win - w / n) / (sd * np.sqrt(w)) - snr[k] * (row - m) / (n * sd * sd))
    return snr, grads


# ---- Pravir plan kind -----------------------------------------------------------
def _pravir_lib():
    l = lib()
    L = ctypes.c_long
    for n in ("orc_pravir_rows", "orc_pravir_level", "orc_pravir_run_f32", "orc_pravir_run_f64",
              "orc_pravir_adjoint_f32", "orc_pravir_adjoint_f64"):
        getattr(l, n).restype = ctypes.c_int
    l.orc_pravir_rows.argtypes = [_F, _F, ctypes.c_int, ctypes.c_int, L, L, L, _P, ctypes.c_int]
    l.orc_pravir_level.argtypes = [_F, _F, ctypes.c_int, ctypes.c_int, L, L, L, ctypes.c_int,
                                   _P, _P, _P, _P, _P, ctypes.c_int]
    for n in ("orc_pravir_run_f32", "orc_pravir_run_f64", "orc_pravir_adjoint_f32", "orc_pravir_adjoint_f64"):
        getattr(l, n).argtypes = [_F, _F, ctypes.c_int, ctypes.c_int, L, L, L, _P, _P]
    return l


def pravir_rows(fmin, fmax, nchans, nsamps, dt_max, dt_step=1, dt_min=0) -> np.ndarray:
    rows = np.zeros(64, np.int32)
    n = _pravir_lib().orc_pravir_rows(_F(fmin), _F(fmax), nchans, nsamps, dt_max, dt_step, dt_min,
                                      _ptr(rows), rows.size)
    if n < 0:
        raise ValueError(f"plan rejected ({n})")
    return rows[: n + 1].copy()


def pravir_level(fmin, fmax, nchans, nsamps, dt_max, dt_step, dt_min, level):
    """(cum, dt, a, b, s) of one level of the Pravir plan (a, b, s empty at level 0)."""
    rows = int(pravir_rows(fmin, fmax, nchans, nsamps, dt_max, dt_step, dt_min)[level])
    cap = max(rows, nchans) + 1
    cum = np.zeros(cap, np.int32); dt = np.zeros(cap, np.int32)
    a = np.zeros(cap, np.int32); b = np.zeros(cap, np.int32); s = np.zeros(cap, np.int32)
    _pravir_lib().orc_pravir_level(_F(fmin), _F(fmax), nchans, nsamps, dt_max, dt_step, dt_min, level,
                                   _ptr(cum), _ptr(dt), _ptr(a), _ptr(b), _ptr(s), cap)
    return cum, dt[:rows], a[:rows], b[:rows], s[:rows]


def pravir_fdmt(fmin, fmax, x: np.ndarray, nchans, nsamps, dt_max, dt_step=1, dt_min=0,
                dtype=np.float32) -> np.ndarray:
    nout = int(pravir_rows(fmin, fmax, nchans, nsamps, dt_max, dt_step, dt_min)[-1])
    out = np.zeros((nout, nsamps), dtype)
    xin = np.ascontiguousarray(x, dtype)
    fn = _pravir_lib().orc_pravir_run_f32 if dtype == np.float32 else _pravir_lib().orc_pravir_run_f64
    if fn(_F(fmin), _F(fmax), nchans, nsamps, dt_max, dt_step, dt_min, _ptr(xin), _ptr(out)) != 0:
        raise ValueError("oracle Pravir FDMT failed")
    return out


def pravir_adjoint(fmin, fmax, gy: np.ndarray, nchans, nsamps, dt_max, dt_step=1, dt_min=0,
                   dtype=np.float32) -> np.ndarray:
    gx = np.zeros((nchans, nsamps), dtype)
    g = np.ascontiguousarray(gy, dtype)
    fn = _pravir_lib().orc_pravir_adjoint_f32 if dtype == np.float32 else _pravir_lib().orc_pravir_adjoint_f64
    if fn(_F(fmin), _F(fmax), nchans, nsamps, dt_max, dt_step, dt_min, _ptr(g), _ptr(gx)) != 0:
        raise ValueError("oracle Pravir adjoint failed")
    return gx


def ref_pravir_cpu(fmin, fmax, x: np.ndarray, nchans, nsamps, dt_max, dt_step=1, dt_min=0,
                   tsamp=1.0, threads=1) -> np.ndarray | None:
    """A fresh reference FDMTCPU(...).execute() (None if not built or it throws)."""
    r = ref_pravir_lib()
    if r is None:
        return None
    n = r.ref_pravir_rows(fmin, fmax, nchans, nsamps, tsamp, dt_max, dt_step, dt_min)
    if n < 0:
        return None
    out = np.zeros((n, nsamps), np.float32)
    xin = np.ascontiguousarray(x, np.float32)
    if r.ref_pravir_execute(fmin, fmax, nchans, nsamps, tsamp, dt_max, dt_step, dt_min, _ptr(xin), _ptr(out),
                            out.size, threads) != 0:
        return None
    return out


def ref_fdmt_cpu(fmin, fmax, x: np.ndarray | None, nchan, ncols, max_dt, b_ones=False,
                 threads=1) -> np.ndarray | None:
    """Runs the reference's CFdmtCpu::process_image (None if not built)."""
    r = ref_lib()
    if r is None:
        return None
    out = np.zeros((max_dt, ncols), np.float32)
    xin = np.ones((nchan, ncols), np.float32) if b_ones else np.ascontiguousarray(x, np.float32)
    r.ref_fdmt_cpu_process(_F(fmin), _F(fmax), nchan, ncols, max_dt, _ptr(xin), _ptr(out),
                           1 if b_ones else 0, threads)
    return out


# ---- search -----------------------------------------------------------------
def boxcar(plane: np.ndarray, thr: float, mode: int, param: int, cap: int = 1 << 22) -> np.ndarray:
    plane = np.ascontiguousarray(plane, np.float32)
    rows, cols = plane.shape
    out = np.zeros(cap, CAND_DTYPE)
    n = lib().orc_boxcar(_ptr(plane), rows, cols, _F(thr), mode, param, _ptr(out), cap)
    if n > cap:
        raise ValueError(f"oracle boxcar capacity {cap} exceeded ({n})")
    return out[:n].copy()


def boxcar_mt(plane: np.ndarray, thr: float, mode: int, param: int, cap: int = 1 << 22):
    plane = np.ascontiguousarray(plane, np.float32)
    rows, cols = plane.shape
    out = np.zeros(cap, CAND_DTYPE)
    n = lib().orc_boxcar_mt(_ptr(plane), rows, cols, _F(thr), mode, param, _ptr(out), cap)
    if n > cap:
        raise ValueError(f"oracle boxcar capacity {cap} exceeded ({n})")
    return out[:n].copy()


def norm_rows(plane: np.ndarray):
    plane = np.ascontiguousarray(plane, np.float32)
    rows, cols = plane.shape
    out = np.zeros_like(plane)
    mean = np.zeros(rows, np.float32); std = np.zeros(rows, np.float32)
    lib().orc_norm_rows(_ptr(plane), _ptr(out), rows, cols, _ptr(mean), _ptr(std))
    return out, mean, std


def cluster(cands: np.ndarray, metrics):
    cands = np.ascontiguousarray(cands, CAND_DTYPE)
    n = len(cands)
    perm = np.zeros(max(n, 1), np.int32)
    offs = np.zeros(n + 1, np.int32)
    dl = np.zeros(max(n, 1), np.int32)
    m = np.asarray(metrics, np.int32)
    g = lib().orc_cluster(_ptr(cands), n, _ptr(m), _ptr(perm), _ptr(offs), _ptr(dl))
    return perm[:n].copy(), offs[: g + 1].copy(), dl[:g].copy()


def select_delegates(cands, perm, offsets, block=64):
    cands = np.ascontiguousarray(cands, CAND_DTYPE)
    perm = np.ascontiguousarray(perm, np.int32)
    offsets = np.ascontiguousarray(offsets, np.int32)
    g = len(offsets) - 1
    out = np.zeros(max(g, 1), np.int32)
    lib().orc_select_delegates(_ptr(cands), _ptr(perm), _ptr(offsets), g, block, _ptr(out))
    return out[:g].copy()


def calc_fdmt_inputs(x: np.ndarray):
    x = np.array(x, np.float32, copy=True, order="C")
    rows, cols = x.shape
    mask = np.zeros_like(x)
    stats = np.zeros(2 * rows + 4, np.float32)
    lib().orc_calc_fdmt_inputs(_ptr(x), rows, cols, _ptr(mask), _ptr(stats))
    return x, mask, stats


def fdmt_normalize(fdmt: np.ndarray, norm: np.ndarray) -> np.ndarray:
    """fdmt / sqrtf(norm + 1e-8): the double-literal sum rounded to float first
    (L/CDMT/Chunk_gpu.cu:842-852)."""
    den = np.sqrt((norm.astype(np.float64) + 1e-8).astype(np.float32))
    return (fdmt.astype(np.float32) / den).astype(np.float32)


# --- GUPPI session geometry ---------------------------------------------------
# A restatement of CSessionB::launch's derivation (MyVSLib_C++/CDMT/
# SessionB.cpp:144-160 len_sft / overlap / chunk length, :384-392
# get_optimal_overlap, :395-401 get_coherent_dms, ChunkB.cpp:171-176 the DM
# grid).  SessionB.cpp includes <fftw3.h>, which is absent here, so the
# reference's own functions cannot be compiled: this restatement is pinned by
# hand-worked cases only.  Types follow the reference: float header fields and
# float products (np.float32), double constants, C round (half away from zero).

def _c_round(x: float) -> float:
    return float(np.copysign(np.floor(abs(x) + 0.5), x))


def _session_delay(dm: float, f_lo: np.float32, f_hi: np.float32) -> np.float32:
    lo2 = float(np.float32(f_lo * f_lo))
    hi2 = float(np.float32(f_hi * f_hi))
    return np.float32(4.148808e3 * dm * (1.0 / lo2 - 1.0 / hi2))


def session_plan(obsfreq: float, obsbw: float, nchan: int, tbin: float, t_p: float, d_min: float,
                 d_max: float, nbin: int, nfft: int) -> dict:
    f32 = np.float32
    obsfreq, obsbw, tbin, t_p = f32(obsfreq), abs(f32(obsbw)), f32(tbin), f32(t_p)
    fmin = f32(float(obsfreq) - float(obsbw) / 2.0)
    fmax = f32(float(obsfreq) + float(obsbw) / 2.0)
    len_sft = int(np.ceil(f32(t_p / tbin)))
    bw_chan = f32(obsbw / f32(nchan * len_sft))
    f_top = f32(fmin + bw_chan)
    optimal = int(_c_round(float(f32(_session_delay(d_max, fmin, f_top) / tbin))))
    half = optimal // 2
    noverlap = int(2.0 ** _c_round(np.log2(half))) if half > 0 else 0
    t_d = _session_delay(d_max, fmin, fmax)
    ncoherent = int(np.ceil(f32(f32(t_d * tbin) / f32(t_p * t_p))))
    return {"len_sft": len_sft, "noverlap": noverlap, "len_chunk": (nbin - 2 * noverlap) * nfft,
            "ncoherent": ncoherent, "optimal_overlap": optimal, "fmin": float(fmin), "fmax": float(fmax),
            "tsamp": float(tbin), "d_min": float(f32(d_min)), "d_max": float(f32(d_max))}


def coherent_dms(d_min: float, d_max: float, ncoherent: int) -> np.ndarray:
    """CChunkB's DM grid (ChunkB.cpp:171-176): step = d_max / ncoherent,
    (d_max - d_min) / step values d_min + i step (double)."""
    step = d_max / ncoherent
    n = int((d_max - d_min) / step)
    return np.array([d_min + i * step for i in range(max(n, 0))], np.float64)
