"""CPU side of the GUPPI session driver (CSession_guppi_gpu / CSessionB::launch):
the chunk geometry the C ABI derives from a header equals the oracle's
restatement of SessionB.cpp:144-206,384-401 over a grid of headers and
pulse lengths and a hand-worked case; bad sessions are refused; the
session's loop hands every chunk of every block, in order, to the chunk
stage (a stand-in chunk on the CPU); the C++ drop-in session driver
compiles."""
import itertools
import subprocess
from pathlib import Path

import numpy as np
import pytest
import torch

from cpp_projects_b200 import _capi, guppi, synth
from cpp_projects_b200._capi import BfsError
from cpp_projects_b200.session import CSession_guppi_gpu
from oracle import pyoracle

ROOT = Path(__file__).resolve().parent.parent
CUDA = Path("/usr/local/cuda")


def header(nchan, obsfreq, obsbw, tbin, npol=4, nsamp=1000):
    return guppi.parse_header(synth.guppi_header(nchan, npol, nsamp, obsfreq, obsbw, tbin) + b"\0" * 10000)


GRID = list(itertools.product(
    [(1264.0, 128.0, 32), (1400.0, 400.0, 64), (820.0, 200.0, 512), (150.0, 16.0, 8), (1216.0, 32.0, 8)],
    [0.25e-6, 1.0e-6, 64e-6],                      # TBIN
    [1.0, 7.9, 32.3, 200.0],                       # t_p in units of TBIN
    [(0.0, 2.0), (0.0, 56.8), (5.0, 100.0), (0.0, 1000.0)],
))


@pytest.mark.parametrize("band,tbin,tp_units,dms", GRID)
def test_session_plan_matches_oracle(band, tbin, tp_units, dms):
    obsfreq, obsbw, nchan = band
    d_min, d_max = dms
    t_p = tp_units * tbin
    h = header(nchan, obsfreq, obsbw, tbin)
    nbin, nfft = 1 << 26, 3
    want = pyoracle.session_plan(obsfreq, obsbw, nchan, h["tbin"], t_p, d_min, d_max, nbin, nfft)
    if want["len_sft"] > 1 << 20 or want["ncoherent"] > 1 << 20 or 2 * want["noverlap"] >= nbin:
        with pytest.raises(BfsError):
            guppi.session_plan(h, t_p, d_min, d_max, nbin, nfft)
        return
    got = guppi.session_plan(h, t_p, d_min, d_max, nbin, nfft)
    assert got == want


def test_session_plan_hand_worked():
    # 32 coarse channels of 4 MHz at 1200..1328 MHz, TBIN 0.25 us, t_p 7.9 us:
    #   len_sft  = ceil(7.9 / 0.25) = ceil(31.6) = 32
    #   fine channel 128 / (32 * 32) = 0.125 MHz; the delay across 1200..1200.125
    #   MHz at DM 100 is 4148.808 * 100 * (1/1200^2 - 1/1200.125^2) s = 60.02 us
    #   = 240.06 samples -> 240; half 120 -> 2^round(6.907) = 128
    #   len_chunk = (2^20 - 256) * 1
    #   whole band: 4148.808 * 100 * (1/1200^2 - 1/1328^2) = 52.86 ms;
    #   52.86 ms * 0.25 us / (7.9 us)^2 = 211.7 -> 212 coherent DMs
    h = header(32, 1264.0, 128.0, 0.25e-6)
    p = guppi.session_plan(h, 7.9e-6, 0.0, 100.0, 1 << 20, 1)
    assert (p["len_sft"], p["optimal_overlap"], p["noverlap"], p["len_chunk"], p["ncoherent"]) == \
        (32, 240, 128, (1 << 20) - 256, 212)
    assert (p["fmin"], p["fmax"]) == (1200.0, 1328.0)
    # a DM range too small for any overlap: optimal 0 -> no overlap
    p = guppi.session_plan(h, 7.9e-6, 0.0, 0.1, 1 << 20, 1)
    assert p["optimal_overlap"] == 0 and p["noverlap"] == 0 and p["len_chunk"] == 1 << 20


def test_session_plan_refusals():
    h = header(32, 1264.0, 128.0, 0.25e-6)
    for args in [(7.9e-6, 0.0, 0.0, 1 << 20, 1),      # d_max 0: the reference divides by zero
                 (0.0, 0.0, 100.0, 1 << 20, 1),       # no pulse length
                 (7.9e-6, 0.0, 100.0, 256, 1),        # 2 * noverlap >= nbin
                 (7.9e-6, 200.0, 100.0, 1 << 20, 1),  # d_min above d_max
                 (7.9e-6, 0.0, 100.0, 1 << 20, 0)]:   # no segment
        with pytest.raises(BfsError):
            guppi.session_plan(h, *args)


class _StandInChunk:
    """Records what the session hands to the chunk stage (CPU)."""

    def __init__(self, p, hdr, calls):
        self.p, self.calls = p, calls
        self.m_coh_dm_Vector = pyoracle.coherent_dms(p["d_min"], p["d_max"], p["ncoherent"])
        self.block = self.chunk = -1
        self.searched = []

    def complex_buffer(self, device):
        return torch.zeros(4, 2)

    def set_blockid(self, b):
        self.block = b

    def set_chunkid(self, j):
        self.chunk = j

    def get_msamp(self):
        return 123

    def process_raw(self, d_raw, spec, stream=None):
        self.calls.append((self.block, self.chunk, np.array(d_raw, copy=True)))
        return torch.full((len(self.m_coh_dm_Vector), 2, 3), float(len(self.calls)))

    def search(self, planes, logfile, t0):
        self.searched.append((float(planes[0, 0, 0]), logfile, t0))
        k = int(planes[0, 0, 0])
        if k % 2 == 0:
            return None                                   # no candidate passed
        return _StandInClusters(k)


class _StandInClusters:
    def __init__(self, k):
        self.k = k

    def delegate_records(self):
        c = np.zeros(self.k, pyoracle.CAND_DTYPE)
        c["mt"] = np.arange(self.k)
        return c

    def group_sizes(self):
        return np.full(self.k, 2, np.int64)


class _CpuSession(CSession_guppi_gpu):
    def __init__(self, *a, **kw):
        super().__init__(*a, **kw)
        self.calls = []

    def createChunk(self, p, hdr):
        self.chunk = _StandInChunk(p, hdr, self.calls)
        return self.chunk

    def open_reader(self, f, p, device, stream):
        return guppi.GuppiReader(f, p["len_chunk"], p["noverlap"], nbuffers=2)   # host buffers


def test_session_loop_hands_every_chunk_in_order(tmp_path):
    rng = np.random.default_rng(7)
    blocks = [rng.integers(-8, 8, (8, n, 4)).astype(np.int8) for n in (9000, 4000, 12000)]
    path = tmp_path / "s.raw"
    synth.write_guppi(path, blocks, 1216.0, 32.0, 0.25e-6, directio=1)
    s = _CpuSession(path, tmp_path, 1.9e-6, 0.0, 2.0, 3.0, 1, 4096, 2, device="cpu")
    p = s.plan()
    assert (p["len_sft"], p["noverlap"], p["len_chunk"]) == (8, 8, (4096 - 16) * 2)
    imgs = []
    assert s.launch(imgs, logfile=str(tmp_path / "c.log")) == 123
    f = guppi.GuppiFile(path)
    want = [(b, j) for b in range(3) for j in range(f.chunk_count(b, p["len_chunk"], p["noverlap"]))]
    assert [(b, j) for b, j, _ in s.calls] == want
    for b, j, data in s.calls:
        assert np.array_equal(data, f.read_chunk(b, j, p["len_chunk"], p["noverlap"]))
    assert [(b, j) for b, j, _, _ in s.results] == want
    assert s.chunk.searched == [(float(k + 1), str(tmp_path / "c.log"), 0.0) for k in range(len(want))]
    for k, (_, _, dl, sizes) in enumerate(s.results):
        n = (k + 1) if (k + 1) % 2 else 0        # odd chunks found k + 1 delegates, even ones none
        assert dl.dtype == pyoracle.CAND_DTYPE and list(dl["mt"]) == list(range(n))
        assert list(sizes) == [2] * n
    ndm = len(pyoracle.coherent_dms(p["d_min"], p["d_max"], p["ncoherent"]))
    assert len(imgs) == ndm and all(np.all(x == len(want)) for x in imgs)   # the last chunk's images


def test_session_refuses_an_empty_dm_range(tmp_path):
    path = tmp_path / "s.raw"
    synth.write_guppi(path, [np.zeros((8, 9000, 4), np.int8)], 1216.0, 32.0, 0.25e-6)
    s = _CpuSession(path, tmp_path, 1.9e-6, 2.0, 2.0, 3.0, 1, 4096, 2, device="cpu")
    with pytest.raises(ValueError):
        s.launch()


def build_session_demo(tmp: Path) -> Path:
    exe = tmp / "session_demo"
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Werror", str(ROOT / "tests/cpp/session_demo.cpp"),
           "-I", str(ROOT / "include"), "-I", str(CUDA / "include"), "-L", str(_capi.LIB_PATH.parent),
           "-lbfs_b200", "-L", str(CUDA / "lib64"), "-lcudart", f"-Wl,-rpath,{_capi.LIB_PATH.parent}",
           f"-Wl,-rpath,{CUDA / 'lib64'}", "-o", str(exe)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_cpp_session_driver_compiles(tmp_path):
    assert build_session_demo(tmp_path).exists()


def test_session_command_line_plan(tmp_path):
    import json
    import sys
    path = tmp_path / "s.raw"
    synth.write_guppi(path, [np.zeros((8, 9000, 4), np.int8)], 1216.0, 32.0, 0.25e-6)
    r = subprocess.run([sys.executable, "-m", "cpp_projects_b200.session", str(path), str(tmp_path / "out"),
                        "--t-p", "1.9e-6", "--d-max", "2", "--nbin", "4096", "--nfft", "2", "--plan-only"],
                       capture_output=True, text=True, cwd=ROOT, timeout=300)
    assert r.returncode == 0, r.stderr
    p = json.loads(r.stdout)
    assert (p["len_sft"], p["noverlap"], p["len_chunk"], p["ncoherent"]) == (8, 8, 8160, 21)


@pytest.mark.parametrize("args", [(0.0, 100.0, 212), (0.0, 1000.0, 4846), (5.0, 100.0, 7), (0.0, 2.0, 21)])
def test_coherent_dm_grid_matches_oracle_at_any_count(args):
    from cpp_projects_b200.chunk import coherent_dms
    got = coherent_dms(*args)
    want = pyoracle.coherent_dms(*args)
    assert len(got) == len(want) and np.array_equal(got, want)


def test_cpp_session_driver_control_flow_with_a_stand_in_gpu(tmp_path):
    """session_demo linked with tests/cpp/session_mock.cpp (CUDA runtime and
    GPU entries replaced by host stand-ins; file index and geometry from the
    real library): the C++ CSession_guppi_gpu reads every chunk, hands the
    last chunk's planes back per DM and writes that chunk's delegate log."""
    exe = tmp_path / "session_demo_mock"
    cmd = ["g++", "-std=c++17", "-O1", "-Wall", "-Werror", str(ROOT / "tests/cpp/session_demo.cpp"),
           str(ROOT / "tests/cpp/session_mock.cpp"), "-I", str(ROOT / "include"), "-I", str(CUDA / "include"),
           "-L", str(_capi.LIB_PATH.parent), "-lbfs_b200", f"-Wl,-rpath,{_capi.LIB_PATH.parent}",
           "-o", str(exe)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    rng = np.random.default_rng(11)
    blocks = [rng.integers(-8, 8, (8, n, 4)).astype(np.int8) for n in (9000, 12000)]
    path = tmp_path / "s.raw"
    synth.write_guppi(path, blocks, 1216.0, 32.0, 0.25e-6, directio=1)
    run = tmp_path / "run"
    run.mkdir()
    t_p = float(np.float32(1.9e-6)).hex()
    r = subprocess.run([str(exe), str(path), str(run / "img.bin"), t_p, "0.0", "2.0", "3.0", "4096", "2"],
                       cwd=run, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    msamp, ndm, len_sft, noverlap, ncoherent, len_chunk = (int(v) for v in r.stdout.split())
    f = guppi.GuppiFile(path)
    p = guppi.session_plan(f.header(0), 1.9e-6, 0.0, 2.0, 4096, 2)
    assert (len_sft, noverlap, ncoherent, len_chunk) == (p["len_sft"], p["noverlap"], p["ncoherent"],
                                                         p["len_chunk"])
    assert ndm == len(pyoracle.coherent_dms(p["d_min"], p["d_max"], p["ncoherent"]))
    assert msamp == 2 * (4096 // len_sft - 2 * (noverlap // len_sft))
    # the stand-in planes of the last chunk
    last = (f.nblocks - 1, f.chunk_count(f.nblocks - 1, len_chunk, noverlap) - 1)
    s = int(f.read_chunk(*last, len_chunk, noverlap).astype(np.int64).sum())
    i, rr, t = np.meshgrid(np.arange(ndm), np.arange(len_sft), np.arange(msamp), indexing="ij")
    want = ((s + 7 * i + 3 * rr + t) % 97).astype(np.float32)
    got = np.fromfile(run / "img.bin", np.float32).reshape(ndm, len_sft, msamp)
    assert np.array_equal(got, want)
    # one candidate per plane row at its first maximum, each its own group, sorted by mt
    flat = want.reshape(ndm * len_sft, msamp)
    mt = flat.argmax(axis=1)
    order = np.argsort(mt, kind="stable")
    rows = [ln.split() for ln in (run / "candidates.log").read_text().splitlines()]
    assert rows[0] == ["N", "t,", "bin", "t,", "sec", "dedisp", "width", "SNR", "num"]
    assert len(rows) == 1 + len(order)
    delt_bin = np.float32(np.float32(p["tsamp"]) * np.float32(len_sft))
    for k, row in enumerate(order):
        n_, t_bin, t_sec, dedisp, width, snr, num = rows[1 + k]
        assert (int(n_), int(t_bin), int(dedisp), int(width), float(snr), int(num)) == \
            (k + 1, int(mt[row]), int(row), 1, 96.0, 1)
        assert abs(float(t_sec) - float(np.float32(mt[row]) * delt_bin)) <= 1e-6 * max(1.0, float(t_sec))
