"""GPU side of the GUPPI session driver (CSession_guppi_gpu::launch): over a
synthetic GUPPI file it gives, chunk by chunk, the delegates and planes of the
chunk stage run directly on the same chunks, its images are the last chunk's
planes, and the C++ drop-in session driver writes the same images and
delegate log."""
import subprocess

import numpy as np
import pytest
import torch

from cpp_projects_b200 import guppi, synth
from cpp_projects_b200.session import CSession_guppi_gpu
from test_session import build_session_demo

pytestmark = pytest.mark.gpu

# 8 coarse channels of 4 MHz (1200..1232 MHz), TBIN 0.25 us; t_p 1.9 us gives
# len_sft 8, DM range 0..2 an overlap of 8 samples and 21 coherent DMs
T_P, D_MIN, D_MAX, SIGMA, NBIN, NFFT = 1.9e-6, 0.0, 2.0, 3.0, 4096, 2


def make_file(tmp_path):
    rng = np.random.default_rng(11)
    blocks = [rng.integers(-8, 8, (8, n, 4)).astype(np.int8) for n in (9000, 12000)]
    path = tmp_path / "s.raw"
    synth.write_guppi(path, blocks, 1216.0, 32.0, 0.25e-6, directio=1)
    return path


def log_rows(path):
    return [ln.split() for ln in path.read_text().splitlines()]


def test_session_matches_the_chunk_stage_run_directly(cuda, tmp_path):
    path = make_file(tmp_path)
    s = CSession_guppi_gpu(path, tmp_path, T_P, D_MIN, D_MAX, SIGMA, 1, NBIN, NFFT, device=cuda)
    imgs = []
    msamp = s.launch(imgs, logfile=str(tmp_path / "session.log"))
    f = guppi.GuppiFile(path)
    p = s.plan(f)
    assert (p["len_sft"], p["noverlap"]) == (8, 8)
    ch = s.createChunk(p, f.header(0))
    assert msamp == ch.get_msamp() == NFFT * (NBIN // 8 - 2)
    spec = ch.complex_buffer(cuda)
    chunks = [(b, j) for b in range(f.nblocks) for j in range(f.chunk_count(b, p["len_chunk"], p["noverlap"]))]
    assert [(b, j) for b, j, _, _ in s.results] == chunks
    planes = None
    for b, j, delegates, sizes in s.results:
        raw = torch.from_numpy(f.read_chunk(b, j, p["len_chunk"], p["noverlap"])).to(cuda)
        planes = ch.process_raw(raw, spec)
        want = ch.search(planes, None, 0.0)
        assert want is not None and len(delegates) == want.ngroups > 0
        assert np.array_equal(delegates, want.delegate_records())
        assert np.array_equal(sizes, want.group_sizes())
    ndm = len(ch.m_coh_dm_Vector)
    assert len(imgs) == ndm and imgs[0].shape == (8, msamp)
    assert np.array_equal(np.stack(imgs).view(np.uint32), planes.cpu().numpy().view(np.uint32))
    ch.search(planes, str(tmp_path / "direct.log"), 0.0)          # the last chunk's log
    assert log_rows(tmp_path / "session.log") == log_rows(tmp_path / "direct.log")


def test_cpp_session_driver_matches_the_python_session(cuda, tmp_path):
    path = make_file(tmp_path)
    exe = build_session_demo(tmp_path)
    run = tmp_path / "cpp"
    run.mkdir()
    r = subprocess.run([str(exe), str(path), str(run / "img.bin"), float(np.float32(T_P)).hex(), repr(D_MIN),
                        repr(D_MAX), repr(SIGMA), str(NBIN), str(NFFT)],
                       cwd=run, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    msamp, ndm, len_sft, noverlap, ncoherent, len_chunk = (int(v) for v in r.stdout.split())
    s = CSession_guppi_gpu(path, tmp_path, T_P, D_MIN, D_MAX, SIGMA, 1, NBIN, NFFT, device=cuda)
    p = s.plan()
    assert (len_sft, noverlap, ncoherent, len_chunk) == (p["len_sft"], p["noverlap"], p["ncoherent"],
                                                         p["len_chunk"])
    imgs = []
    assert s.launch(imgs, logfile=str(tmp_path / "py.log")) == msamp
    got = np.fromfile(run / "img.bin", np.float32).reshape(ndm, len_sft, msamp)
    assert np.array_equal(got.view(np.uint32), np.stack(imgs).view(np.uint32))
    assert log_rows(run / "candidates.log") == log_rows(tmp_path / "py.log")
