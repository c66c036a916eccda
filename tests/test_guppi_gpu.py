"""GPU side of the GUPPI input: the streaming reader's pinned double buffers
copied to the device on a stream give exactly the chunks read directly, and
a GUPPI file streamed chunk by chunk through CChunk_gpu gives the same
planes as the same raw chunks handed over directly."""
import numpy as np
import pytest
import torch

from cpp_projects_b200 import guppi, synth
from cpp_projects_b200.chunk import CChunk_gpu

pytestmark = pytest.mark.gpu

GEO = dict(fmin=1200.0, fmax=1232.0, npol=4, nchan=8, len_sft=8, nbin=4096, nfft=2, noverlap=64,
           tsamp=0.25e-6, max_dt=16)


def test_device_reader_matches_direct_reads(cuda, tmp_path):
    rng = np.random.default_rng(1)
    blocks = [rng.integers(-128, 128, (8, 20000, 4)).astype(np.int8) for _ in range(3)]
    path = tmp_path / "a.raw"
    synth.write_guppi(path, blocks, 1216.0, 32.0, 0.25e-6, directio=1, descending=True)
    f = guppi.GuppiFile(path)
    s = torch.cuda.Stream()
    seen = []
    for b, j, d in guppi.GuppiReader(f, 7936, 64, nbuffers=2, device=cuda, ndevice=2, stream=s):
        s.synchronize()
        assert np.array_equal(d.cpu().numpy(), f.read_chunk(b, j, 7936, 64))
        seen.append((b, j))
    assert seen == [(b, j) for b in range(3) for j in range(f.chunk_count(b, 7936, 64))]


def test_guppi_stream_through_the_chunk_stage(cuda, tmp_path):
    g = GEO
    len_chunk = (g["nbin"] - 2 * g["noverlap"]) * g["nfft"]
    rng = np.random.default_rng(2)
    blocks = [rng.integers(-8, 8, (g["nchan"], 2 * len_chunk, g["npol"])).astype(np.int8) for _ in range(2)]
    path = tmp_path / "b.raw"
    synth.write_guppi(path, blocks, 1216.0, 32.0, g["tsamp"], directio=1)
    f = guppi.GuppiFile(path)
    h = f.header(0)
    assert (h["fmin"], h["fmax"]) == (1200.0, 1232.0)
    ch = CChunk_gpu(h["fmin"], h["fmax"], g["npol"], h["nchan"], g["len_sft"], 0, 0, 0.0, 0.0, 1, 6.0, 1,
                    g["nbin"], g["nfft"], g["noverlap"], h["tbin"], max_dt=g["max_dt"], dms=[0.0, 56.8])
    cplx = ch.complex_buffer(cuda)
    n = 0
    for b, j, d in guppi.GuppiReader(f, len_chunk, g["noverlap"], device=cuda):
        ch.unpack(d, cplx)
        got = ch.process(cplx).cpu().numpy()
        direct = torch.from_numpy(f.read_chunk(b, j, len_chunk, g["noverlap"])).to(cuda)
        ch.unpack(direct, cplx)
        want = ch.process(cplx).cpu().numpy()
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
        n += 1
    assert n == sum(f.chunk_count(b, len_chunk, g["noverlap"]) for b in range(2))
