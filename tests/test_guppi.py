"""GUPPI RAW input: header parsing agrees with the reference's own reader
(CTelescopeHeader::readGuppiHeader, built from its source); blocks are
indexed; chunks are the per-channel strided slices with overlap (ascending
frequency, the last chunk of a block ending at its last sample); the
streaming reader returns every chunk of every block in order."""
import numpy as np
import pytest

from cpp_projects_b200 import BfsError, guppi, synth
from oracle import pyoracle

VARIANTS = [dict(directio=0, telescope="GBT", descending=False),
            dict(directio=1, telescope="GBT", descending=True),
            dict(directio=1, telescope="PARKES", descending=False),
            dict(directio=0, telescope="PARKES", descending=True)]


def _blocks(seed, n=3, nchan=4, nsamp=3000, npol=4):
    rng = np.random.default_rng(seed)
    return [rng.integers(-128, 128, (nchan, nsamp, npol)).astype(np.int8) for _ in range(n)]


@pytest.mark.parametrize("v", VARIANTS)
def test_header_matches_the_reference_reader(tmp_path, v):
    path = tmp_path / "a.raw"
    synth.write_guppi(path, _blocks(1), 1400.0, 16.0, 2.5e-7, **v)
    f = guppi.GuppiFile(path)
    assert f.nblocks == 3
    hdr_len = len(synth.guppi_header(4, 4, 3000, 1400.0, 16.0, 2.5e-7, v["directio"]))
    data_len = 48000
    if v["directio"]:  # header and data each padded to 512 bytes
        hdr_len = (hdr_len + 511) // 512 * 512
        data_len = (data_len + 511) // 512 * 512
    for b in range(f.nblocks):
        h = f.header(b)
        start = b * (hdr_len + data_len)
        assert h["data_offset"] == start + hdr_len
        ref = pyoracle.ref_guppi_header(path, start)
        if ref is None:
            pytest.skip("reference GUPPI reader not built (oracle/_ref)")
        assert ref["ok"]
        assert ref["data_pos"] == h["data_offset"]
        for k in ("nbits", "npol", "directio", "nchan", "blocsize", "telescope"):
            assert ref[k] == h[k], k
        for k in ("obsfreq", "obsbw", "tbin"):
            assert np.float32(ref[k]) == np.float32(h[k]), k
        assert np.float32(abs(ref["chan_bw"])) == np.float32(h["chan_bw"])
        assert h["straight_order"] == (ref["chan_bw"] >= 0)
        assert (h["fmin"], h["fmax"]) == (np.float32(1392.0), np.float32(1408.0))


@pytest.mark.parametrize("v", VARIANTS[:2])
@pytest.mark.parametrize("geom", [(1000, 100), (3000, 0), (777, 50), (2999, 1)])
def test_chunks_are_strided_slices_with_overlap(tmp_path, v, geom):
    L, ov = geom
    blocks = _blocks(2)
    path = tmp_path / "b.raw"
    synth.write_guppi(path, blocks, 1400.0, 16.0, 2.5e-7, **v)
    f = guppi.GuppiFile(path)
    for b in range(f.nblocks):
        n = f.chunk_count(b, L, ov)
        assert n == (3000 - 2 * ov - 1) // (L - 2 * ov) + 1
        for j in range(n):
            s0 = 3000 - L if j == n - 1 else j * (L - 2 * ov)
            assert np.array_equal(f.read_chunk(b, j, L, ov), blocks[b][:, s0:s0 + L, :])


def test_streaming_reader_order_and_contents(tmp_path):
    blocks = _blocks(3, n=4)
    path = tmp_path / "c.raw"
    synth.write_guppi(path, blocks, 1400.0, 16.0, 2.5e-7, directio=1)
    f = guppi.GuppiFile(path)
    for nbuf in (1, 2, 5):
        got = [(b, j, x.copy()) for b, j, x in guppi.GuppiReader(f, 1000, 100, nbuffers=nbuf)]
        want = [(b, j) for b in range(4) for j in range(f.chunk_count(b, 1000, 100))]
        assert [(b, j) for b, j, _ in got] == want
        assert all(np.array_equal(x, f.read_chunk(b, j, 1000, 100)) for b, j, x in got)


def test_rejections(tmp_path):
    hdr = synth.guppi_header(4, 4, 3000, 1400.0, 16.0, 2.5e-7)
    with pytest.raises(BfsError):
        guppi.parse_header(hdr.replace(b"NBITS   = 8", b"NBITS   = 4") + b"\0" * 10000)
    with pytest.raises(BfsError):
        guppi.parse_header(hdr.replace(b"'RAW     '", b"'SEARCH  '") + b"\0" * 10000)
    with pytest.raises(BfsError):
        guppi.parse_header(hdr.replace(b"TBIN", b"TBXN") + b"\0" * 10000)
    path = tmp_path / "d.raw"
    path.write_bytes(b"not a guppi file" * 100)
    with pytest.raises(BfsError):
        guppi.GuppiFile(path)
    # a truncated last block is not indexed
    synth.write_guppi(path, _blocks(4, n=2), 1400.0, 16.0, 2.5e-7)
    data = path.read_bytes()
    path.write_bytes(data[:-100])
    assert guppi.GuppiFile(path).nblocks == 1


def test_read_chunk_rejects_bad_chunking(tmp_path):
    path = tmp_path / "d.raw"
    synth.write_guppi(path, _blocks(4, n=1), 1400.0, 16.0, 2.5e-7)
    f = guppi.GuppiFile(path)
    with pytest.raises(BfsError):
        f.read_chunk(0, 0, 1000, -1)           # negative overlap
    with pytest.raises(BfsError):
        f.read_chunk(0, 0, 200, 100)           # len_chunk <= 2 * noverlap
    with pytest.raises(BfsError):
        f.read_chunk(0, 10 ** 6, 1000, 100)    # chunk past the block
    with pytest.raises(BfsError):
        f.read_chunk(1, 0, 1000, 100)          # block past the file
