"""The fused GUPPI unpack + forward FFT of 2^20-sample segments, and the
coherent stage at the reference's FFT sizes.

CPU: an emulation of the kernels' index arithmetic (32-point decimation-in-
frequency transforms, bit reversal, the 32 x 33 exchange tile, the four-step
twiddles) against numpy's FFT.  GPU:
bfs_chunk_unpack_fft against the FP64 FFT of the oracle's unpack and against
unpack + cuFFT, the voltages against the FP64 oracle, and
bfs_chunk_process_raw against unpack + bfs_chunk_process (tolerance: 1e-5 of
the largest magnitude, the required bound for voltages; the forward FFT
itself is held to 2e-6)."""
import numpy as np
import pytest
import torch

from cpp_projects_b200.chunk import CChunk_gpu
from oracle import chunk_oracle as co

N1 = 1024


def _bitrev5(k):
    return int(f"{k:05b}"[::-1], 2)


def _dft32_dif(r):
    """The kernel's in-place radix-2 DIF over axis 0 (32 rows); X[k] = r[bitrev5(k)]."""
    r = r.astype(np.complex128).copy()
    h = 16
    while h >= 1:
        for g in range(0, 32, 2 * h):
            for j in range(h):
                a, b = r[g + j].copy(), r[g + j + h].copy()
                r[g + j] = a + b
                r[g + j + h] = (a - b) * np.exp(-2j * np.pi * (j * (16 // h)) / 32)
        h //= 2
    return r


def _fft1024_warp(v):
    """v: (1024, m) columns -> (1024, m), as one warp per column computes it."""
    m = v.shape[1]
    r = v.reshape(32, 32, m)                      # r[a][b] = v[32 a + b]
    r = _dft32_dif(r)                             # over a
    br = np.array([_bitrev5(k) for k in range(32)])
    u = r[br]                                     # u[m1][b]
    b = np.arange(32)[None, :, None]
    m1 = np.arange(32)[:, None, None]
    u = u * np.exp(-2j * np.pi * ((b * m1) % 1024) / 1024)
    tile = np.transpose(u, (1, 0, 2))             # tile[b][m1] (lane m1 reads column m1)
    r2 = _dft32_dif(tile)                         # over b
    out = r2[br]                                  # out[m2][m1] = V[m1 + 32 m2]
    return out.reshape(1024, m)


def test_four_step_index_math_matches_numpy():
    rng = np.random.default_rng(0)
    x = (rng.standard_normal(N1 * N1) + 1j * rng.standard_normal(N1 * N1))
    a = x.reshape(N1, N1)                         # a[n1][n2] = x[n1 N2 + n2]
    bmat = _fft1024_warp(a)                       # column pass over n1: b[k1][n2]
    k1 = np.arange(N1)[:, None]
    n2 = np.arange(N1)[None, :]
    bmat = bmat * np.exp(-2j * np.pi * ((n2 * k1) % (N1 * N1)) / (N1 * N1))
    rows = _fft1024_warp(bmat.T)                  # row pass over n2: rows[k2][k1]
    got = rows.reshape(-1)                        # X[k2 N1 + k1]
    want = np.fft.fft(x)
    assert np.abs(got - want).max() / np.abs(want).max() < 1e-12


GEO = dict(fmin=1200.0, fmax=1208.0, npol=4, nchan=2, len_sft=32, nbin=1 << 20, nfft=2,
           noverlap=8192, tsamp=0.25e-6, max_dt=32)


def _chunk(g, dms=(0.0,)):
    return CChunk_gpu(g["fmin"], g["fmax"], g["npol"], g["nchan"], g["len_sft"], 0, 0, 0.0, 0.0, 1,
                      6.0, 1, g["nbin"], g["nfft"], g["noverlap"], g["tsamp"], max_dt=g["max_dt"],
                      dms=list(dms))


def _raw(geo, seed):
    return np.random.default_rng(seed).integers(-8, 8, size=(geo.nchan, geo.len_chunk, geo.npol),
                                                dtype=np.int8)


@pytest.mark.gpu
@pytest.mark.parametrize("npol", [4, 2])
def test_unpack_fft_matches_fp64_and_cufft(cuda, npol):
    gd = dict(GEO, npol=npol)
    ch, g = _chunk(gd), co.Geometry(**gd)
    raw = _raw(g, 11)
    d_raw = torch.from_numpy(raw).to(cuda)
    spec = ch.complex_buffer(cuda)
    ch.unpack_fft(d_raw, spec)
    got = spec.cpu().numpy().view(np.complex64).reshape(g.npol // 2, g.nfft, g.nchan, g.nbin)
    want = np.fft.fft(co.unpack(g, raw).astype(np.complex128), axis=-1)
    scale = np.abs(want).max()
    assert np.abs(got - want).max() / scale < 2e-6
    ref = ch.complex_buffer(cuda)
    ch.unpack(d_raw, ref)
    ch.forward_fft(ref)
    ref = ref.cpu().numpy().view(np.complex64).reshape(got.shape)
    assert np.abs(got - ref).max() / scale < 2e-6
    # a second call on the same buffers gives the same bits
    ch.unpack_fft(d_raw, spec)
    assert np.array_equal(spec.cpu().numpy().view(np.complex64).reshape(got.shape), got)


@pytest.mark.gpu
@pytest.mark.parametrize("dm", [0.0, 56.8])
def test_voltages_of_2e15_subbands_within_1e5_of_fp64(cuda, dm):
    """The reference's sizes (nbin 2^20, 32 sub-bands of 2^15 samples): chirp
    + inverse FFTs against the FP64 oracle applied to the same spectra."""
    ch, g = _chunk(GEO), co.Geometry(**GEO)
    spec = ch.complex_buffer(cuda)
    ch.unpack_fft(torch.from_numpy(_raw(g, 14)).to(cuda), spec)
    volt = ch.complex_buffer(cuda)
    ch.voltages(spec, dm, volt)
    shape = (g.npol // 2, g.nfft, g.nchan, g.nbin)
    got = volt.cpu().numpy().view(np.complex64).reshape(shape)
    want = co.voltages(g, spec.cpu().numpy().view(np.complex64).reshape(shape).astype(np.complex128), dm)
    err = np.abs(got - want).max() / np.abs(want).max()
    assert err < 1e-5, err
    ch.voltages(spec, dm, volt)                   # the same bits again
    assert np.array_equal(volt.cpu().numpy().view(np.complex64).reshape(shape), got)


@pytest.mark.gpu
def test_process_raw_matches_unpack_then_process(cuda):
    ch, g = _chunk(GEO, dms=(0.0, 56.8)), co.Geometry(**GEO)
    raw = _raw(g, 12)
    d_raw = torch.from_numpy(raw).to(cuda)
    spec = ch.complex_buffer(cuda)
    got = ch.process_raw(d_raw, spec).cpu().numpy()
    cplx = ch.complex_buffer(cuda)
    ch.unpack(d_raw, cplx)
    want = ch.process(cplx).cpu().numpy()
    assert got.shape == want.shape
    assert np.abs(got - want).max() <= 1e-5 * max(1.0, np.abs(want).max())


@pytest.mark.gpu
def test_unpack_fft_other_sizes_use_unpack_and_cufft(cuda):
    gd = dict(GEO, nbin=4096, len_sft=8, noverlap=64, max_dt=8)
    ch, g = _chunk(gd), co.Geometry(**gd)
    d_raw = torch.from_numpy(_raw(g, 13)).to(cuda)
    a, b = ch.complex_buffer(cuda), ch.complex_buffer(cuda)
    ch.unpack_fft(d_raw, a)
    ch.unpack(d_raw, b)
    ch.forward_fft(b)
    assert torch.equal(a, b)


@pytest.mark.gpu
def test_unpack_fft_misaligned_raw_takes_the_unpack_path(cuda):
    """A raw chunk that does not start on a sample (npol-byte) boundary cannot
    be read as whole words: the call falls back to unpack + cuFFT."""
    ch, g = _chunk(GEO), co.Geometry(**GEO)
    raw = _raw(g, 15)
    buf = torch.zeros(raw.size + 8, dtype=torch.int8, device=cuda)
    d_raw = buf[1:1 + raw.size].view(raw.shape)
    d_raw.copy_(torch.from_numpy(raw).to(cuda))
    assert d_raw.data_ptr() % g.npol != 0
    a, b = ch.complex_buffer(cuda), ch.complex_buffer(cuda)
    ch.unpack_fft(d_raw, a)
    ch.unpack(d_raw, b)
    ch.forward_fft(b)
    assert torch.equal(a, b)
