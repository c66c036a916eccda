"""Coherent-dedispersion chunk stage: the GUPPI unpack, FFTs + FP64 chirp,
the fused detect/roll/unpad/reverse/dedisperse gather and the full
CChunkB::process chain, against the FP64 oracle (oracle/chunk_oracle.py).

Tolerances: unpack and the detect gather are exact (the gather is checked on
the GPU's own voltages with the reference's float rounding of each
polarisation's power); cuFFT + chirp against FP64 numpy within 1e-5 of the
largest magnitude (the required bound: voltages within 1e-5 relative)."""
import numpy as np
import pytest
import torch

from cpp_projects_b200.chunk import CChunk_gpu, coherent_dms
from oracle import chunk_oracle as co
from oracle import pyoracle

GEO = dict(fmin=1200.0, fmax=1232.0, npol=4, nchan=8, len_sft=8, nbin=4096, nfft=2,
           noverlap=64, tsamp=0.25e-6, max_dt=16)
DM = 56.8


def _chunk():
    g = GEO
    return CChunk_gpu(g["fmin"], g["fmax"], g["npol"], g["nchan"], g["len_sft"], 0, 0, 0.0, 0.0, 1,
                      6.0, 1, g["nbin"], g["nfft"], g["noverlap"], g["tsamp"], max_dt=g["max_dt"],
                      dms=[0.0, DM])


def _geo():
    return co.Geometry(**GEO)


def _raw(seed=3):
    g = _geo()
    return np.random.default_rng(seed).integers(-8, 8, size=(g.nchan, g.len_chunk, g.npol),
                                                dtype=np.int8)


@pytest.mark.parametrize("nbin,len_sft,noverlap,nfft,nchan", [
    (64, 8, 8, 3, 2),      # mbin 8, mbin_adj 6, msamp 18 (not a multiple of 4)
    (32, 8, 8, 5, 3),      # mbin_adj 2: several (ifft, ibin) carries per thread
    (4096, 8, 64, 2, 2),   # the GPU tests' geometry
    (16, 4, 4, 7, 1),      # mbin_adj 2, msamp 14
])
def test_detect_gather_column_stepping_matches_direct_indexing(nbin, len_sft, noverlap, nfft, nchan):
    """k_detect gives each thread 4 consecutive output columns and steps the
    source column with single carries (idx wraps at msamp, ibin at mbin_adj,
    q at nbin); emulated here against the direct formula for every column,
    with shifts of both signs, and every source index checked in bounds."""
    cols_per_thread = 4
    mbin = nbin // len_sft
    nov_pc = noverlap // len_sft
    mbin_adj = mbin - 2 * nov_pc
    msamp = nfft * mbin_adj
    rows = nchan * len_sft
    npol2 = 2
    volt_len = npol2 * nfft * nchan * nbin
    pol_stride = nfft * nchan * nbin
    rng = np.random.default_rng(nbin + nfft)
    shifts = rng.integers(-3 * msamp, 3 * msamp, size=rows)
    for r in range(rows):
        isub, ifine = r // len_sft, len_sft - 1 - (r % len_sft)
        coarse = nchan - 1 - isub
        q0 = ifine * mbin + nov_pc + nbin // 2
        q0 = q0 - nbin if q0 >= nbin else q0
        for c in range(0, msamp, cols_per_thread):
            idx = int(np.fmod(c - shifts[r], msamp))   # C remainder, sign of the dividend
            if idx < 0:
                idx += msamp
            ifft, ibin = idx // mbin_adj, idx % mbin_adj
            for j in range(cols_per_thread):
                q = q0 + ibin
                q = q - nbin if q >= nbin else q
                if c + j < msamp:
                    d = (c + j - shifts[r]) % msamp
                    want = (d // mbin_adj * nchan + coarse) * nbin + \
                        (ifine * mbin + d % mbin_adj + nov_pc + nbin // 2) % nbin
                    base = (ifft * nchan + coarse) * nbin + q
                    assert base == want
                    assert 0 <= base and base + (npol2 - 1) * pol_stride < volt_len
                idx += 1
                if idx == msamp:
                    idx, ifft, ibin = 0, 0, 0
                else:
                    ibin += 1
                    if ibin == mbin_adj:
                        ibin, ifft = 0, ifft + 1


def test_coherent_dm_grid_matches_reference_rule():
    # CChunkB: step = d_max / ncoherent, count = (int)((d_max - d_min) / step)
    assert list(coherent_dms(0.0, 100.0, 4)) == [0.0, 25.0, 50.0, 75.0]
    assert list(coherent_dms(30.0, 50.0, 5)) == [30.0, 40.0]
    assert len(coherent_dms(0.0, 0.0, 3)) == 0


def test_oracle_coherent_dedispersion_compacts_a_dispersed_pulse():
    g = co.Geometry(1200.0, 1216.0, 2, 4, 4, 8192, 1, 512, 0.25e-6, 8)
    raw = co.dispersed_pulse_raw(g, 300.0, 3000, 6.0, noise=0.5)
    spec = co.forward_fft(co.unpack(g, raw))
    p_right = co.detect(g, co.voltages(g, spec, 300.0), 0.0).max()
    p_zero = co.detect(g, co.voltages(g, spec, 0.0), 0.0).max()
    assert p_right > 3 * p_zero


@pytest.mark.gpu
def test_unpack_exact(cuda):
    ch, g = _chunk(), _geo()
    raw = _raw()
    d = ch.complex_buffer(cuda)
    ch.unpack(torch.from_numpy(raw).to(cuda), d)
    got = d.cpu().numpy().view(np.complex64).reshape(g.npol // 2, g.nfft, g.nchan, g.nbin)
    np.testing.assert_array_equal(got, co.unpack(g, raw).astype(np.complex64))


@pytest.mark.gpu
@pytest.mark.parametrize("dm", [0.0, DM])
def test_voltages_within_1e5_of_fp64(cuda, dm):
    ch, g = _chunk(), _geo()
    raw = _raw()
    d = ch.complex_buffer(cuda)
    ch.unpack(torch.from_numpy(raw).to(cuda), d)
    ch.forward_fft(d)
    v = ch.complex_buffer(cuda)
    ch.voltages(d, dm, v)
    got = v.cpu().numpy().view(np.complex64).reshape(g.npol // 2, g.nfft, g.nchan, g.nbin)
    want = co.voltages(g, co.forward_fft(co.unpack(g, raw)), dm)
    err = np.abs(got - want).max() / np.abs(want).max()
    print(f"voltages dm={dm}: max |err| / max |v| = {err:.2e}")
    assert err < 1e-5


@pytest.mark.gpu
def test_detect_gather_exact_and_plane_within_1e5(cuda):
    ch, g = _chunk(), _geo()
    raw = _raw()
    d = ch.complex_buffer(cuda)
    ch.unpack(torch.from_numpy(raw).to(cuda), d)
    ch.forward_fft(d)
    v = ch.complex_buffer(cuda)
    ch.voltages(d, DM, v)
    plane = torch.empty((g.rows, g.msamp), device=cuda)
    ch.detect(v, DM, plane)
    got = plane.cpu().numpy()
    volt = v.cpu().numpy().view(np.complex64).reshape(g.npol // 2, g.nfft, g.nchan, g.nbin)
    exact = co.detect(g, volt, DM, float32_power=True)
    assert np.array_equal(got, exact)
    fp64 = co.detect(g, co.voltages(g, co.forward_fft(co.unpack(g, raw)), DM), DM)
    assert np.abs(got - fp64).max() / np.abs(fp64).max() < 1e-5


@pytest.mark.gpu
def test_process_chain_matches_oracle(cuda):
    ch, g = _chunk(), _geo()
    raw = _raw(7)
    d = ch.complex_buffer(cuda)
    ch.unpack(torch.from_numpy(raw).to(cuda), d)
    spec_copy = ch.complex_buffer(cuda)
    planes = ch.process(d)                      # overwrites d with its FFT, like the reference
    assert planes.shape == (2, g.max_dt, g.msamp)
    # oracle chain on the GPU's own detection planes
    d2 = ch.complex_buffer(cuda)
    ch.unpack(torch.from_numpy(raw).to(cuda), d2)
    ch.forward_fft(d2)
    for i, dm in enumerate([0.0, DM]):
        ch.voltages(d2, dm, spec_copy)
        plane = torch.empty((g.rows, g.msamp), device=cuda)
        ch.detect(spec_copy, dm, plane)
        x, mask, _ = pyoracle.calc_fdmt_inputs(plane.cpu().numpy())
        fd = pyoracle.fdmt_f32(g.fmin, g.fmax, x, g.rows, g.msamp, g.max_dt)
        nm = pyoracle.fdmt_f32(g.fmin, g.fmax, mask, g.rows, g.msamp, g.max_dt)
        want = pyoracle.fdmt_normalize(fd, nm)
        got = planes[i].cpu().numpy()
        assert np.abs(got - want).max() <= 1e-5 * max(1.0, np.abs(want).max())


@pytest.mark.gpu
def test_dispersed_pulse_recovered_at_its_dm(cuda):
    g = co.Geometry(1200.0, 1216.0, 2, 4, 4, 8192, 1, 512, 0.25e-6, 8)
    ch = CChunk_gpu(1200.0, 1216.0, 2, 4, 4, 0, 0, 0.0, 0.0, 1, 6.0, 1, 8192, 1, 512, 0.25e-6,
                    max_dt=8, dms=[0.0, 300.0])
    raw = co.dispersed_pulse_raw(g, 300.0, 3000, 6.0, noise=0.5)
    d = ch.complex_buffer(cuda)
    ch.unpack(torch.from_numpy(raw).to(cuda), d)
    ch.forward_fft(d)
    peaks = []
    for dm in (0.0, 300.0):
        v = ch.complex_buffer(cuda)
        ch.voltages(d, dm, v)
        plane = torch.empty((g.rows, g.msamp), device=cuda)
        ch.detect(v, 0.0, plane)
        peaks.append(float(plane.max()))
    assert peaks[1] > 3 * peaks[0]


# ---- the own sub-band transforms (mbin = 32768) --------------------------------
# geometries whose sub-bands are 32768 bins: the two-pass chirp + inverse
# transform (+ detection) of this library instead of chirp + cuFFT (+ gather)
OWN_GEOS = {
    "nbin65536": dict(fmin=1200.0, fmax=1264.0, npol=4, nchan=2, len_sft=2, nbin=65536, nfft=2, noverlap=512,
                      tsamp=1.0 / 32.0 * 1e-6, max_dt=4),
    "nbin2^20": dict(fmin=1200.0, fmax=1232.0, npol=2, nchan=1, len_sft=32, nbin=1 << 20, nfft=1,
                     noverlap=8192, tsamp=1.0 / 32.0 * 1e-6, max_dt=32),
}


def _own(name, dms=(0.0, DM)):
    g = OWN_GEOS[name]
    ch = CChunk_gpu(g["fmin"], g["fmax"], g["npol"], g["nchan"], g["len_sft"], 0, 0, 0.0, 0.0, 1, 6.0, 1,
                    g["nbin"], g["nfft"], g["noverlap"], g["tsamp"], max_dt=g["max_dt"], dms=list(dms))
    return ch, co.Geometry(**g)


def _own_spectrum(ch, g, cuda, seed=11):
    raw = np.random.default_rng(seed).integers(-8, 8, size=(g.nchan, g.len_chunk, g.npol), dtype=np.int8)
    d = ch.complex_buffer(cuda)
    ch.unpack(torch.from_numpy(raw).to(cuda), d)
    ch.forward_fft(d)
    return raw, d


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(OWN_GEOS))
def test_own_subband_voltages_within_1e5_of_fp64(cuda, name):
    ch, g = _own(name)
    raw, d = _own_spectrum(ch, g, cuda)
    v = ch.complex_buffer(cuda)
    ch.voltages(d, DM, v)     # separate buffers: the own transform
    got = v.cpu().numpy().view(np.complex64).reshape(g.npol // 2, g.nfft, g.nchan, g.nbin)
    want = co.voltages(g, co.forward_fft(co.unpack(g, raw)), DM)
    err = np.abs(got - want).max() / np.abs(want).max()
    print(f"own sub-band voltages {name}: max |err| / max |v| = {err:.2e}")
    assert err < 1e-5
    # the in-place call runs chirp + cuFFT: the same voltages to FP32 rounding
    ref = d.clone()
    ch.voltages(ref, DM, ref)
    cu = ref.cpu().numpy().view(np.complex64).reshape(g.npol // 2, g.nfft, g.nchan, g.nbin)
    assert np.abs(got - cu).max() / np.abs(cu).max() < 2e-6


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(OWN_GEOS))
def test_own_subband_detection_equals_detect_of_voltages(cuda, name):
    """The second pass's detection (roll, unpadding, reversal, shift) gives
    bit for bit the gather's plane of the voltages the same transform returns."""
    ch, g = _own(name)
    _, d = _own_spectrum(ch, g, cuda, seed=5)
    for dm in (0.0, DM):
        v = ch.complex_buffer(cuda)
        ch.voltages(d, dm, v)
        want = torch.full((g.rows, g.msamp), float("nan"), device=cuda)
        ch.detect(v, dm, want)
        got = torch.full((g.rows, g.msamp), float("nan"), device=cuda)
        ch.detect_spectrum(d, dm, got)
        assert torch.equal(got.view(torch.int32), want.view(torch.int32)), (name, dm)


@pytest.mark.gpu
def test_own_subband_process_chain_matches_oracle(cuda):
    ch, g = _own("nbin65536")
    raw = np.random.default_rng(21).integers(-8, 8, size=(g.nchan, g.len_chunk, g.npol), dtype=np.int8)
    d = ch.complex_buffer(cuda)
    ch.unpack(torch.from_numpy(raw).to(cuda), d)
    planes = ch.process(d)
    d2 = ch.complex_buffer(cuda)
    ch.unpack(torch.from_numpy(raw).to(cuda), d2)
    ch.forward_fft(d2)
    for i, dm in enumerate([0.0, DM]):
        plane = torch.empty((g.rows, g.msamp), device=cuda)
        ch.detect_spectrum(d2, dm, plane)
        x, mask, _ = pyoracle.calc_fdmt_inputs(plane.cpu().numpy())
        fd = pyoracle.fdmt_f32(g.fmin, g.fmax, x, g.rows, g.msamp, g.max_dt)
        nm = pyoracle.fdmt_f32(g.fmin, g.fmax, mask, g.rows, g.msamp, g.max_dt)
        want = pyoracle.fdmt_normalize(fd, nm)
        got = planes[i].cpu().numpy()
        assert np.abs(got - want).max() <= 1e-5 * max(1.0, np.abs(want).max())
