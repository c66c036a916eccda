"""Seeded synthetic filterbanks for the search path's test and bench shapes.

No observational data ships with the repository, so every workload is
generated: i.i.d. N(0,1) float32 noise from ``numpy.random.default_rng(seed)``
plus pulses injected along the cold-plasma dispersion track
``t(f) = t0 + span * (f^-2 - fmax^-2) / (fmin^-2 - fmax^-2)``: a pulse starts
at sample ``t0`` in the highest channel and arrives ``span`` samples later in
the lowest one (the FDMT's delay convention: output row ``d`` sums channel
``c`` at sample ``t - delay_c(d)`` with delay 0 at ``fmin``).  Channel centres
are uniform: ``fmin + (c + 0.5) * (fmax - fmin) / nchan``.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


@dataclass
class Pulse:
    t0: int            # arrival sample in the highest-frequency channel
    span: float        # delay (samples) between the highest and lowest channel
    width: int         # samples
    amp: float         # added to every channel over the width


@dataclass
class Beam:
    nchan: int
    nsamp: int
    fmin: float
    fmax: float
    max_dt: int
    seed: int
    pulses: list = field(default_factory=list)
    gain: np.ndarray | None = None   # optional per-channel bandpass gain
    rfi: list = field(default_factory=list)  # (channel, cycles per sample, phase, amplitude)


def channel_centres(nchan: int, fmin: float, fmax: float) -> np.ndarray:
    return fmin + (np.arange(nchan) + 0.5) * (fmax - fmin) / nchan


def track(nchan, fmin, fmax, t0, span) -> np.ndarray:
    f = channel_centres(nchan, fmin, fmax)
    frac = (f ** -2 - fmax ** -2) / (fmin ** -2 - fmax ** -2)
    return t0 + np.rint(span * frac).astype(np.int64)


def filterbank(beam: Beam) -> np.ndarray:
    rng = np.random.default_rng(beam.seed)
    x = rng.standard_normal((beam.nchan, beam.nsamp), dtype=np.float32)
    if beam.gain is not None:
        x *= beam.gain[:, None].astype(np.float32)
    t = np.arange(beam.nsamp, dtype=np.float64)
    for c, f, ph, a in beam.rfi:
        x[c] += (a * np.sin(2 * np.pi * f * t + ph)).astype(np.float32)
    for p in beam.pulses:
        tt = track(beam.nchan, beam.fmin, beam.fmax, p.t0, p.span)
        for c in range(beam.nchan):
            a, b = int(tt[c]), int(tt[c]) + int(p.width)
            a, b = max(a, 0), min(b, beam.nsamp)
            if a < b:
                x[c, a:b] += np.float32(p.amp)
    return x


# ---- named workloads ---------------------------------------------------------
def config0(seed: int = 1) -> Beam:
    """512 ch x 32768 samples, 1200-1600 MHz, max delay 512, one pulse of width
    4 and amplitude 2.0 starting at sample 10000, track spanning 256 samples."""
    return Beam(512, 32768, 1200.0, 1600.0, 512, seed, [Pulse(10000, 256.0, 4, 2.0)])


def config4(seed: int = 4, rfi: bool = False) -> Beam:
    """1024 ch x 65536 samples, 1200-1600 MHz, max delay 1024, N(0,1) noise
    plus 8 injected pulses (the differentiable-FDMT case); with ``rfi``, 10 %
    of the channels also carry a narrowband sinusoid of amplitude 5."""
    rng = np.random.default_rng(seed)
    pulses = [Pulse(int(rng.integers(0, 60000)), float(rng.uniform(0.1, 0.9) * 1023),
                    int(rng.integers(1, 33)), float(rng.uniform(1.0, 3.0))) for _ in range(8)]
    lines = []
    if rfi:
        chans = rng.choice(1024, 102, replace=False)
        lines = [(int(c), float(rng.uniform(0.005, 0.25)), float(rng.uniform(0, 2 * np.pi)), 5.0)
                 for c in sorted(chans)]
    return Beam(1024, 65536, 1200.0, 1600.0, 1024, seed, pulses, rfi=lines)


def config3(seed: int = 3) -> Beam:
    """4096 ch x 2^17 samples, 1100-1500 MHz, max delay 4096: N(0,1) noise
    times a slow per-channel bandpass gain in [0.5, 2] (2 to the power of two
    low-order sinusoids across the band), plus 20 pulses of width 1-64,
    amplitude 1-3 and delay span 10-90 % of the max delay (the
    reduced-precision FDMT case)."""
    rng = np.random.default_rng(seed)
    nchan, nsamp = 4096, 1 << 17
    u = np.arange(nchan) / nchan
    ph = rng.uniform(0.0, 2 * np.pi, 2)
    gain = 2.0 ** (0.6 * np.sin(2 * np.pi * u + ph[0]) + 0.4 * np.sin(4 * np.pi * u + ph[1]))
    pulses = []
    for _ in range(20):
        span = float(rng.uniform(0.1, 0.9) * (nchan - 1))
        width = int(rng.integers(1, 65))
        amp = float(rng.uniform(1.0, 3.0))
        t0 = int(rng.integers(0, nsamp - int(span) - width))
        pulses.append(Pulse(t0, span, width, amp))
    return Beam(nchan, nsamp, 1100.0, 1500.0, nchan, seed, pulses, gain.astype(np.float32))


@dataclass
class VoltageChunk:
    """A GUPPI-like voltage chunk and the coherent-dedispersion geometry the
    reference's CChunkB derives from it (MyVSLib_C++/CDMT/ChunkB.h:77-98)."""
    fmin: float
    fmax: float
    npol: int          # 4 = two complex polarisations (the reference's count)
    nchan: int         # coarse channels
    len_sft: int       # fine channels per coarse channel
    nbin: int          # forward FFT length
    nfft: int          # FFTs per chunk
    noverlap: int      # overlap-save samples on each side
    tsamp: float       # coarse sample time (s) = 1 / channel bandwidth
    max_dt: int
    dm: float          # DM of the injected pulse (pc cm^-3)
    t0: int            # arrival sample of the pulse at the top of the band
    amp: float         # impulse amplitude before dispersion
    seed: int

    @property
    def len_chunk(self) -> int:
        return (self.nbin - 2 * self.noverlap) * self.nfft


def config1(seed: int = 1) -> VoltageChunk:
    """32 coarse channels of 4 MHz (1200-1328 MHz), 2 polarisations, one chunk
    of 4 x (2^20 - 2 x 8192) = 4 128 768 samples per channel (2^22 less the
    overlap), int8 uniform in [-8, 7] plus a pulse at DM 56.8; FFT length 2^20
    with 8192 samples of overlap-save on each side (the intra-channel smear at
    DM 56.8 is ~4300 samples), 32 fine channels per coarse channel (1024 in
    all), FDMT max delay 1024."""
    return VoltageChunk(1200.0, 1328.0, 4, 32, 32, 1 << 20, 4, 8192, 0.25e-6, 1024, 56.8, 1_000_000,
                        200.0, seed)


def voltage_chunk(vc: VoltageChunk, device):
    """Raw int8 chunk [nchan][len_chunk][npol] generated on the device: an
    impulse in every coarse channel at t0 plus the cold-plasma delay of the
    channel centre relative to the top of the band, dispersed inside the
    channel by the transfer function exp(2 pi i k DM f^2 / (f0^2 (f0 + f)))
    (k = 4.148808e9 MHz^2 s / (pc cm^-3) in these units), plus uniform integer
    noise in [-8, 7], rounded and clipped to int8."""
    import torch
    n = vc.len_chunk
    g = torch.Generator(device=device).manual_seed(int(vc.seed))
    raw = torch.randint(-8, 8, (vc.nchan, n, vc.npol), generator=g, device=device, dtype=torch.int16)
    bw_sub = (vc.fmax - vc.fmin) / vc.nchan
    fb = torch.fft.fftfreq(n, d=1.0, device=device, dtype=torch.float64) * bw_sub  # MHz offsets
    for c in range(vc.nchan):
        f0 = vc.fmin + bw_sub * (0.5 + c)
        delay = 4.148808e3 * vc.dm * (f0 ** -2 - vc.fmax ** -2) / vc.tsamp
        x = torch.zeros(n, dtype=torch.complex128, device=device)
        x[(vc.t0 + int(round(delay))) % n] = vc.amp
        r = fb / f0
        phase = vc.dm * r * r / (f0 + fb) * 4.148808e9
        x = torch.fft.ifft(torch.fft.fft(x) * torch.exp(2j * np.pi * phase))
        for p in range(vc.npol // 2):
            raw[c, :, 2 * p] += torch.round(x.real).to(torch.int16)
            raw[c, :, 2 * p + 1] += torch.round(x.imag).to(torch.int16)
    return raw.clamp_(-8, 7).to(torch.int8)


def guppi_header(nchan: int, npol: int, nsamp: int, obsfreq: float, obsbw: float, tbin: float,
                 directio: int = 0, telescope: str = "GBT", chan_bw: float | None = None) -> bytes:
    """A GUPPI RAW header: 80-byte "KEY     = value" cards ending with an END
    card (BACKEND and OBSEND carry the two "END"s that precede it, so the
    data start after the third, as the reference's reader expects).  The
    reader puts the data right after the letters "END"; with DIRECTIO the
    512-byte alignment covers the rest of the card, without it the card is
    written as the bare "END"."""
    chan_bw = obsbw / nchan if chan_bw is None else chan_bw

    def card(k, v):
        return f"{k:<8}= {v}".ljust(80)[:80]

    cards = [card("BACKEND", "'GUPPI   '"), card("TELESCOP", f"'{telescope}'"),
             card("OBS_MODE", "'RAW     '"), card("OBSFREQ", f"{obsfreq:.6f}"),
             card("OBSBW", f"{obsbw:.6f}"), card("OBSNCHAN", f"{nchan}"), card("CHAN_BW", f"{chan_bw:.6f}"),
             card("NPOL", f"{npol}"), card("NBITS", "8"), card("TBIN", f"{tbin:.12e}"),
             card("BLOCSIZE", f"{nchan * npol * nsamp}"), card("DIRECTIO", f"{directio}"),
             card("OBSEND", "0"), "END".ljust(80) if directio else "END"]
    return "".join(cards).encode()


def write_guppi(path, blocks: list[np.ndarray], obsfreq: float, obsbw: float, tbin: float,
                directio: int = 0, telescope: str = "GBT", descending: bool = False) -> None:
    """Writes int8 blocks [nchan][nsamp][npol] (ascending frequency) as a
    GUPPI RAW file; with ``descending`` the channels are stored from the top
    of the band down and CHAN_BW is negative."""
    with open(path, "wb") as f:
        for b in blocks:
            nchan, nsamp, npol = b.shape
            hdr = guppi_header(nchan, npol, nsamp, obsfreq, obsbw, tbin, directio, telescope,
                               -obsbw / nchan if descending else None)
            f.write(hdr)
            if directio:
                f.write(b"\0" * ((-len(hdr)) % 512))
            data = (b[::-1] if descending else b).astype(np.int8).tobytes()
            f.write(data)
            if directio:
                f.write(b"\0" * ((-len(data)) % 512))


CONFIG0_SEARCH = dict(widths_mode=0, param=5, thr=7.0, metrics=(16, 8, 1 << 30))


def config2(seed: int = 2, nbeams: int = 48, max_nchan: int = 4096) -> list[Beam]:
    """48 beams of uneven shapes: nchan from {256, 512, 1024, 4096}, lengths
    uniform in 2^14..2^17, max delay = nchan, band 1200-1600 MHz, 0-3 pulses
    of width 1-32, amplitude 1.5-4, delay span 10-90 % of the max delay."""
    rng = np.random.default_rng(seed)
    choices = [c for c in (256, 512, 1024, 4096) if c <= max_nchan]
    beams = []
    for b in range(nbeams):
        nchan = int(rng.choice(choices))
        nsamp = int(rng.integers(1 << 14, (1 << 17) + 1))
        npulse = int(rng.integers(0, 4))
        pulses = []
        for _ in range(npulse):
            span = float(rng.uniform(0.1, 0.9) * (nchan - 1))
            width = int(rng.integers(1, 33))
            amp = float(rng.uniform(1.5, 4.0))
            t0 = int(rng.integers(0, max(1, nsamp - int(span) - width)))
            pulses.append(Pulse(t0, span, width, amp))
        beams.append(Beam(nchan, nsamp, 1200.0, 1600.0, nchan, int(seed * 1000 + b), pulses))
    return beams


def manifest(beams: list[Beam]) -> list[dict]:
    return [dict(nchan=b.nchan, nsamp=b.nsamp, max_dt=b.max_dt, seed=b.seed,
                 pulses=[p.__dict__ for p in b.pulses],
                 gain=None if b.gain is None else "per-channel, [0.5, 2]") for b in beams]
