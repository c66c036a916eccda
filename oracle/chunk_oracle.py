"""ORACLE — test infrastructure only.

FP64 numpy restatement of the reference's coherent-dedispersion chunk stage:
  unpack       L/CDMT/Session_guppi_gpu.cu:117-141 (unpack_chunk_guppi_gpu)
  forward FFT  L/CDMT/Chunk_gpu.cu:199-205,267 (C2C, length nbin, unnormalised)
  chirp        L/CDMT/Chunk_fly_gpu.cu:94-163 (kernel_el_wise_mult_onthe_fly):
               fine-channel centre rounded to float, FP64 phase, fractional
               part (modf) to sincospi, taper 1/sqrt(1+(f/(0.47 bw))^80), 1/nbin,
               applied at the fft-shifted spectrum position
  inverse FFT  L/CDMT/Chunk_gpu.cu:208,288 (C2C, length mbin, unnormalised)
  detection    L/CDMT/Chunk_gpu.cu:476-494 (|x|^2/nbin^2 summed over pols, roll nbin/2)
  transpose    L/CDMT/Chunk_gpu.cu:497-516 (unpad, reverse the frequency axis)
  dedisperse   L/CDMT/Chunk_gpu.cu:613-632 (per-row circular shift)
(L = MyVSLib_C++).  Only tests/ use it, as the checker.
"""
from __future__ import annotations

import numpy as np


class Geometry:
    def __init__(self, fmin, fmax, npol, nchan, len_sft, nbin, nfft, noverlap, tsamp, max_dt=0):
        self.fmin, self.fmax = np.float32(fmin), np.float32(fmax)
        self.npol, self.nchan, self.len_sft = npol, nchan, len_sft
        self.nbin, self.nfft, self.noverlap = nbin, nfft, noverlap
        self.tsamp = np.float32(tsamp)
        self.mbin = nbin // len_sft
        self.nov_pc = noverlap // len_sft
        self.mbin_adj = self.mbin - 2 * self.nov_pc
        self.msamp = nfft * self.mbin_adj
        self.rows = nchan * len_sft
        self.len_chunk = (nbin - 2 * noverlap) * nfft
        self.max_dt = max_dt or len_sft


def unpack(g: Geometry, raw: np.ndarray) -> np.ndarray:
    """raw int8 [nchan][len_chunk][npol] -> complex128 [npol/2][nfft][nchan][nbin]."""
    raw = raw.reshape(g.nchan, g.len_chunk, g.npol).astype(np.float64)
    out = np.zeros((g.npol // 2, g.nfft, g.nchan, g.nbin), np.complex128)
    ibin = np.arange(g.nbin)
    for f in range(g.nfft):
        isamp = ibin + (g.nbin - 2 * g.noverlap) * f - g.noverlap
        ok = (isamp >= 0) & (isamp < g.len_chunk)
        for p in range(g.npol // 2):
            out[p, f][:, ok] = raw[:, isamp[ok], 2 * p] + 1j * raw[:, isamp[ok], 2 * p + 1]
    return out


def forward_fft(spec: np.ndarray) -> np.ndarray:
    return np.fft.fft(spec, axis=-1)


def chirp(g: Geometry, dm: float) -> np.ndarray:
    """complex128 [nchan][nbin] factor, already at the fft-shifted positions."""
    bw = np.float64(np.float32(g.fmax - g.fmin))
    bw_sub = bw / g.nchan
    bw_chan = bw_sub / g.len_sft
    out = np.zeros((g.nchan, g.nbin), np.complex128)
    ibin = np.arange(g.mbin, dtype=np.float64)
    fb = -0.5 * bw_chan + (ibin + 0.5) * bw_chan / g.mbin
    taper = 1.0 / np.sqrt(1.0 + (fb / (0.47 * bw_chan)) ** 80)
    for c in range(g.nchan):
        for s in range(g.len_sft):
            f0 = np.float64(np.float32(np.float64(g.fmin) + bw_sub * (0.5 + c)
                                       + bw_chan * (s - g.len_sft / 2.0 + 0.5)))
            r = fb / f0
            phase = dm * r * r / (f0 + fb) * 4.148808e9
            frac = -np.modf(phase)[0] * 2.0
            val = (np.cos(np.pi * frac) + 1j * np.sin(np.pi * frac)) * taper / g.nbin
            pos = (s * g.mbin + np.arange(g.mbin) + g.nbin // 2) % g.nbin
            out[c, pos] = val
    return out


def voltages(g: Geometry, spec: np.ndarray, dm: float) -> np.ndarray:
    """Chirped spectrum -> inverse FFTs of every mbin block (unnormalised)."""
    x = spec * chirp(g, dm)[None, None, :, :]
    blocks = x.reshape(x.shape[:-1] + (g.len_sft, g.mbin))
    v = np.fft.ifft(blocks, axis=-1) * g.mbin
    return v.reshape(x.shape)


def shifts(g: Geometry, dm: float) -> np.ndarray:
    fmin = np.float64(g.fmin)
    foff = (np.float64(g.fmax) - np.float64(g.fmin)) / (g.nchan * g.len_sft)
    tw = np.float64(np.float32(np.float32(g.len_sft) * g.tsamp))
    out = np.zeros(g.rows, np.int64)
    for i in range(g.rows):
        f = np.float64(g.rows - 1 - i) * foff + fmin
        d = 4.148808e3 * dm * (1.0 / (fmin * fmin) - 1.0 / (f * f))
        out[i] = int(np.floor(d / tw + 0.5)) if d / tw >= 0 else -int(np.floor(-d / tw + 0.5))
    return out


def detect(g: Geometry, volt: np.ndarray, dm: float, float32_power: bool = False) -> np.ndarray:
    """Voltages -> dedispersed fine-channel plane [rows][msamp].  With
    float32_power the per-polarisation powers are rounded to float and summed
    in float, as the reference kernel does (bit-level check of the indexing)."""
    npol2 = g.npol // 2
    if float32_power:
        p = np.zeros(volt.shape[1:], np.float32)
        for k in range(npol2):
            x = volt[k].real.astype(np.float64)
            y = volt[k].imag.astype(np.float64)
            p = (p + ((x * x + y * y) / g.nbin / g.nbin).astype(np.float32)).astype(np.float32)
    else:
        p = (np.abs(volt) ** 2).sum(axis=0) / g.nbin / g.nbin
    rolled = np.roll(p, g.nbin // 2, axis=-1)                        # [fft][chan][nbin]
    r5 = rolled.reshape(g.nfft, g.nchan, g.len_sft, g.mbin)
    seg = r5[..., g.nov_pc: g.nov_pc + g.mbin_adj]                   # unpad
    seg = seg[:, ::-1, ::-1, :]                                      # reverse coarse and fine
    plane = seg.transpose(1, 2, 0, 3).reshape(g.rows, g.msamp)
    sh = shifts(g, dm)
    out = np.empty_like(plane)
    for i in range(g.rows):
        out[i] = np.roll(plane[i], int(sh[i]))
    return out


def dispersed_pulse_raw(g: Geometry, dm: float, t0: int, amp: float, seed: int = 0,
                        noise: float = 2.0) -> np.ndarray:
    """int8 GUPPI chunk: uniform noise plus an impulse at sample t0 in every
    coarse channel, dispersed within each coarse channel by the inverse of the
    coherent chirp (so coherent dedispersion at `dm` restores an impulse)."""
    rng = np.random.default_rng(seed)
    n = g.len_chunk
    x = np.zeros((g.nchan, n), np.complex128)
    x[:, t0] = amp
    # one long FFT per coarse channel with a chirp of the same form
    bw = np.float64(np.float32(g.fmax - g.fmin))
    bw_sub = bw / g.nchan
    fb = np.fft.fftfreq(n, d=1.0) * bw_sub               # MHz offsets within the channel
    for c in range(g.nchan):
        f0 = np.float64(g.fmin) + bw_sub * (0.5 + c)
        r = fb / f0
        phase = dm * r * r / (f0 + fb) * 4.148808e9
        x[c] = np.fft.ifft(np.fft.fft(x[c]) * np.exp(2j * np.pi * phase))
    raw = np.empty((g.nchan, n, g.npol), np.int8)
    for p in range(g.npol // 2):
        re = np.clip(np.rint(x.real + rng.uniform(-noise, noise, x.shape)), -8, 7)
        im = np.clip(np.rint(x.imag + rng.uniform(-noise, noise, x.shape)), -8, 7)
        raw[:, :, 2 * p] = re
        raw[:, :, 2 * p + 1] = im
    return raw
