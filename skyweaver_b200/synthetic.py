"""Seeded synthetic inputs for the beamforming path (there is no network access
for MeerKAT recordings or metadata, so these stand in for them with the same
shapes, sizes and value distributions).

* voltages: complex Gaussian, sigma per component (default 8), rounded and
  clipped to [-127, 127], TAFTP order [heap][antenna][channel][256][pol][re,im]
* narrowband RFI tones; dispersed bursts (BurstInjector, on the device)
* delay models: antenna positions uniform in a disk of `array_radius` metres,
  beam directions uniform within `fov_deg` of boresight,
  tau_ab = (x_a l_b + y_a m_b) / c, stored as float3 (weight, offset, rate)
"""
from __future__ import annotations

import numpy as np

C_LIGHT = 299792458.0
DM_CONST = 4.148806423e15  # Hz^2 pc^-1 cm^3 s


def rng(seed: int = 20261203) -> np.random.Generator:
    return np.random.default_rng(seed)


def voltages_taftp(g: np.random.Generator, nheaps: int, nant: int, nchans: int,
                   sigma: float = 8.0) -> np.ndarray:
    shape = (nheaps, nant, nchans, 256, 2, 2)
    v = np.rint(g.normal(0.0, sigma, size=shape).astype(np.float32))
    return np.clip(v, -127, 127).astype(np.int8)


def channel_frequencies(centre: float, bandwidth: float, nchans: int) -> np.ndarray:
    """PipelineConfig::calculate_channel_frequencies (PipelineConfig.cpp:188-203)."""
    chbw = bandwidth / nchans
    return centre - bandwidth / 2.0 + chbw / 2.0 + chbw * np.arange(nchans)


def inject_tones(taftp: np.ndarray, channels, amplitude: float) -> None:
    """Narrowband RFI: a coherent complex sinusoid in the given channels."""
    nheaps = taftp.shape[0]
    t = np.arange(nheaps * 256).reshape(nheaps, 256)
    for k, c in enumerate(channels):
        ph = 2 * np.pi * (0.01 + 0.037 * k) * t
        tone = np.stack([amplitude * np.cos(ph), amplitude * np.sin(ph)], -1)  # [h][s][2]
        cur = taftp[:, :, c].astype(np.float32) + tone[:, None, :, None, :]
        taftp[:, :, c] = np.clip(np.rint(cur), -127, 127).astype(np.int8)


def delay_model(g: np.random.Generator, nbeams: int, nant: int,
                array_radius: float = 4000.0, fov_deg: float = 0.5,
                antenna_weights: np.ndarray | None = None) -> np.ndarray:
    """float32 [nbeams][nant][3] = (weight, delay offset s, delay rate s/s)."""
    r = array_radius * np.sqrt(g.uniform(0, 1, nant))
    th = g.uniform(0, 2 * np.pi, nant)
    x, y = r * np.cos(th), r * np.sin(th)
    rb = np.deg2rad(fov_deg) * np.sqrt(g.uniform(0, 1, nbeams))
    tb = g.uniform(0, 2 * np.pi, nbeams)
    l, m = rb * np.cos(tb), rb * np.sin(tb)
    tau = (np.outer(l, x) + np.outer(m, y)) / C_LIGHT
    out = np.zeros((nbeams, nant, 3), np.float32)
    out[..., 0] = 1.0 if antenna_weights is None else antenna_weights
    out[..., 1] = tau.astype(np.float32)
    return out


def beamset_masks(g: np.random.Generator, nant: int, counts) -> np.ndarray:
    """Antenna weight masks (0/1) with the given number of active antennas."""
    w = np.zeros((len(counts), nant), np.float32)
    for s, k in enumerate(counts):
        w[s, g.choice(nant, size=k, replace=False)] = 1.0
    return w


# ------------------------------------------------------- dispersed bursts
def dispersion_response(nchans: int, n: int, low_freq: float, bw: float,
                        dm: float) -> np.ndarray:
    """Transfer function that disperses the baseband voltages of each channel
    by `dm`: the complex conjugate of the coherent-dedispersion chirp of the
    reference's DMResponse (CoherentDedisperser.cu:293-336) on an n-point
    window, phase +2 pi D dm nu^2 / ((nu0 + nu) nu0^2) at the non-wrapped fine
    frequency nu = k (bw / nchans) / n, with nu0 = low_freq + (c - 1/2) bw /
    nchans for channel c and dm rounded to float32 as the reference takes
    it.  complex128 [nchans][n]."""
    cbw = bw / nchans
    nu0 = low_freq + np.arange(nchans, dtype=np.float64)[:, None] * cbw - 0.5 * cbw
    nu = np.arange(n, dtype=np.float64)[None, :] * (cbw / n)
    ph = 2.0 * np.pi * DM_CONST * float(np.float32(dm)) * nu * nu / ((nu0 + nu) * nu0 * nu0)
    return np.exp(1j * ph)


def pulse_train(g: np.random.Generator, npulses: int, duration: float,
                dm_range=(250.0, 350.0), width_range=(1e-3, 10e-3),
                snr_range=(8.0, 30.0), t_first: float = 1.0,
                t_last: float = 1.5) -> list:
    """`npulses` bursts with DM, width (s) and target S/N drawn uniformly from
    the given ranges; arrival times at the top of the band (s), one in the
    first half of each of `npulses` equal slots of [t_first, duration -
    t_last], so that neighbouring bursts are at least half a slot apart."""
    edges = np.linspace(t_first, duration - t_last, npulses + 1)
    half = 0.5 * (edges[1] - edges[0])
    return [{"t_top": float(g.uniform(edges[i], edges[i] + half)),
             "dm": float(g.uniform(*dm_range)),
             "width": float(g.uniform(*width_range)),
             "snr": float(g.uniform(*snr_range))} for i in range(npulses)]


def burst_amplitude(snr: float, nchans: int, width_samples: int, nant: int,
                    sigma: float = 8.0) -> float:
    """Per-component sigma of a boresight burst (the same complex Gaussian
    signal on every antenna) for a target S/N of the dedispersed Stokes-I
    boxcar of beam 0.  The beam power of N = nchans x width_samples samples
    of 4 Gaussian components has mean 4 N s^2 and standard deviation
    s^2 sqrt(8 N) (s^2 = nant sigma^2 per beam component); the burst raises
    the mean by the fraction eps = nant amp^2 / sigma^2, so S/N = eps sqrt(2 N)
    (ignoring the incoherent-beam subtraction, which scales it by about
    sqrt(1 - 1/nant), and the int8 quantisation)."""
    eps = snr / np.sqrt(2.0 * nchans * width_samples)
    return float(sigma * np.sqrt(eps / nant))


class BurstInjector:
    """Adds dispersed bursts to TAFTP int8 gulps on the device.  Each burst is
    complex Gaussian noise (independent per pol, identical on every antenna:
    a source at boresight) over its width in every channel, dispersed within
    the channel by dispersion_response (FFT over a padded window) and across
    channels by the cold-plasma delay DM_CONST dm (1/f^2 - 1/f_top^2) from
    its arrival at the top channel.  The int8 gulp already holds rounded
    noise n; a burst value a is added as n + round(u + a) with u uniform in
    [-1/2, 1/2), which has the distribution of rounding the continuous sum
    (the burst amplitudes are a fraction of one LSB)."""

    def __init__(self, torch, pulses, freqs, tsamp, low_freq, bw, nant,
                 seed=0, sigma=8.0, device="cuda"):
        self.torch = torch
        self.nant = nant
        self.device = device
        F = len(freqs)
        gen = torch.Generator(device=device).manual_seed(seed)
        self.gen = gen
        ftop = float(np.max(freqs))
        self.segs = []
        for p in pulses:
            w = max(1, int(round(p["width"] / tsamp)))
            chbw = bw / F
            f_lo = float(np.min(freqs)) - 0.5 * chbw
            smear = int(np.ceil(DM_CONST * p["dm"] * (1 / f_lo ** 2 - 1 / (f_lo + chbw) ** 2)
                                / tsamp))
            pad = smear + 256
            L = 1 << int(np.ceil(np.log2(w + 2 * pad)))
            amp = burst_amplitude(p["snr"], F, w, nant, sigma)
            x = torch.zeros((F, 2, L), dtype=torch.complex64, device=device)
            re = torch.randn((F, 2, w), generator=gen, device=device) * amp
            im = torch.randn((F, 2, w), generator=gen, device=device) * amp
            x[:, :, pad:pad + w] = torch.complex(re, im)
            H = torch.from_numpy(dispersion_response(F, L, low_freq, bw, p["dm"]).astype(
                np.complex64)).to(device)
            x = torch.fft.ifft(torch.fft.fft(x, dim=-1) * H[:, None, :], dim=-1)
            delay = DM_CONST * p["dm"] * (1 / np.asarray(freqs) ** 2 - 1 / ftop ** 2) / tsamp
            start = np.rint(p["t_top"] / tsamp + delay).astype(np.int64) - pad
            self.segs.append((torch.from_numpy(start).to(device), L, x, int(start.min()),
                              int(start.max()) + L))

    def inject(self, taftp, first_sample, chans_per_pass=32):
        """Add the bursts that overlap the gulp starting at raw sample
        `first_sample` to int8 TAFTP [heap][antenna][channel][256][pol][re,im]
        in place."""
        torch = self.torch
        H, A, F = taftp.shape[:3]
        T = H * 256
        vv = taftp.permute(2, 0, 3, 1, 4, 5)  # [c][h][s][a][pol][ri] view
        for start, L, x, lo, hi in self.segs:
            if hi <= first_sample or lo >= first_sample + T:
                continue
            j = torch.arange(L, device=self.device)
            for c0 in range(0, F, chans_per_pass):
                c1 = min(F, c0 + chans_per_pass)
                t = start[c0:c1, None] + j[None, :] - first_sample        # [c][L]
                m = (t >= 0) & (t < T)
                if not bool(m.any()):
                    continue
                ci, ji = m.nonzero(as_tuple=True)
                tt = t[ci, ji]
                val = x[c0 + ci, :, ji]                                   # [n][pol]
                add = torch.stack([val.real, val.imag], -1)[:, None]     # [n][1][pol][ri]
                c_idx, h_idx, s_idx = c0 + ci, tt // 256, tt % 256
                cur = vv[c_idx, h_idx, s_idx].float()                     # [n][a][pol][ri]
                u = torch.rand(cur.shape, generator=self.gen, device=self.device) - 0.5
                new = (cur + torch.round(u + add)).clamp_(-127, 127).to(torch.int8)
                vv[c_idx, h_idx, s_idx] = new
