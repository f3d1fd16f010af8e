"""Seeded synthetic inputs for the beamforming path (there is no network access
for MeerKAT recordings or metadata, so these stand in for them with the same
shapes, sizes and value distributions).

* voltages: complex Gaussian, sigma per component (default 8), rounded and
  clipped to [-127, 127], TAFTP order [heap][antenna][channel][256][pol][re,im]
* optional dispersed pulse and narrowband RFI tones
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


def inject_pulse(taftp: np.ndarray, freqs: np.ndarray, tsamp: float, dm: float,
                 t0: int, width: int, amplitude: float, g: np.random.Generator) -> None:
    """Add a dispersed broadband pulse (arrival referenced to the top channel)
    in place: extra complex Gaussian power of `amplitude` sigma-units."""
    nheaps, nant, nchans = taftp.shape[:3]
    fref = freqs.max()
    for c, f in enumerate(freqs):
        delay = int(round(DM_CONST * dm * (1 / f ** 2 - 1 / fref ** 2) / tsamp))
        start = t0 + delay
        for t in range(start, start + width):
            h, s = divmod(t, 256)
            if 0 <= h < nheaps:
                extra = g.normal(0, amplitude, size=(nant, 2, 2))
                cur = taftp[h, :, c, s].astype(np.float32) + extra
                taftp[h, :, c, s] = np.clip(np.rint(cur), -127, 127).astype(np.int8)


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
