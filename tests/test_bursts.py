"""Dispersed-burst inputs of the UHF stream and the S/N measurement (CPU).

The stream's bursts are dispersed within each channel by the conjugate of the
reference's dedispersion chirp (DMResponse, CoherentDedisperser.cu:293-336)
and across channels by the cold-plasma delay; coherent dedispersion at the
burst's DM must then compact it again.  pulse_snr is the statistic the bench
applies to the GPU's and the oracle's dedispersed output alike."""
import math

import numpy as np
import pytest


def test_dispersion_response_is_the_conjugate_chirp(oracle):
    from skyweaver_b200 import synthetic
    F, n, low, bw = 8, 4096, 952e6, 8 * 0.53125e6
    for dm in (0.0, 123.4, 300.0):
        h = synthetic.dispersion_response(F, n, low, bw, dm)
        ref = oracle.chirp(F, n, low, bw, dm)
        assert np.abs(h - np.conj(ref)).max() < 1e-9


def test_pulse_train_spacing_and_ranges():
    from skyweaver_b200 import synthetic
    p = synthetic.pulse_train(synthetic.rng(3), 10, 30.0)
    t = np.array([x["t_top"] for x in p])
    assert len(p) == 10 and np.all(np.diff(t) > 1.3)
    assert t.min() >= 1.0 and t.max() <= 28.5
    for x in p:
        assert 250 <= x["dm"] <= 350 and 1e-3 <= x["width"] <= 10e-3 and 8 <= x["snr"] <= 30


def test_burst_amplitude_radiometer():
    """eps sqrt(2 N) with eps = nant amp^2 / sigma^2."""
    from skyweaver_b200 import synthetic
    amp = synthetic.burst_amplitude(20.0, 256, 1000, 64)
    eps = 64 * amp ** 2 / 64.0
    assert abs(eps * math.sqrt(2 * 256 * 1000) - 20.0) < 1e-9


def test_injected_burst_is_compact_after_coherent_dedispersion(oracle):
    """A strong burst injected on the CPU into zero voltages: per channel, the
    oracle's coherent dedispersion at the burst's DM puts nearly all of its
    power back inside the burst's width, starting where the cross-channel
    delay says (the rest is the +-1 dither of the burst's weak tails); the
    raw (dispersed) voltages spread it over the smear."""
    torch = pytest.importorskip("torch")
    from skyweaver_b200 import synthetic
    F, A, T = 4, 2, 32768
    chbw = 0.53125e6
    top = 1088e6
    bw = F * chbw
    low = float(np.float32(top - bw))
    freqs = synthetic.channel_frequencies(top - bw / 2, bw, F)
    ts = 1.0 / chbw
    dm, width = 300.0, 400 * ts
    p = [{"t_top": 20000 * ts, "dm": dm, "width": width, "snr": 4.0e4}]
    inj = synthetic.BurstInjector(torch, p, freqs, ts, low, bw, A, seed=1, device="cpu")
    taftp = torch.zeros((T // 256, A, F, 256, 2, 2), dtype=torch.int8)
    inj.inject(taftp, 0)
    v = taftp.numpy()
    assert np.abs(v).max() > 10
    # FTPA of antenna 0 -> dedisperse each channel with the oracle
    ftpa = np.ascontiguousarray(v.transpose(2, 0, 3, 4, 1, 5).reshape(F, T, 2, A, 2))
    fft_len, ov = 8192, 1024
    ext = np.concatenate([np.zeros((F, ov, 2, A, 2), np.int8), ftpa], axis=1)
    dd = oracle.cdd_ftpa(ext, T, oracle.chirp(F, fft_len, low, bw, dm), ov, lag=0)
    k = synthetic.DM_CONST
    for c in range(F):
        delay = int(round(k * dm * (1 / freqs[c] ** 2 - 1 / freqs[-1] ** 2) / ts))
        start = 20000 + delay
        pw = (dd[c].astype(np.float64) ** 2).sum(axis=(1, 2, 3))
        raw = (ftpa[c].astype(np.float64) ** 2).sum(axis=(1, 2, 3))
        inside = pw[start - 8:start + 400 + 8].sum() / pw.sum()
        raw_inside = raw[start - 8:start + 400 + 8].sum() / raw.sum()
        assert inside > 0.92, (c, inside)
        assert raw_inside < 0.5, (c, raw_inside)


def test_pulse_snr_recovers_a_boxcar():
    import bench
    g = np.random.default_rng(5)
    x = g.normal(0, 3.0, size=(40000, 3))
    x[20000:20362, 1] += 3.0 * 30.0 / math.sqrt(362)   # S/N 30 over 362 samples
    snr, j, w, st = bench.pulse_snr(x, 20181)
    assert j == 1 and 27.0 < snr < 33.0
    assert 200 <= w <= 400 and abs(st - 20000) < 80
