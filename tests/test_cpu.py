"""CPU tests (no GPU): the oracle pinned to the reference's golden vectors
and known answers, the C ABI library loading and exporting every symbol that
include/skyweaver_b200.h declares, and the host-side planning logic."""
import hashlib
import json
import math
import os
import re

import numpy as np
import pytest

from conftest import GOLDEN, REPO


def test_golden_manifest():
    with open(os.path.join(GOLDEN, "MANIFEST.json")) as f:
        man = json.load(f)
    for name, meta in man.items():
        with open(os.path.join(GOLDEN, name), "rb") as f:
            assert hashlib.sha256(f.read()).hexdigest() == meta["sha256"], name


def test_oracle_coherent_dedispersion_golden_bit_exact(oracle):
    """The FP64 oracle reproduces the reference's golden vector exactly
    (codedisp_output_DM1000_1chan.bin; CoherentDedisperserTester.cu:113-204)."""
    inp = np.fromfile(os.path.join(GOLDEN, "codedisp_input_DM1000_1chan.bin"),
                      np.int8).reshape(1024, 2, 64, 2)
    want = np.fromfile(os.path.join(GOLDEN, "codedisp_output_DM1000_1chan.bin"),
                       np.int8).reshape(446, 2, 64, 2)
    tsamp = 4096 / 856e6
    ov = math.ceil(oracle.dm_delay(856e6, 856e6 + 856e6 / 4096, 1000.0) / tsamp)
    assert ov == 578
    ch = oracle.chirp(64, 1024, 856e6, 13.375e6, 1000.0)
    got = np.stack([np.stack([oracle.cdd_segment(inp[:, p, a], ch[0], ov)
                              for a in range(64)], 1) for p in range(2)], 1)
    assert np.array_equal(got, want)
    # the golden output has int8 wrap-around (the reference's static_cast<char>)
    _, f64 = oracle.cdd_segment(inp[:, 0, 0], ch[0], ov, want_f64=True)
    assert np.abs(f64.real).max() > 127 or np.abs(f64.imag).max() > 127


def test_oracle_dm0_identity(oracle):
    """DM 0 coherent dedispersion is the identity (CoherentDedisperserTester.cu:69-111)."""
    g = np.random.default_rng(0)
    x = np.clip(np.rint(g.normal(0, 17, (1024, 2))), -127, 127).astype(np.int8)
    ch = oracle.chirp(1, 1024, 856e6, 13.375e6, 0.0)
    out = oracle.cdd_segment(x, ch[0], 578)
    assert np.array_equal(out, x[289:289 + 446])


def test_oracle_chirp_multiply_matches_reference_formula(oracle):
    # DMResponse: phase = nu^2 * pref / ((nu0 + nu) * nu0^2), nu0 = low + c*cbw - cbw/2
    ch = oracle.chirp(2, 16, 856e6, 13.375e6, 100.0)
    cbw = 13.375e6 / 2
    nu0 = 856e6 + 1 * cbw - 0.5 * cbw
    nu = 5 * cbw / 16
    pref = -2 * math.pi * 4.148806423e15 * 100.0
    ph = nu * nu * pref / ((nu0 + nu) * nu0 * nu0)
    assert abs(ch[1, 5] - complex(math.cos(ph), math.sin(ph))) < 1e-12


def test_oracle_idd_known_answers(oracle):
    """IncoherentDedisperserTester.cu:39-126: zero-DM delays, all-ones input."""
    freqs = 580e6 - 16e6 + 0.25e6 + 0.5e6 * np.arange(64)
    d0, m0 = oracle.idd_delays(freqs, [0.0], 16 / 0.5e6)
    assert m0 == 0 and not d0.any()
    dms = [0.0, 10.0, 20.0, 30.0, 40.0]
    delays, maxd = oracle.idd_delays(freqs, dms, 16 / 0.5e6)
    assert maxd > 0
    for ts in (1, 2):
        T = 3 * maxd
        T -= (T - maxd) % ts
        out = oracle.idd(np.ones((T, 64, 32), np.int8), delays, maxd, ts,
                         np.float32(math.sqrt(64 * ts)))
        assert np.all(out == int(math.sqrt(64 * ts)))
    with pytest.raises(RuntimeError):  # too_few_samples_test
        oracle.idd(np.ones((maxd, 64, 32), np.int8), delays, maxd, 1, np.float32(8.0))


def test_oracle_weights_known_answers(oracle):
    """Zero delay -> (127, 0) for unit antenna weight (WeightsManagerTester.cu:99-112)."""
    d = np.tile(np.array([1.0, 0.0, 0.0], np.float32), (4, 8, 1))
    w = oracle.weights(d, np.array([1e9, 1.1e9]), 10.0, 9.0)
    assert np.all(w[..., 0] == 127) and np.all(w[..., 1] == 0)


def test_oracle_transpose_and_stats(oracle):
    g = np.random.default_rng(1)
    taftp = g.integers(-100, 100, size=(2, 3, 4, 256, 2, 2), dtype=np.int8)
    ftpa = oracle.transpose(taftp, 8)
    assert ftpa.shape == (4, 512, 2, 8, 2)
    assert np.array_equal(ftpa[2, 256 + 7, 1, 1], taftp[1, 1, 2, 7, 1])
    assert not ftpa[:, :, :, 3:].any()
    st = oracle.statistics(ftpa[:, :, :, :3])
    x = np.concatenate([ftpa[0, :, 1, 2, 0], ftpa[0, :, 1, 2, 1]]).astype(np.float64)
    assert abs(st[0, 1, 2, 0] - x.mean()) < 1e-5
    assert abs(st[0, 1, 2, 1] - x.std(ddof=1)) / x.std() < 1e-6


def test_delay_file_fixture_layout():
    """test_delays.bin: 5 models x (24-byte header + 67 x 57 float3)
    (DelayManagerTester.cu:38-52; DelayModel.to_bytes, skyweaver.py:77-90)."""
    from skyweaver_b200 import delays
    models = delays.read_delay_file(os.path.join(GOLDEN, "test_delays.bin"))
    assert len(models) == 5
    for m in models:
        assert m.delays.shape == (67, 57, 3)
        assert m.end_epoch > m.start_epoch
    assert abs(models[0].start_epoch - 1708082168.957) < 1e-3
    sets = delays.parse_beamsets(models[0].delays, nbeams=96, nantennas=64)
    assert sets.nbeamsets == 2


def test_delay_manager_epochs_and_beamsets():
    """DelayManagerTester.cu:54-92 on the same file: reads in the first and the
    nth validity window give nbeams x nantennas delays (padded with zeros
    past the model's 67 beams x 57 antennas), an epoch before the first
    window raises InvalidDelayEpoch, one after the last window raises
    RuntimeError, and the file holds 2 beamsets."""
    from skyweaver_b200 import delays
    path = os.path.join(GOLDEN, "test_delays.bin")
    models = delays.read_delay_file(path)
    dm = delays.DelayManager(path, nbeams=96, nantennas=64)
    first = dm.delays(1708082169.0)
    assert first.shape == (96, 64, 3)
    assert np.array_equal(first[:67, :57], models[0].delays)
    assert not first[67:].any() and not first[:, 57:].any()
    nth = dm.delays(1708082409.957)
    k = next(i for i, m in enumerate(models) if m.start_epoch <= 1708082409.957 <= m.end_epoch)
    assert k > 0 and np.array_equal(nth[:67, :57], models[k].delays)
    assert abs(models[-1].end_epoch - 1708082468.957) < 1e-3
    assert dm.nbeamsets() == 2
    with pytest.raises(delays.InvalidDelayEpoch):
        delays.DelayManager(path, nbeams=96, nantennas=64).delays(1708082165.0)
    with pytest.raises(RuntimeError):
        delays.DelayManager(path, nbeams=96, nantennas=64).delays(1708082470.957)
    with pytest.raises(RuntimeError, match="too many beams"):
        delays.DelayManager(path, nbeams=64, nantennas=64)


def _declared_functions():
    with open(os.path.join(REPO, "include", "skyweaver_b200.h")) as f:
        txt = f.read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(sw_[a-z0-9_]+)\s*\(", txt)))


def test_c_abi_exports_every_declared_symbol():
    import ctypes
    from skyweaver_b200 import _lib
    if not os.path.exists(_lib.LIB_PATH):
        from skyweaver_b200 import build
        build.build()
    L = ctypes.CDLL(_lib.LIB_PATH)
    names = _declared_functions()
    assert len(names) > 20
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    assert L.sw_version() >= 100


def test_c_abi_rejects_bad_arguments_without_gpu():
    from skyweaver_b200 import _lib
    L = _lib.lib()
    assert L.sw_transpose_ftpa(None, None, 1, 1, 1, 1, None) == 1
    assert b"null" in L.sw_last_error()
    assert L.sw_cdd_setup_bytes(1, 1, 1000) == 0      # not a power of two
    assert L.sw_cdd_setup_bytes(2, 4, 4096) > 2 * 4 * 4096 * 8
    # argument checks run on the host before any launch, so stand-in device
    # addresses are never dereferenced
    import ctypes
    fake = ctypes.c_void_p(0x10000)
    # incoherent beam, 4-byte loads (tscrunch 16): misaligned voltage pointer
    rc = L.sw_incoherent_beamform(ctypes.c_void_p(0x10001), 64, 0, 1, 64, 16, 16, fake, fake,
                                  fake, 1, 0, fake, fake, None)
    assert rc == 1 and b"multiples of 4" in L.sw_last_error()
    # coherent dedispersion: the lag must lie in [0, overlap]
    outs = (ctypes.c_void_p * 1)(0x20000)
    rc = L.sw_coherent_dedisperse_ws(fake, 4096, 1, 2, 4, 2048, 1024, 256, 300, fake, 1, outs,
                                     2048, None, 0, None, None)
    assert rc == 1 and b"lag" in L.sw_last_error()
    # coherent beamformer pipeline depths outside 2..8 / 2..3
    shape = _lib.CbShape(1, 64, 16, 128, 4, 0, 1, 64, 0, 0, 9, 2)
    prob = _lib.CbProblem(0x10000, 0x20000, 0x30000, 0, 128)
    rc = L.sw_coherent_beamform(ctypes.byref(shape), ctypes.byref(prob), fake, fake, fake, fake,
                                None, None)
    assert rc == 1 and b"stages" in L.sw_last_error()


def test_output_description_follows_described_vector():
    """stages.describe: the DescribedVector metadata of a pipeline output
    (DescribedVector.hpp:96-573, CoherentBeamformer.cu:235,
    CoherentDedisperser.cu:82,224, PipelineConfig.cpp:188-203)."""
    from skyweaver_b200 import stages
    d = stages.describe("TFB", (4096, 64, 1024), 1284e6, 64 * 856e6 / 1024, 64, 16, 128, 150.0)
    chbw = 856e6 / 1024
    assert d["dims"] == "TFB" and d["extents"] == (4096, 64, 1024)
    assert len(d["frequencies"]) == 64
    assert abs(d["frequencies"][0] - (1284e6 - 32 * chbw + chbw / 2)) < 1e-3
    assert abs(d["frequencies"][63] - (1284e6 + 32 * chbw - chbw / 2)) < 1e-3
    assert abs(d["tsamp"] - 16 / chbw) < 1e-15
    assert abs(d["utc_offset"] - 128 / chbw) < 1e-15
    assert d["reference_dm"] == 150.0 and d["dms"] == []


# ------------------------------------------------ overlap-save plan (host)
C1_BAND = dict(centre=1284e6, chbw=856e6 / 1024, nchans=64, dms=[0.0, 50.0, 150.0, 500.0])


def test_cdd_plan_matches_restatement_and_rejects_impossible(oracle):
    """sw_cdd_plan (host only, no GPU) against the oracle's restatement of the
    plan, over bands, DM sets and requested lags and FFT lengths."""
    from skyweaver_b200 import stages
    O = oracle
    for centre, nch, dms in ((1284e6, 64, [0, 50, 150, 500]), (1284e6, 4, [0, 10]),
                             (1088e6 - 8 * 0.53125e6, 16, [0, 300]),
                             (1284e6, 64, [2000.0]), (600e6, 8, [0.0])):
        chbw = 856e6 / 1024 if centre == 1284e6 else 0.53125e6
        for lag in (0, 64, 100, 256):
            for n in (0, 8192, 65536):
                want = O.cdd_plan(centre, nch * chbw, nch, dms, n, lag or 128)
                if want[0] <= want[1]:
                    with pytest.raises(RuntimeError):
                        stages.cdd_plan(centre, nch * chbw, nch, dms, n, lag)
                    continue
                assert stages.cdd_plan(centre, nch * chbw, nch, dms, n, lag) == want
    # C1 at DM 500: 1458-sample smear -> head 1472, lag 128, 8192-point windows
    assert stages.cdd_plan(1284e6, 64 * 856e6 / 1024, 64, [0, 50, 150, 500]) == (8192, 1600, 128)


def test_chirp_response_is_causal_within_the_head_trim(oracle):
    """Why the plan trims the smear at the window start: the reference chirp's
    impulse response (DMResponse, CoherentDedisperser.cu:313-335) holds at
    least 97% of its energy at causal lags 0 .. head, and its anti-causal
    part beyond the plan's lag is small."""
    from skyweaver_b200 import stages
    b = C1_BAND
    bw = b["nchans"] * b["chbw"]
    low = float(np.float32(b["centre"] - bw / 2))
    n, ov, lag = stages.cdd_plan(b["centre"], bw, b["nchans"], b["dms"])
    head = ov - lag
    for dm in (50.0, 150.0, 500.0):
        ch = oracle.chirp(b["nchans"], n, low, bw, dm)
        for c in (0, 32, 63):
            e = np.abs(np.fft.ifft(ch[c])) ** 2
            e /= e.sum()
            assert e[:head + 1].sum() > 0.97, (dm, c, e[:head + 1].sum())
            assert e[n - 1024:n - lag].sum() < 2e-3, (dm, c)


def _long_window(x, chirp, trim):
    """Overlap-save with a long window and a large symmetric trim: the
    wrap-free result the plan is compared with (FP64, numpy)."""
    n = len(chirp)
    hop = n - 2 * trim
    y = np.full(len(x), np.nan + 0j)
    s = 0
    while s + n <= len(x):
        z = np.fft.ifft(np.fft.fft(x[s:s + n]) * chirp)
        y[s + trim:s + n - trim] = z[trim:n - trim]
        s += hop
    return y


def _stream_plan(oracle, xr, gulp, chirp, overlap, lag):
    hist = np.zeros((overlap, 2), np.int8)
    outs = []
    for g in range(len(xr) // gulp):
        cur = xr[g * gulp:(g + 1) * gulp]
        outs.append(oracle.cdd_stream(np.concatenate([hist, cur]), gulp, chirp, overlap, lag=lag))
        hist = cur[gulp - overlap:]
    return np.concatenate(outs)


def test_plan_is_wrap_free_where_the_symmetric_trim_wraps(oracle):
    """The headline band's DM 500 on its lowest channel, three 65536-sample
    gulps through the overlap-save stream of the oracle: the pipeline's plan
    (8192-point windows, trims 1472 + 128) stays within 2 LSB of a
    65536-point window with 16384-sample trims everywhere, while trimming the
    same overlap symmetrically (736 + 736, the reference's per-window trim at
    the smear-sized overlap) wraps the causal response and is off by tens of
    LSB.  The residual one-LSB differences come from the reference chirp's
    phase jump at the bin wrap, whose 1/n tails make every plan's output
    depend on its window geometry."""
    from skyweaver_b200 import stages
    b = C1_BAND
    bw = b["nchans"] * b["chbw"]
    low = float(np.float32(b["centre"] - bw / 2))
    n, ov, lag = stages.cdd_plan(b["centre"], bw, b["nchans"], b["dms"])
    G = 65536
    g = np.random.default_rng(7)
    xr = np.clip(np.rint(g.normal(0, 8, (3 * G, 2))), -127, 127).astype(np.int8)
    x = xr[:, 0] + 1j * xr[:, 1].astype(np.float64)
    yl = _long_window(x, oracle.chirp(b["nchans"], 65536, low, bw, 500.0)[0], 16384)
    sl = np.arange(16384 + G // 2, 3 * G - 32768)
    want = np.rint(np.stack([yl[sl].real, yl[sl].imag], -1).astype(np.float32))
    want = (want + 128) % 256 - 128
    ch = oracle.chirp(b["nchans"], n, low, bw, 500.0)[0]
    for o_lag, bound in ((lag, 2), (ov // 2, None)):
        got = _stream_plan(oracle, xr, G, ch, ov, o_lag)[sl + o_lag].astype(np.float64)
        d = np.abs(got - want)
        d = np.minimum(d, 256 - d)
        print(f"lag {o_lag}: {np.mean(d > 0):.3%} of values differ, max {d.max():.0f} LSB")
        if bound is None:
            assert d.max() > 10
        else:
            assert d.max() <= bound and np.mean(d > 0) < 0.08
