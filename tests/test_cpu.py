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


def test_output_description_follows_described_vector():
    """stages.describe: the DescribedVector metadata of a pipeline output
    (DescribedVector.hpp:96-573, CoherentBeamformer.cu:235,
    CoherentDedisperser.cu:82,224, PipelineConfig.cpp:188-203)."""
    from skyweaver_b200 import stages
    d = stages.describe("TFB", (4096, 64, 1024), 1284e6, 64 * 856e6 / 1024, 64, 16, 1472, 150.0)
    chbw = 856e6 / 1024
    assert d["dims"] == "TFB" and d["extents"] == (4096, 64, 1024)
    assert len(d["frequencies"]) == 64
    assert abs(d["frequencies"][0] - (1284e6 - 32 * chbw + chbw / 2)) < 1e-3
    assert abs(d["frequencies"][63] - (1284e6 + 32 * chbw - chbw / 2)) < 1e-3
    assert abs(d["tsamp"] - 16 / chbw) < 1e-15
    assert abs(d["utc_offset"] - 736 / chbw) < 1e-15
    assert d["reference_dm"] == 150.0 and d["dms"] == []
