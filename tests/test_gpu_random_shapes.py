"""Seeded random shapes through the CUDA stages against the oracle: beam,
channel and antenna counts, tscrunch, Stokes modes, beamset masks and
mappings, trial DMs and scale factors drawn at random, so that combinations
the hand-written cases do not name (a partial beam block with full Stokes at
tscrunch 1, fractional beamset weights on the incoherent beam, odd channel
counts in the dedisperser) are checked too.  Every draw is fixed by its seed;
the tolerances are the ones the per-stage tests use: bit-exact for the
beamformers and the incoherent dedisperser, 1e-5 relative for the statistics.
"""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

STOKES = ["I", "Q", "U", "V", "IQUV"]


def _dev(cuda, a):
    return cuda.from_numpy(np.ascontiguousarray(a)).cuda()


def _np(t):
    return t.cpu().numpy()


@pytest.mark.parametrize("seed", range(24))
def test_random_coherent_beam(cuda, oracle, seed):
    """CoherentBeamformerTester.cu:43-152 on a random shape: int32 beam
    voltages and the int8 TFB identical to the oracle."""
    from skyweaver_b200 import stages, synthetic
    g = synthetic.rng(9000 + seed)
    A = int(g.choice([16, 32, 64]))
    B = int(g.integers(1, 321))
    F = int(g.integers(1, 5))
    H = int(g.integers(1, 4))
    T = 256 * H
    ts = int(g.choice([1, 2, 4, 8, 16, 32]))
    stokes = STOKES[int(g.integers(0, 5))]
    ib_sub = bool(g.integers(0, 2))
    S = int(g.integers(1, 4))
    taftp = synthetic.voltages_taftp(g, H, A, F, sigma=float(g.uniform(8, 40)))
    ftpa = oracle.transpose(taftp, A)
    th = g.uniform(0, 2 * np.pi, size=(F, B, A))
    amp = g.integers(1, 128, size=(F, B, A))
    w = np.stack([np.rint(amp * np.cos(th)), np.rint(amp * np.sin(th))], -1).astype(np.int8)
    bw = synthetic.beamset_masks(g, A, [int(g.integers(1, A + 1)) for _ in range(S)])
    mapping = g.integers(0, S, size=B).astype(np.int32)
    level = 32.0
    dof = 2 * ts * 2
    cb_scale = (127 * level * math.sqrt(A)) ** 2
    scales = (cb_scale * math.sqrt(2 * dof) / level *
              g.uniform(0.5, 2.0, size=S * F)).astype(np.float32)
    offsets = (cb_scale * dof * g.uniform(0.5, 2.0, size=S * F)).astype(np.float32)
    ib_s = np.full(S * F, 1e4, np.float32)
    fp = stages.transpose_fpact(_dev(cuda, taftp), A)
    raw_ib, _ = stages.incoherent_beamform(fp, T, ts, _dev(cuda, ib_s), _dev(cuda, ib_s),
                                           _dev(cuda, bw), stokes=stokes)
    out, dbg = stages.coherent_beamform(fp, stages.pack_weights(_dev(cuda, w)),
                                        _dev(cuda, scales), _dev(cuda, offsets),
                                        _dev(cuda, mapping), raw_ib, T, ts, stokes=stokes,
                                        ib_subtract=ib_sub, debug=True)
    ref, volts = oracle.coherent_beam(ftpa, w, ts, scales, offsets, bw, mapping, stokes,
                                      ib_sub, want_voltages=True)
    case = dict(A=A, B=B, F=F, T=T, ts=ts, stokes=stokes, ib_sub=ib_sub, beamsets=S)
    assert np.array_equal(_np(dbg), volts), case
    got = _np(out)
    assert np.array_equal(got, ref), (case, int((got != ref).sum()))


@pytest.mark.parametrize("seed", range(16))
def test_random_incoherent_beam(cuda, oracle, seed):
    """IncoherentBeamformerTester.cu:41-103 on a random shape, with 0/1 masks
    (the exact integer path) or fractional weights (the reference-order float
    chain): raw powers and int8 output bit-identical."""
    from skyweaver_b200 import stages, synthetic
    g = synthetic.rng(9100 + seed)
    A = int(g.integers(1, 65))
    F = int(g.integers(1, 6))
    H = int(g.integers(1, 3))
    T = 256 * H
    ts = int(g.choice([1, 2, 4, 8, 16, 32]))
    stokes = STOKES[int(g.integers(0, 5))]
    S = int(g.integers(1, 5))
    if seed % 2:
        bw = g.uniform(0.0, 1.5, size=(S, A)).astype(np.float32)
    else:
        bw = synthetic.beamset_masks(g, A, [int(g.integers(1, A + 1)) for _ in range(S)])
    taftp = synthetic.voltages_taftp(g, H, A, F, sigma=float(g.uniform(8, 60)))
    ftpa = oracle.transpose(taftp, A)
    scale = g.uniform(1e2, 1e4, size=S * F).astype(np.float32)
    offset = g.uniform(0, 1e5, size=S * F).astype(np.float32)
    fp = stages.transpose_fpact(_dev(cuda, taftp), A)
    raw, out = stages.incoherent_beamform(fp, T, ts, _dev(cuda, scale), _dev(cuda, offset),
                                          _dev(cuda, bw), stokes=stokes)
    raw_ref, out_ref = oracle.incoherent_beam(ftpa, ts, scale, offset, bw, S, stokes)
    case = dict(A=A, F=F, T=T, ts=ts, stokes=stokes, beamsets=S, fractional=bool(seed % 2))
    assert np.array_equal(_np(raw).view(np.uint32), raw_ref.view(np.uint32)), case
    assert np.array_equal(_np(out), out_ref), case


@pytest.mark.parametrize("seed", range(12))
def test_random_incoherent_dedispersion(cuda, oracle, seed):
    """IncoherentDedisperser.cu:66-125 on a random shape: TDB identical."""
    from skyweaver_b200 import stages, synthetic
    g = synthetic.rng(9200 + seed)
    F = int(g.integers(1, 80))
    B = 4 * int(g.integers(1, 150))
    ts = int(g.choice([1, 2, 3, 4, 8]))
    ndms = int(g.integers(1, 40))
    chbw = 856e6 / 1024
    freqs = synthetic.channel_frequencies(1284e6, F * chbw, F)
    dms = np.sort(g.uniform(0, 300, size=ndms)).astype(np.float32)
    delays, maxd = oracle.idd_delays(freqs, dms, ts * 16 / chbw)
    nout = int(g.integers(1, 48))
    T = maxd + nout * ts
    tfb = g.integers(-128, 128, size=(T, F, B), dtype=np.int8)
    sf = np.float32(g.uniform(0.5, 2.0) * math.sqrt(F * ts))
    ref = oracle.idd(tfb, delays, maxd, ts, sf)
    got = _np(stages.incoherent_dedisperse(_dev(cuda, tfb), _dev(cuda, delays), maxd, ts,
                                           float(sf)))
    assert np.array_equal(got, ref), dict(F=F, B=B, ts=ts, ndms=ndms, nout=nout, maxd=maxd)


@pytest.mark.parametrize("seed", range(8))
def test_random_transpose_statistics(cuda, oracle, seed):
    """Transposer + StatisticsCalculator in one pass on a random shape: FPACT
    bytes exact, statistics within 1e-5 relative, padded antennas zero."""
    from skyweaver_b200 import stages, synthetic
    g = synthetic.rng(9300 + seed)
    in_nant = int(g.integers(1, 65))
    out_nant = in_nant + int(g.integers(0, 65 - in_nant))
    F = int(g.integers(1, 7))
    H = int(g.integers(1, 12))
    T = 256 * H
    off = 16 * int(g.integers(0, 5))
    taftp = synthetic.voltages_taftp(g, H, in_nant, F, sigma=float(g.uniform(4, 60)))
    fp, st = stages.transpose_fpact_statistics(_dev(cuda, taftp), out_nant,
                                               row_stride=off + T + 16, offset=off)
    ftpa = oracle.transpose(taftp, out_nant)                  # [F][T][P][A][2]
    got = _np(fp)[..., off:off + T]                           # [F][P][A][2][T]
    assert np.array_equal(got, ftpa.transpose(0, 2, 3, 4, 1))
    ref = oracle.statistics(ftpa)
    valid = np.arange(out_nant) < in_nant
    np.testing.assert_allclose(_np(st)[:, :, valid], ref[:, :, valid], rtol=1e-5, atol=1e-6)
