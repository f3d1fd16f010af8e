"""Floating-point stages against FP64: the max and RMS error of every float
result the path produces before it is requantised, printed (`pytest -s`)
and bounded.

* coherent dedispersion (8192-point on-chip path): the dedispersed voltages
  before rounding, against the FP64 FFT oracle;
* incoherent beam: the detected power (Stokes I) before rescaling, against
  the power summed in FP64, for unit and fractional antenna weights;
* statistics: mean, standard deviation, skewness and kurtosis per
  (channel, pol, antenna), against FP64 moments of the same samples.

The coherent beams and the incoherent dedispersion are integer sums (exact)
followed by the reference's own float chain, which the stage tests check bit
for bit against the reference's CPU implementation."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CHBW = 856e6 / 1024


def _dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _rel(got, want):
    got = np.asarray(got, np.float64)
    want = np.asarray(want, np.float64)
    err = np.abs(got - want)
    rms = math.sqrt(np.mean(err ** 2) / max(np.mean(want ** 2), 1e-300))
    return err.max(), float((err / np.maximum(np.abs(want), 1e-30)).max()), rms


def test_coherent_dedispersion_float_error(cuda, oracle):
    from skyweaver_b200 import stages, synthetic
    g = synthetic.rng(91)
    F, A, T, N = 2, 4, 16384, 8192
    dms = [0.0, 50.0, 150.0, 500.0]
    bw = F * CHBW
    low = 1284e6 - 32 * CHBW
    smear = stages.dm_delay(low, low + CHBW, max(dms)) * CHBW
    overlap = int(math.ceil(smear)) + 15 & ~15
    ext = np.clip(np.rint(g.normal(0, 12, size=(F, 2, A, 2, overlap + T))), -127, 127)
    ext = ext.astype(np.int8)
    outs, dbg = stages.CoherentDedisperser(F, A, N, overlap, low, bw, dms).dedisperse(
        _dev(cuda, ext), T, debug=True)
    dbg = dbg.cpu().numpy()                                  # [D][F][P][A][T][2]
    ftpa_ext = ext.transpose(0, 4, 1, 2, 3)
    for d, dm in enumerate(dms):
        _, f64 = oracle.cdd_ftpa(ftpa_ext, T, oracle.chirp(F, N, low, bw, dm), overlap,
                                 want_f64=True)
        got = dbg[d][..., 0] + 1j * dbg[d][..., 1]           # [F][P][A][T]
        want = f64.transpose(0, 2, 3, 1)
        err = np.abs(got - want)
        rms = math.sqrt(np.mean(err ** 2) / np.mean(np.abs(want) ** 2))
        print(f"CDD 8192 DM {dm}: max |err| {err.max():.2e}, RMS relative {rms:.2e}")
        assert rms < 1e-6 and err.max() < 1e-3


@pytest.mark.parametrize("weights", ["unit", "fractional"])
def test_incoherent_beam_power_error(cuda, oracle, weights):
    from skyweaver_b200 import stages, synthetic
    g = synthetic.rng(92)
    A, F, H, ts = 64, 4, 4, 16
    taftp = synthetic.voltages_taftp(g, H, A, F, sigma=8)
    ftpa = oracle.transpose(taftp, A).astype(np.float64)     # [F][T][P][A][2]
    T = H * 256
    w = (np.ones(A) if weights == "unit" else g.uniform(0.3, 1.0, A)).astype(np.float32)
    sc = np.full(F, 1e4, np.float32)
    raw, _ = stages.incoherent_beamform(stages.transpose_fpact(_dev(cuda, taftp), A), T, ts,
                                        _dev(cuda, sc), _dev(cuda, sc), _dev(cuda, w[None]))
    raw = raw.cpu().numpy()[0]                               # [T/ts][F]
    p = (ftpa ** 2).sum(axis=(2, 4))                          # [F][T][A]
    want = (p * w.astype(np.float64)).sum(axis=2)             # [F][T]
    want = want.reshape(F, T // ts, ts).sum(axis=2).T         # [T/ts][F]
    mx, mxrel, rms = _rel(raw, want)
    print(f"IB power ({weights} weights): max |err| {mx:.2e}, max relative {mxrel:.2e}, "
          f"RMS relative {rms:.2e}")
    if weights == "unit":
        assert mxrel <= 2 ** -24  # exact integer sums, one rounding to float
    else:
        assert rms < 1e-6


def test_statistics_error(cuda, oracle):
    from skyweaver_b200 import stages, synthetic
    g = synthetic.rng(93)
    taftp = synthetic.voltages_taftp(g, 8, 64, 4, sigma=20)
    T = 8 * 256
    got = stages.statistics(stages.transpose_fpact(_dev(cuda, taftp), 64), T).cpu().numpy()
    x = oracle.transpose(taftp, 64).astype(np.float64)       # [F][T][P][A][2]
    x = x.transpose(0, 2, 3, 1, 4).reshape(4, 2, 64, 2 * T)   # re and im of a series together
    n = x.shape[-1]
    m = x.mean(axis=-1)
    c = x - m[..., None]
    m2, m3, m4 = (c ** 2).sum(-1), (c ** 3).sum(-1), (c ** 4).sum(-1)
    std = np.sqrt(m2 / (n - 1))
    skew = (m3 / n) / (m2 / n) ** 1.5
    kurt = (m4 / n) / (m2 / n) ** 2 - 3.0
    for k, (name, want) in enumerate([("mean", m), ("std", std), ("skewness", skew),
                                      ("kurtosis", kurt)]):
        mx, _, rms = _rel(got[..., k], want)
        print(f"statistics {name}: max |err| {mx:.2e}, RMS relative {rms:.2e}")
        assert mx < 1e-5 * max(1.0, np.abs(want).max())
