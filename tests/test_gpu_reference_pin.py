"""Pin the oracle, and the B200 kernels, to the reference implementation
itself: the reference's own stage classes (Transposer, StatisticsCalculator,
WeightsManager, IncoherentBeamformer, CoherentBeamformer,
IncoherentDedisperser, CoherentDedisperser) built from its sources into oracle/_ref/libswref.so
(oracle/Makefile `ref`), at that build's compile-time shape (64 antennas,
16 channels, 128 beams, tscrunch 16).

Tolerances are the reference's own GPU-vs-CPU test tolerances: exact for the
transpose, weights and incoherent dedispersion (TransposerTester.cu:90-91,
WeightsManagerTester.cu:94-95, a host implementation), 1e-5 relative for the
statistics (StatisticsCalculatorTester.cu:152-170), +-1 for the int8 beams
(CoherentBeamformerTester.cu:43, its GPU kernel contracts the float chain
into FMAs).  The oracle and the B200 kernels follow the reference's CPU
implementations and agree with each other bit for bit."""
import math
import sys

import numpy as np
import pytest

from conftest import REPO

sys.path.insert(0, REPO + "/oracle")
import swb_ref  # noqa: E402

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not swb_ref.available(),
                                 reason="oracle/_ref not built (needs the reference sources)")]

CENTRE, CHBW = 1284e6, 856e6 / 1024


def _dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def test_transpose_matches_reference(cuda, oracle):
    from skyweaver_b200 import stages, synthetic
    s = swb_ref.shape()
    taftp = synthetic.voltages_taftp(synthetic.rng(1), 8, 57, s["nchans"], sigma=30)
    ref = swb_ref.transpose(taftp, 57)
    assert np.array_equal(oracle.transpose(taftp, s["nant"]), ref)
    got = stages.transpose_ftpa(_dev(cuda, taftp), s["nant"]).cpu().numpy()
    assert np.array_equal(got, ref)


def test_statistics_and_weights_match_reference(cuda, oracle):
    from skyweaver_b200 import stages, synthetic
    s = swb_ref.shape()
    g = synthetic.rng(2)
    ftpa = oracle.transpose(synthetic.voltages_taftp(g, 16, s["nant"], s["nchans"]), s["nant"])
    ref = swb_ref.statistics(ftpa)
    np.testing.assert_allclose(oracle.statistics(ftpa), ref, rtol=1e-5, atol=1e-5)
    bw = s["nchans"] * CHBW
    freqs = stages.channel_frequencies(CENTRE, bw, s["nchans"])
    delays = synthetic.delay_model(g, s["nbeams"], s["nant"])
    wref = swb_ref.weights(delays, 10.0, 9.0, CENTRE, bw)
    assert np.array_equal(oracle.weights(delays, freqs, 10.0, 9.0), wref)
    fba, _ = stages.generate_weights(_dev(cuda, delays), _dev(cuda, freqs), 10.0, 9.0)
    assert np.array_equal(fba.cpu().numpy(), wref)


def test_beamformers_match_reference(cuda, oracle):
    from skyweaver_b200 import stages, synthetic
    s = swb_ref.shape()
    A, F, B, ts = s["nant"], s["nchans"], s["nbeams"], s["cb_ts"]
    g = synthetic.rng(3)
    T = 8192                                   # the reference CB needs T/ts % 512 == 0
    taftp = synthetic.voltages_taftp(g, T // 256, A, F, sigma=32)
    ftpa = oracle.transpose(taftp, A)
    th = g.uniform(0, 2 * np.pi, size=(F, B, A))
    w = np.stack([np.rint(127 * np.cos(th)), np.rint(127 * np.sin(th))], -1).astype(np.int8)
    level = 32.0
    cb_s = (127 * level * math.sqrt(A)) ** 2
    dof = 2 * ts * 2
    cb_scale = np.full(F, cb_s * math.sqrt(2 * dof) / level, np.float32)
    cb_off = np.full(F, cb_s * dof, np.float32)
    ib_dof = 2 * ts * A * 2
    ib_scale = np.full(F, level ** 2 * math.sqrt(2 * ib_dof) / level, np.float32)
    ib_off = np.full(F, level ** 2 * ib_dof, np.float32)
    bw1 = np.ones((1, A), np.float32)
    mapping = np.zeros(B, np.int32)
    raw_r, ib_r, cb_r = swb_ref.beamform(ftpa, w, cb_scale, cb_off, ib_scale, ib_off, bw1,
                                         mapping)
    raw_o, ib_o = oracle.incoherent_beam(ftpa, ts, ib_scale, ib_off, bw1, 1)
    cb_o = oracle.coherent_beam(ftpa, w, ts, cb_scale, cb_off, bw1, mapping)
    np.testing.assert_allclose(raw_o, raw_r, rtol=1e-6)
    assert np.abs(ib_o.astype(int) - ib_r.astype(int)).max() <= 1
    d = np.abs(cb_o.astype(int) - cb_r.astype(int))
    print(f"CB oracle vs reference GPU kernel: {(d > 0).mean():.2e} of samples differ, max {d.max()}")
    assert d.max() <= 1 and (d > 0).mean() < 1e-2
    # the B200 kernels equal the oracle exactly
    fp = stages.transpose_fpact(_dev(cuda, taftp), A)
    raw_g, ib_g = stages.incoherent_beamform(fp, T, ts, _dev(cuda, ib_scale), _dev(cuda, ib_off),
                                             _dev(cuda, bw1))
    cb_g = stages.coherent_beamform(fp, stages.pack_weights(_dev(cuda, w)), _dev(cuda, cb_scale),
                                    _dev(cuda, cb_off), _dev(cuda, mapping), raw_g, T, ts)
    assert np.array_equal(raw_g.cpu().numpy(), raw_o)
    assert np.array_equal(cb_g.cpu().numpy(), cb_o)


def test_incoherent_dedisperser_matches_reference(cuda, oracle):
    from skyweaver_b200 import stages, synthetic
    s = swb_ref.shape()
    F, B = s["nchans"], s["nbeams"]
    bw = F * CHBW
    dms = np.array([0.0, 100.0, 300.0, 500.0], np.float32)
    for ts in (1, 4):
        g = synthetic.rng(4 + ts)
        freqs = stages.channel_frequencies(CENTRE, bw, F)
        delays, maxd = oracle.idd_delays(freqs, dms, s["cb_ts"] / CHBW)
        T = maxd + 64 * ts
        tfb = g.integers(-128, 128, size=(T, F, B), dtype=np.int8)
        ref, dref, mref = swb_ref.idd(tfb, dms, ts, CENTRE, bw)
        assert mref == maxd and np.array_equal(dref, delays)
        sf = np.float32(math.sqrt(F * ts))
        assert np.array_equal(oracle.idd(tfb, delays, maxd, ts, sf), ref)
        got = stages.incoherent_dedisperse(_dev(cuda, tfb), _dev(cuda, delays), maxd, ts, float(sf))
        assert np.array_equal(got.cpu().numpy(), ref)


def test_coherent_dedisperser_matches_reference(cuda, oracle):
    """One 8192-point overlap-save window of one channel (64 antennas x 2
    pols, sigma-12 voltages), DMs {0, 50, 500}, through the reference's own
    CoherentDedisperser (cuFFT in FP32) and through ours, each against the
    FP64 oracle: both within one LSB of it (CoherentDedisperserTester.cu
    allows +-1), and ours within one LSB of the reference on at most 1e-5 of
    the samples (measured: 0, 2.3e-6 and 3.5e-6; the reference itself differs
    from the oracle on 0, 2.9e-6 and 3.5e-6)."""
    from skyweaver_b200 import stages, synthetic
    s = swb_ref.shape()
    F, A = s["nchans"], s["nant"]
    N, ov, chan = 8192, 1472, 5
    bw = F * CHBW
    low = float(np.float32(CENTRE - bw / 2))
    dms = [0.0, 50.0, 500.0]
    g = synthetic.rng(77)
    win = np.clip(np.rint(g.normal(0, 12, size=(2, A, 2, N))), -127, 127).astype(np.int8)
    ext = np.zeros((F, 2, A, 2, N), np.int8)
    ext[chan] = win
    outs = stages.CoherentDedisperser(F, A, N, ov, low, bw, dms).dedisperse(_dev(cuda, ext), N - ov)
    tpa = np.ascontiguousarray(win.transpose(3, 0, 1, 2))          # [N][P][A][2]
    for d, dm in enumerate(dms):
        ref = swb_ref.cdd(tpa, ov, dms, d, chan, low, bw)             # [T][P][A][2]
        ora = oracle.cdd_ftpa(tpa[None], N - ov, oracle.chirp(F, N, low, bw, dm)[chan:chan + 1],
                              ov)[0]
        got = outs[d].cpu().numpy()[chan].transpose(3, 0, 1, 2)
        d_ref = np.abs(ref.astype(int) - ora.astype(int))
        d_got = np.abs(got.astype(int) - ora.astype(int))
        d_rg = np.abs(got.astype(int) - ref.astype(int))
        print(f"DM {dm}: differing from the FP64 oracle: reference {(d_ref > 0).mean():.2e}, "
              f"ours {(d_got > 0).mean():.2e}; ours vs reference {(d_rg > 0).mean():.2e} "
              f"of {d_ref.size} values")
        assert d_ref.max() <= 1 and d_got.max() <= 1 and d_rg.max() <= 1
        assert (d_got > 0).mean() <= 1e-5 and (d_rg > 0).mean() <= 1e-5


@pytest.mark.skipif(not __import__("os").path.exists(swb_ref.LIB_C1),
                    reason="oracle/_ref/c1 not built")
def test_reference_gpu_beamformer_timing(cuda):
    """The reference's own GPU beamformers (dp4a CUDA-core kernels built for
    sm_100a at the benchmark shape: 64 antennas, 64 channels, 1024 beams,
    tscrunch 16, one DM of 65536 samples) timed beside ours on the same
    B200; ours must be faster."""
    torch = cuda
    from skyweaver_b200 import stages
    ms_ib_ref, ms_cb_ref = swb_ref.time_beamform_c1()
    A, F, B, T, ts = 64, 64, 1024, 65536, 16
    gen = torch.Generator(device="cuda").manual_seed(3)
    fp = (torch.randn((F, 2, A, 2, T), generator=gen, device="cuda") * 8).round_().clamp_(-127, 127)
    fp = fp.to(torch.int8)
    gemm = torch.randint(-127, 128, (F, 2, B, A, 2), dtype=torch.int8, device="cuda")
    sc = torch.full((F,), 1e9, device="cuda")
    bw = torch.ones((1, A), device="cuda")
    mapping = torch.zeros(B, dtype=torch.int32, device="cuda")
    raw, _ = stages.incoherent_beamform(fp, T, ts, sc, sc, bw)

    def timeit(fn, reps=5):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    ms_ib = timeit(lambda: stages.incoherent_beamform(fp, T, ts, sc, sc, bw))
    ms_cb = timeit(lambda: stages.coherent_beamform(fp, gemm, sc, sc, mapping, raw, T, ts))
    ops = 8.0 * A * B * 2 * F * T
    print(f"reference GPU: IB {ms_ib_ref:.3f} ms, CB {ms_cb_ref:.3f} ms "
          f"({ops / ms_cb_ref / 1e9:.0f} TOPS); "
          f"B200 kernels: IB {ms_ib:.3f} ms, CB {ms_cb:.3f} ms ({ops / ms_cb / 1e9:.0f} TOPS)")
    assert ms_cb < ms_cb_ref and ms_ib < ms_ib_ref


@pytest.mark.skipif(not __import__("os").path.exists(swb_ref.LIB_C1),
                    reason="oracle/_ref/c1 not built")
def test_reference_gpu_dedisperser_timing(cuda):
    """The reference's own coherent dedispersion (cuFFT, one call per
    channel and DM, 65536-point windows) for a gulp of 64 channels x 2 pols x
    64 antennas at DMs {0, 50, 150, 500}, timed beside ours on the same B200;
    ours must be faster."""
    torch = cuda
    from skyweaver_b200 import stages
    dms = [0.0, 50.0, 150.0, 500.0]
    ms_ref = swb_ref.time_cdd_c1(dms)
    F, A, T, ov = 64, 64, 65536, 1472
    bw = F * CHBW
    low = float(np.float32(CENTRE - bw / 2))
    cdd = stages.CoherentDedisperser(F, A, 8192, ov, low, bw, dms)
    ext = torch.randint(-40, 40, (F, 2, A, 2, ov + T), dtype=torch.int8, device="cuda")
    outs = [torch.empty((F, 2, A, 2, T), dtype=torch.int8, device="cuda") for _ in dms]
    cdd.dedisperse(ext, T, outs)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(3):
        cdd.dedisperse(ext, T, outs)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / 3
    print(f"reference GPU coherent dedispersion: {ms_ref:.1f} ms per gulp; "
          f"B200 kernel: {ms:.2f} ms per gulp ({ms_ref / ms:.1f}x)")
    assert ms < ms_ref
