"""GPU parity tests: every CUDA stage against the oracle (a C restatement of
the reference's CPU test implementations) on the same seeded inputs.

Tolerances follow the reference's own tests and are written next to each
check: integer/byte stages are bit-exact; the tensor-core beamformer's int32
voltages are bit-exact and its int8 output is identical; statistics within
1e-5 relative (StatisticsCalculatorTester.cu:157-169); coherent
dedispersion within +-1 int8 LSB of the FP64 oracle
(CoherentDedisperserTester.cu:195-203).
"""
import math
import os

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu


def _dev(cuda, a):
    return cuda.from_numpy(np.ascontiguousarray(a)).cuda()


def _np(t):
    return t.cpu().numpy()


# ------------------------------------------------------------ transposer
@pytest.mark.parametrize("in_nant,nheaps,out_nant", [(12, 12, 16), (16, 16, 64), (64, 3, 64)])
def test_transpose_ftpa_exact(cuda, oracle, in_nant, nheaps, out_nant):
    from skyweaver_b200 import stages, synthetic
    g = synthetic.rng(1 + in_nant)
    taftp = synthetic.voltages_taftp(g, nheaps, in_nant, 8, sigma=40)
    ref = oracle.transpose(taftp, out_nant)
    got = _np(stages.transpose_ftpa(_dev(cuda, taftp), out_nant))
    assert np.array_equal(got, ref)  # TransposerTester.cu:89-92 exact


def test_transpose_fpact_matches_ftpa(cuda, oracle):
    from skyweaver_b200 import stages, synthetic
    g = synthetic.rng(7)
    taftp = synthetic.voltages_taftp(g, 4, 57, 4, sigma=30)
    ref = oracle.transpose(taftp, 64)                     # FTPA [F][T][P][A][2]
    fp = stages.transpose_fpact(_dev(cuda, taftp), 64, row_stride=1024 + 32, offset=32)
    got = _np(fp)[..., 32:32 + 1024]                      # [F][P][A][C][T]
    assert np.array_equal(got, ref.transpose(0, 2, 3, 4, 1))
    back = _np(stages.fpact_to_ftpa(fp, 1024, offset=32))
    assert np.array_equal(back, ref)
    fp2 = _np(stages.ftpa_to_fpact(_dev(cuda, ref), row_stride=1024 + 32, offset=32))
    assert np.array_equal(fp2[..., 32:], got)


def test_keep_history(cuda):
    from skyweaver_b200._lib import call
    import ctypes
    rows, hist, T = 6, 32, 96
    a = np.arange(rows * (hist + T), dtype=np.int64).astype(np.int8).reshape(rows, hist + T)
    d = _dev(cuda, a)
    call("sw_fpact_keep_history", ctypes.c_void_p(d.data_ptr()), rows, hist + T, hist,
         ctypes.c_void_p(cuda.cuda.current_stream().cuda_stream))
    got = _np(d)
    assert np.array_equal(got[:, :hist], a[:, T:T + hist])
    assert np.array_equal(got[:, hist:], a[:, hist:])


def test_copy_history_between_row_sets(cuda):
    """sw_fpact_copy_history: the last `hist` samples of every row of one row
    set land at the front of the same row of the other; the source rows and
    the rest of the destination rows are untouched (the pipeline alternates
    two row sets this way)."""
    from skyweaver_b200._lib import call
    import ctypes
    rows, hist, T = 7, 48, 160
    g = np.random.default_rng(3)
    a = g.integers(-128, 128, size=(rows, hist + T), dtype=np.int8)
    b = g.integers(-128, 128, size=(rows, hist + T), dtype=np.int8)
    da, db = _dev(cuda, a), _dev(cuda, b)
    call("sw_fpact_copy_history", ctypes.c_void_p(da.data_ptr()), ctypes.c_void_p(db.data_ptr()),
         rows, hist + T, hist, ctypes.c_void_p(cuda.cuda.current_stream().cuda_stream))
    ga, gb = _np(da), _np(db)
    assert np.array_equal(ga, a)
    assert np.array_equal(gb[:, :hist], a[:, T:T + hist])
    assert np.array_equal(gb[:, hist:], b[:, hist:])


# ------------------------------------------------------------ statistics
def test_statistics(cuda, oracle):
    from skyweaver_b200 import stages, synthetic
    g = synthetic.rng(1337)
    taftp = synthetic.voltages_taftp(g, 8, 64, 4, sigma=20)   # StatisticsCalculatorTester: sigma 20
    ftpa = oracle.transpose(taftp, 64)
    ref = oracle.statistics(ftpa)
    fp = stages.transpose_fpact(_dev(cuda, taftp), 64, row_stride=2048 + 64, offset=64)
    got = _np(stages.statistics(fp, 2048, offset=64))
    np.testing.assert_allclose(got, ref, rtol=1e-5, atol=1e-6)


@pytest.mark.parametrize("fill", ["zeros", "constant", "two_values"])
def test_statistics_degenerate_inputs(cuda, oracle, fill):
    """StatisticsCalculatorTester.cu:195-205 runs the statistics on a
    zero-initialised gulp. Zero and constant series have no variance, so
    skewness and kurtosis are 0/0 = NaN in the reference's formulas
    (StatisticsCalculator.cu:80-83), and must be NaN here too; a series of
    two values has exact moments."""
    from skyweaver_b200 import stages
    T, A, F = 1024, 8, 3
    taftp = np.zeros((T // 256, A, F, 256, 2, 2), np.int8)
    if fill == "constant":
        taftp[:] = -7
    elif fill == "two_values":
        taftp[..., 0] = 3
        taftp[..., 1] = -5
    ref = oracle.statistics(oracle.transpose(taftp, A))
    got = _np(stages.statistics(stages.transpose_fpact(_dev(cuda, taftp), A), T))
    np.testing.assert_allclose(got, ref, rtol=1e-5, atol=1e-6, equal_nan=True)
    if fill != "two_values":
        assert np.isnan(got[..., 2:]).all() and not np.isnan(got[..., :2]).any()
    else:
        assert np.allclose(got[..., 0], -1.0) and np.allclose(got[..., 1], 4.0 * math.sqrt(
            2 * T / (2 * T - 1)), rtol=1e-6)


@pytest.mark.parametrize("nheaps,in_nant,out_nant", [(8, 64, 64), (20, 57, 64), (3, 12, 16),
                                                    (5, 9, 18)])
def test_transpose_statistics_fused_equals_separate(cuda, oracle, nheaps, in_nant, out_nant):
    """The one-pass transpose + statistics writes the same FPACT bytes and the
    same statistics (bit for bit) as the two separate stages, padded
    antennas and a heap count that is not a multiple of the CTA's 8 heaps
    included; the statistics match the oracle within its tolerance."""
    from skyweaver_b200 import stages, synthetic
    g = synthetic.rng(4242)
    taftp = _dev(cuda, synthetic.voltages_taftp(g, nheaps, in_nant, 5, sigma=20))
    T, off = nheaps * 256, 80
    fp0 = stages.transpose_fpact(taftp, out_nant, row_stride=T + off + 16, offset=off)
    st0 = stages.statistics(fp0, T, offset=off)
    fp1, st1 = stages.transpose_fpact_statistics(taftp, out_nant, row_stride=T + off + 16,
                                                 offset=off)
    assert cuda.equal(fp0, fp1)
    a, b = _np(st0), _np(st1)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    ref = oracle.statistics(oracle.transpose(_np(taftp), out_nant))
    valid = np.arange(out_nant) < in_nant
    np.testing.assert_allclose(b[:, :, valid], ref[:, :, valid], rtol=1e-5, atol=1e-6)


def test_scalings_bit_exact(cuda, oracle):
    from skyweaver_b200 import stages, synthetic
    g = synthetic.rng(5)
    stats = np.abs(g.normal(8, 2, size=(16, 2, 32, 4))).astype(np.float32)
    bw = synthetic.beamset_masks(g, 32, [32, 20, 7])
    ref = oracle.scalings(stats, bw, 3, 16, 8, 24.0)
    got = stages.update_scalings(_dev(cuda, stats), _dev(cuda, bw), 16, 8, 24.0)
    for r, x in zip(ref, got):
        assert np.array_equal(_np(x), r)


# --------------------------------------------------------------- weights
@pytest.mark.parametrize("case", ["zero", "real_value", "real_values", "synthetic"])
def test_weights(cuda, oracle, case):
    from skyweaver_b200 import stages, synthetic
    B, A, F = 64, 64, 16
    freqs = synthetic.channel_frequencies(1284e6, 13.375e6, F)
    if case == "zero":          # WeightsManagerTester.cu:99-112
        d = np.tile(np.array([1.0, 0.0, 0.0], np.float32), (B, A, 1))
    elif case == "real_value":  # :114-127
        d = np.tile(np.array([1.0, 1e-11, 1e-10], np.float32), (B, A, 1))
    elif case == "real_values":  # :129-145
        ii = np.arange(B * A, dtype=np.float32)
        d = np.stack([ii * np.float32(1e-11), ii * np.float32(1e-15),
                      np.zeros_like(ii)], -1).reshape(B, A, 3).astype(np.float32)
    else:
        d = synthetic.delay_model(synthetic.rng(3), B, A)
    ref = oracle.weights(d, freqs, 10.0, 9.0)
    fba, gemm = stages.generate_weights(_dev(cuda, d), _dev(cuda, freqs), 10.0, 9.0)
    got = _np(fba)
    # exact except where the reference's round-half-away and the GPU's
    # round-half-even differ on an exact .5 (not present in these inputs)
    assert np.array_equal(got, ref)
    gm = _np(gemm)
    assert np.array_equal(gm[:, 0, ..., 0], ref[..., 0])
    assert np.array_equal(gm[:, 0, ..., 1], -ref[..., 1])
    assert np.array_equal(gm[:, 1, ..., 0], ref[..., 1])
    assert np.array_equal(gm[:, 1, ..., 1], ref[..., 0])
    assert np.array_equal(_np(stages.pack_weights(fba)), gm)


# ----------------------------------------------------- incoherent beam
@pytest.mark.parametrize("stokes", ["I", "Q", "U", "V", "IQUV"])
@pytest.mark.parametrize("nbeamsets", [1, 4])
def test_incoherent_beam_bit_exact(cuda, oracle, stokes, nbeamsets):
    from skyweaver_b200 import stages, synthetic
    g = synthetic.rng(11)
    A, F, H, ts = 64, 4, 4, 16
    taftp = synthetic.voltages_taftp(g, H, A, F, sigma=32)   # IncoherentBeamformerTester: sigma 32
    ftpa = oracle.transpose(taftp, A)
    T = H * 256
    level = 32.0
    dof = 2 * ts * A * 2
    scale = np.full(nbeamsets * F, level ** 2 * math.sqrt(2 * dof) / level, np.float32)
    offset = np.full(nbeamsets * F, level ** 2 * dof, np.float32)
    bw = synthetic.beamset_masks(g, A, [64, 40, 17, 3][:nbeamsets])
    raw_ref, out_ref = oracle.incoherent_beam(ftpa, ts, scale, offset, bw, nbeamsets, stokes)
    fp = stages.transpose_fpact(_dev(cuda, taftp), A)
    raw, out = stages.incoherent_beamform(fp, T, ts, _dev(cuda, scale), _dev(cuda, offset),
                                          _dev(cuda, bw), stokes=stokes)
    assert np.array_equal(_np(raw), raw_ref)
    assert np.array_equal(_np(out), out_ref)


@pytest.mark.parametrize("stokes,ts,A", [("I", 32, 64), ("IQUV", 32, 64), ("I", 8, 64),
                                         ("I", 4, 48), ("I", 16, 80)])
def test_incoherent_beam_float_chain_path(cuda, oracle, stokes, ts, A):
    """Strong RFI and non-integer weights force the reference-order float chain:
    through the 16-sample product table (tscrunch a multiple of 16, at most 64
    antennas) and byte by byte otherwise."""
    from skyweaver_b200 import stages, synthetic
    g = synthetic.rng(12)
    F, H = 2, 2
    taftp = synthetic.voltages_taftp(g, H, A, F, sigma=8)
    synthetic.inject_tones(taftp, [1], amplitude=110.0)
    ftpa = oracle.transpose(taftp, A)
    bw = np.stack([np.ones(A, np.float32), g.uniform(0.3, 1.0, A).astype(np.float32)])
    scale = np.full(2 * F, 5000.0, np.float32)
    offset = np.full(2 * F, 1e5, np.float32)
    raw_ref, out_ref = oracle.incoherent_beam(ftpa, ts, scale, offset, bw, 2, stokes)
    fp = stages.transpose_fpact(_dev(cuda, taftp), A)
    raw, out = stages.incoherent_beamform(fp, H * 256, ts, _dev(cuda, scale),
                                          _dev(cuda, offset), _dev(cuda, bw), stokes=stokes)
    assert np.array_equal(_np(raw), raw_ref)
    assert np.array_equal(_np(out), out_ref)


# ------------------------------------------------------- coherent beam
def _cb_case(cuda, oracle, A, B, F, H, ts, stokes, ib_sub, nbeamsets=2, seed=21):
    from skyweaver_b200 import stages, synthetic
    g = synthetic.rng(seed)
    taftp = synthetic.voltages_taftp(g, H, A, F, sigma=32)
    T = H * 256
    ftpa = oracle.transpose(taftp, A)
    # weights 127*exp(i theta) like CoherentBeamformerTester.cu:301-309
    th = g.uniform(0, 2 * np.pi, size=(F, B, A))
    w = np.stack([np.rint(127 * np.cos(th)), np.rint(127 * np.sin(th))], -1).astype(np.int8)
    level = 32.0
    cb_scale = (127 * level * math.sqrt(A)) ** 2
    dof = 2 * ts * 2
    scales = np.full(nbeamsets * F, cb_scale * math.sqrt(2 * dof) / level, np.float32)
    offsets = np.full(nbeamsets * F, cb_scale * dof, np.float32)
    bw = np.ones((nbeamsets, A), np.float32)
    mapping = np.zeros(B, np.int32)
    mapping[0] = 1 % nbeamsets                 # CoherentBeamformerTester.cu:259
    ib_dof = 2 * ts * A * 2
    ib_scale = np.full(nbeamsets * F, level ** 2 * math.sqrt(2 * ib_dof) / level, np.float32)
    ib_off = np.full(nbeamsets * F, level ** 2 * ib_dof, np.float32)
    fp = stages.transpose_fpact(_dev(cuda, taftp), A)
    raw_ib, _ = stages.incoherent_beamform(fp, T, ts, _dev(cuda, ib_scale), _dev(cuda, ib_off),
                                           _dev(cuda, bw), stokes=stokes)
    gemm = stages.pack_weights(_dev(cuda, w))
    out, dbg = stages.coherent_beamform(fp, gemm, _dev(cuda, scales), _dev(cuda, offsets),
                                        _dev(cuda, mapping), raw_ib, T, ts, stokes=stokes,
                                        ib_subtract=ib_sub, debug=True)
    ref, volts = oracle.coherent_beam(ftpa, w, ts, scales, offsets, bw, mapping, stokes,
                                      ib_sub, want_voltages=True)
    return _np(out), ref, _np(dbg), volts


@pytest.mark.parametrize("A", [16, 32, 64])
def test_coherent_beam_voltages_and_power_exact(cuda, oracle, A):
    out, ref, dbg, volts = _cb_case(cuda, oracle, A, 128, 2, 2, 16, "I", True)
    assert np.array_equal(dbg, volts)     # int32 beam voltages bit-exact
    assert np.array_equal(out, ref)       # int8 TFB identical to the CPU reference


def _report(out, ref):
    bad = np.argwhere(out != ref)
    lines = [f"{len(bad)} of {out.size} differ"]
    for idx in bad[:8]:
        lines.append(f"  {tuple(idx)}: got {out[tuple(idx)]} want {ref[tuple(idx)]}")
    return "\n".join(lines)


@pytest.mark.parametrize("tpi", [1, 3, 5, 7, 64, 1024])
def test_coherent_beam_work_item_sizes(cuda, oracle, tpi):
    """The persistent beamformer splits each (problem, channel, 128-beam
    block) into work items of `tpi` 64-sample tiles, and its two epilogue
    groups take alternate tiles across item boundaries: odd item lengths
    (and items cut short at the end of the gulp) must give the same bytes."""
    from skyweaver_b200 import stages, synthetic
    A, F, B, H, ts = 32, 3, 256, 7, 16          # 1792 samples = 28 tiles
    g = synthetic.rng(40 + tpi)
    taftp = synthetic.voltages_taftp(g, H, A, F, sigma=32)
    T = H * 256
    ftpa = oracle.transpose(taftp, A)
    th = g.uniform(0, 2 * np.pi, size=(F, B, A))
    w = np.stack([np.rint(127 * np.cos(th)), np.rint(127 * np.sin(th))], -1).astype(np.int8)
    level = 32.0
    cb_s = (127 * level * math.sqrt(A)) ** 2
    dof = 2 * ts * 2
    scales = np.full(F, cb_s * math.sqrt(2 * dof) / level, np.float32)
    offsets = np.full(F, cb_s * dof, np.float32)
    bw = np.ones((1, A), np.float32)
    mapping = np.zeros(B, np.int32)
    ib_dof = 2 * ts * A * 2
    ib_scale = np.full(F, level ** 2 * math.sqrt(2 * ib_dof) / level, np.float32)
    ib_off = np.full(F, level ** 2 * ib_dof, np.float32)
    fp = stages.transpose_fpact(_dev(cuda, taftp), A)
    raw_ib, _ = stages.incoherent_beamform(fp, T, ts, _dev(cuda, ib_scale), _dev(cuda, ib_off),
                                           _dev(cuda, bw))
    gemm = stages.pack_weights(_dev(cuda, w))
    out = stages.coherent_beamform(fp, gemm, _dev(cuda, scales), _dev(cuda, offsets),
                                   _dev(cuda, mapping), raw_ib, T, ts, tiles_per_item=tpi)
    ref = oracle.coherent_beam(ftpa, w, ts, scales, offsets, bw, mapping)
    assert np.array_equal(_np(out), ref), _report(_np(out), ref)


def test_coherent_beam_bounded_wait_times_out_and_context_survives(cuda, oracle):
    """Every wait in the persistent beamformer is bounded.  The self-test
    launches it with a copy producer that issues nothing, so the MMA role's
    first wait can only end at its 20 ms deadline: the kernel must record
    the timeout in the device error word, every role must leave, and the
    context must stay usable (a normal launch afterwards is exact)."""
    from skyweaver_b200 import _lib, stages
    stages.reset_device_error()
    assert stages.cb_timeout_selftest(20000) == _lib.SW_ERR_TIMEOUT
    assert stages.device_error() == 0          # the self-test clears the word
    out, ref, dbg, volts = _cb_case(cuda, oracle, 16, 128, 2, 1, 16, "I", True)
    assert np.array_equal(dbg, volts) and np.array_equal(out, ref)
    stages.check_device_error()                # nothing recorded by the normal launch


@pytest.mark.parametrize("stokes", ["I", "Q", "U", "V", "IQUV"])
@pytest.mark.parametrize("ib_sub", [True, False])
def test_coherent_beam_stokes(cuda, oracle, stokes, ib_sub):
    out, ref, dbg, volts = _cb_case(cuda, oracle, 64, 256, 3, 2, 4, stokes, ib_sub, seed=22)
    assert np.array_equal(dbg, volts)
    assert np.array_equal(out, ref), _report(out, ref)
    # run-to-run determinism of the whole chain
    out2, _, _, _ = _cb_case(cuda, oracle, 64, 256, 3, 2, 4, stokes, ib_sub, seed=22)
    assert np.array_equal(out, out2), _report(out2, out)


@pytest.mark.parametrize("ts", [1, 2, 8])
@pytest.mark.parametrize("stokes", ["I", "Q", "U", "V", "IQUV"])
def test_coherent_beam_short_tscrunch(cuda, oracle, ts, stokes):
    """tscrunch 1, 2 and 8 (bit-exact like 4, 16 and 32 above), where the
    epilogue hands its accumulator buffer back before the last column
    group's arithmetic; full Stokes at tscrunch <= 4 reads 8-column groups."""
    out, ref, dbg, volts = _cb_case(cuda, oracle, 64, 256, 3, 2, ts, stokes, stokes == "I",
                                    seed=24)
    assert np.array_equal(dbg, volts)
    assert np.array_equal(out, ref), _report(out, ref)


@pytest.mark.parametrize("A", [16, 32, 64])
def test_coherent_beam_partial_block_and_tscrunch(cuda, oracle, A):
    """96 beams (a partial 128-beam block), tscrunch 32, and every supported
    antenna count: K = 2 A bytes = 1, 2 or 4 MMA K steps with the SW32, SW64 or
    SW128 weight layouts."""
    out, ref, dbg, volts = _cb_case(cuda, oracle, A, 96, 2, 1, 32, "I", True, seed=23)
    assert np.array_equal(dbg, volts)
    assert np.array_equal(out, ref)


def test_coherent_beam_grouped_equals_plain(cuda, oracle):
    from skyweaver_b200 import stages, synthetic
    g = synthetic.rng(31)
    A, B, F, H, ts = 64, 384, 2, 2, 16
    T = H * 256
    fps = [stages.transpose_fpact(_dev(cuda, synthetic.voltages_taftp(g, H, A, F)), A)
           for _ in range(3)]
    th = g.uniform(0, 2 * np.pi, size=(F, B, A))
    w = np.stack([np.rint(127 * np.cos(th)), np.rint(127 * np.sin(th))], -1).astype(np.int8)
    gemm = stages.pack_weights(_dev(cuda, w))
    mapping = np.repeat(np.arange(3, dtype=np.int32), [200, 120, 64])
    scales = _dev(cuda, np.full(3 * F, 1e6, np.float32))
    offs = _dev(cuda, np.full(3 * F, 1e5, np.float32))
    ibs = [cuda.rand((3, T // ts, F), device="cuda") * 100 for _ in fps]
    plain = []
    for fp, ib in zip(fps, ibs):
        outs = cuda.zeros((T // ts, F, B), dtype=cuda.int8, device="cuda")
        for b0, n in ((0, 200), (200, 120), (320, 64)):
            stages.coherent_beamform(fp, gemm, scales, offs, _dev(cuda, mapping), ib, T, ts,
                                     beam_start=b0, beam_count=n, out=outs)
        plain.append(_np(outs))
    outs = [cuda.zeros((T // ts, F, B), dtype=cuda.int8, device="cuda") for _ in fps]
    probs = [(fp, o, ib, b0, n) for fp, o, ib in zip(fps, outs, ibs)
             for b0, n in ((0, 200), (200, 120), (320, 64))]
    stages.coherent_beamform_grouped(probs, gemm, scales, offs, _dev(cuda, mapping), T, ts)
    for a, b in zip(plain, outs):
        assert np.array_equal(a, _np(b))
    # every pipeline depth the autotuner may pick gives the same beams
    for vst, wst in ((2, 2), (3, 2), (6, 2), (8, 2), (4, 3), (6, 3)):
        for o in outs:
            o.zero_()
        stages.coherent_beamform_grouped(probs, gemm, scales, offs, _dev(cuda, mapping), T, ts,
                                         tiles_per_item=2, voltage_stages=vst, weight_stages=wst)
        for a, b in zip(plain, outs):
            assert np.array_equal(a, _np(b)), (vst, wst)


# ------------------------------------------------- coherent dedispersion
def test_coherent_dedispersion_golden_vector(cuda):
    """CoherentDedisperserTester.cu:113-204: DM 1000, fft 1024, 1 channel,
    python-generated golden output, +-1 LSB."""
    from skyweaver_b200 import stages
    inp = np.fromfile(os.path.join(GOLDEN, "codedisp_input_DM1000_1chan.bin"),
                      np.int8).reshape(1024, 2, 64, 2)
    want = np.fromfile(os.path.join(GOLDEN, "codedisp_output_DM1000_1chan.bin"),
                       np.int8).reshape(446, 2, 64, 2)
    tsamp = 4096 / 856e6
    overlap = math.ceil(stages.dm_delay(856e6, 856e6 + 856e6 / 4096, 1000.0) / tsamp)
    assert overlap == 578
    # channel 0 of the reference's 64-channel, 13.375 MHz configuration: a
    # one-channel table with the same coarse channel width and centre
    cdd = stages.CoherentDedisperser(1, 64, 1024, overlap, 856e6, 13.375e6 / 64, [0.0, 1000.0])
    fp = _dev(cuda, inp.transpose(1, 2, 3, 0)[None].copy())   # [1][P][A][C][1024]
    outs = cdd.dedisperse(fp, 1024 - overlap)
    got = _np(outs[1])[0].transpose(3, 0, 1, 2)                # [446][P][A][C]
    diff = np.abs(got.astype(int) - want.astype(int))
    print(f"golden DM 1000: {(diff > 0).sum()} of {diff.size} differ by one LSB")
    assert diff.max() <= 1                                     # reference tolerance
    assert (diff > 0).mean() <= 1e-5                           # measured: 1 of 114176
    # DM 0 is the identity shifted by overlap/2 (CoherentDedisperserTester.cu:69-111)
    got0 = _np(outs[0])[0].transpose(3, 0, 1, 2)
    assert np.abs(got0.astype(int) - inp[overlap // 2: overlap // 2 + 446].astype(int)).max() <= 1


@pytest.mark.parametrize("fft_len,dms,lag", [(2048, [0.0, 50.0, 150.0], None),
                                             (4096, [0.0, 500.0], 128), (8192, [150.0], 128),
                                             (8192, [0.0, 50.0, 500.0], None), (1024, [30.0], 64),
                                             (16384, [0.0, 500.0], 128), (32768, [150.0], None)])
def test_coherent_dedispersion_overlap_save(cuda, oracle, fft_len, dms, lag):
    """Every window trims overlap - lag samples at its start and lag at its
    end: lag None is the reference's overlap / 2 at each end, the others the
    pipeline's one-sided plan.  Against the FP64 oracle at the same plan."""
    from skyweaver_b200 import stages, synthetic
    g = synthetic.rng(fft_len + (lag or 0))
    F, A, T = 2, 4, 8192
    chbw = 856e6 / 1024                      # MeerKAT L-band 1024-channel mode
    bw = F * chbw
    low = 1284e6 - 32 * chbw                 # bottom of a 64-channel subband
    tsamp = 1.0 / chbw
    smear = stages.dm_delay(low, low + bw / F, max(dms)) / tsamp
    if lag is None:
        overlap = int(math.ceil(smear)) + 1 & ~1
    else:
        overlap = (int(math.ceil(smear)) + 15 & ~15) + lag
    assert overlap < fft_len
    ext = np.clip(np.rint(g.normal(0, 12, size=(F, 2, A, 2, overlap + T))), -127, 127).astype(np.int8)
    cdd = stages.CoherentDedisperser(F, A, fft_len, overlap, low, bw, dms, lag=lag)
    outs = cdd.dedisperse(_dev(cuda, ext), T)
    for d, dm in enumerate(dms):
        chirps = oracle.chirp(F, fft_len, low, bw, dm)
        ftpa_ext = ext.transpose(0, 4, 1, 2, 3)                  # [F][O+T][P][A][2]
        ref, f64 = oracle.cdd_ftpa(ftpa_ext, T, chirps, overlap, want_f64=True, lag=lag)
        got = _np(outs[d]).transpose(0, 4, 1, 2, 3)
        diff = np.abs(got.astype(int) - ref.astype(int))
        frac = (diff > 0).mean()
        print(f"fft {fft_len} lag {lag} DM {dm}: {(diff > 0).sum()} of {diff.size} differ "
              f"by one LSB")
        assert diff.max() <= 1, (dm, diff.max())
        assert frac <= 1e-5, (dm, frac)                       # measured: at most 2 of 262144


def test_coherent_dedispersion_fft65536_precision(cuda, oracle):
    """Precision study with 2^16-point overlap-save FFTs (L-band, 64-channel
    subband bottom, DMs {0, 50, 150, 500}): the float dedispersed voltages
    before requantisation against the FP64 oracle, and the int8 outputs
    within one LSB.  The workspace is limited so that the segments run in
    several chunks."""
    from skyweaver_b200 import stages, synthetic
    g = synthetic.rng(65536)
    F, A, T, N = 2, 4, 98304, 65536
    dms = [0.0, 50.0, 150.0, 500.0]
    chbw = 856e6 / 1024
    bw = F * chbw
    low = 1284e6 - 32 * chbw
    smear = stages.dm_delay(low, low + chbw, max(dms)) * chbw
    overlap = int(math.ceil(smear)) + 15 & ~15
    ext = np.clip(np.rint(g.normal(0, 8, size=(F, 2, A, 2, overlap + T))), -127, 127).astype(np.int8)
    cdd = stages.CoherentDedisperser(F, A, N, overlap, low, bw, dms)
    outs, dbg = cdd.dedisperse(_dev(cuda, ext), T, debug=True,
                               workspace_limit=3 * len(dms) * N * 8)
    dbg = _np(dbg)                                   # [D][F][P][A][T][2]
    ftpa_ext = ext.transpose(0, 4, 1, 2, 3)
    for d, dm in enumerate(dms):
        ref, f64 = oracle.cdd_ftpa(ftpa_ext, T, oracle.chirp(F, N, low, bw, dm), overlap,
                                   want_f64=True)
        got_f = dbg[d][..., 0] + 1j * dbg[d][..., 1]  # [F][P][A][T]
        want_f = f64.transpose(0, 2, 3, 1)
        err = np.abs(got_f - want_f)
        rms_rel = math.sqrt(np.mean(err ** 2) / np.mean(np.abs(want_f) ** 2))
        print(f"DM {dm}: max |err| {err.max():.3e}, rms rel {rms_rel:.3e}")
        assert rms_rel < 1e-5, (dm, rms_rel)
        assert err.max() < 0.05, (dm, err.max())
        got = _np(outs[d]).transpose(0, 4, 1, 2, 3)
        diff = np.abs(got.astype(int) - ref.astype(int))
        print(f"fft 65536 DM {dm}: {(diff > 0).sum()} of {diff.size} differ by one LSB")
        assert diff.max() <= 1 and (diff > 0).mean() <= 1e-5, (dm, (diff > 0).mean())


# ------------------------------------------------- incoherent dedispersion
def test_incoherent_dedispersion_exact(cuda, oracle):
    from skyweaver_b200 import stages, synthetic
    g = synthetic.rng(41)
    F, B, ts = 64, 64, 2
    freqs = synthetic.channel_frequencies(580e6, 32e6, F)
    dms = np.array([0, 10, 20, 30, 40], np.float32)
    tsamp = 16 / (32e6 / F)
    delays, maxd = oracle.idd_delays(freqs, dms, tsamp)
    T = maxd + 64 * ts
    tfb = g.integers(-128, 128, size=(T, F, B), dtype=np.int8)
    sf = np.float32(math.sqrt(F * ts))
    ref = oracle.idd(tfb, delays, maxd, ts, sf)
    got = stages.incoherent_dedisperse(_dev(cuda, tfb), _dev(cuda, delays), maxd, ts, float(sf))
    assert np.array_equal(_np(got), ref)


@pytest.mark.parametrize("fill", ["random", -128, 127])
def test_incoherent_dedispersion_many_channels(cuda, oracle, fill):
    """More than 256 terms per sum (301 channels x tscrunch 3, an odd channel
    count) at the int8 extremes: the 16-bit partial sums of the 16-beam path
    are flushed every 256 channels, and every sum must still be exact."""
    from skyweaver_b200 import stages, synthetic
    g = synthetic.rng(43)
    F, B, ts = 301, 48, 3
    freqs = synthetic.channel_frequencies(1284e6, 64 * 856e6 / 1024, F)
    dms = np.array([0, 3, 7], np.float32)
    delays, maxd = oracle.idd_delays(freqs, dms, 16 / (856e6 / 1024))
    T = maxd + 16 * ts
    if fill == "random":
        tfb = g.integers(-128, 128, size=(T, F, B), dtype=np.int8)
        sf = np.float32(64.0)
    else:
        tfb = np.full((T, F, B), fill, np.int8)
        sf = np.float32(1000.0)
    ref = oracle.idd(tfb, delays, maxd, ts, sf)
    got = _np(stages.incoherent_dedisperse(_dev(cuda, tfb), _dev(cuda, delays), maxd, ts,
                                           float(sf)))
    assert np.array_equal(got, ref)
    if fill != "random":
        assert np.all(ref == int(fill * F * ts / 1000.0))


@pytest.mark.parametrize("F,B,ndms,ts,misalign", [
    (8, 1040, 37, 1, 0),   # 16-beam path: 65 lanes -> beam blocks of 32, 32, 1; DM groups 16, 16, 5
    (16, 528, 3, 5, 0),    # 16-beam path: 33 lanes -> two beam blocks, one DM group
    (12, 20, 5, 3, 0),     # 4-beam path: 5 beam quads
    (16, 64, 18, 2, 4),    # beams a multiple of 16 but the TFB only 4-byte aligned -> 4-beam path
])
def test_incoherent_dedispersion_launch_shapes(cuda, oracle, F, B, ndms, ts, misalign):
    """Beam counts and DM counts that leave partial beam blocks and partial DM
    groups in the launch grid, and a TFB that does not start on a 16-byte
    boundary: every output must still equal the oracle's."""
    from skyweaver_b200 import stages, synthetic
    g = synthetic.rng(1000 + B + ndms)
    freqs = synthetic.channel_frequencies(1284e6, F * 856e6 / 1024, F)
    dms = np.linspace(0.0, 60.0, ndms).astype(np.float32)
    delays, maxd = oracle.idd_delays(freqs, dms, 16 / (856e6 / 1024))
    T = maxd + 40 * ts
    tfb = g.integers(-128, 128, size=(T, F, B), dtype=np.int8)
    sf = np.float32(math.sqrt(F * ts))
    ref = oracle.idd(tfb, delays, maxd, ts, sf)
    buf = cuda.empty(tfb.size + 16, dtype=cuda.int8, device="cuda")
    d_tfb = buf[misalign:misalign + tfb.size].view(T, F, B)
    d_tfb.copy_(cuda.from_numpy(tfb))
    assert d_tfb.data_ptr() % 16 == misalign
    got = _np(stages.incoherent_dedisperse(d_tfb, _dev(cuda, delays), maxd, ts, float(sf)))
    assert got.shape == (40, ndms, B)
    assert np.array_equal(got, ref)


def test_incoherent_dedispersion_ones(cuda, oracle):
    """IncoherentDedisperserTester.cu:96-126: all-ones input -> sqrt(F*ts)."""
    from skyweaver_b200 import stages, synthetic
    F, B, ts = 64, 32, 2
    freqs = synthetic.channel_frequencies(580e6, 32e6, F)
    dms = np.array([0, 10, 20, 30, 40], np.float32)
    delays, maxd = oracle.idd_delays(freqs, dms, 16 / (32e6 / F))
    T = 3 * maxd
    T -= (T - maxd) % ts
    tfb = np.ones((T, F, B), np.int8)
    got = _np(stages.incoherent_dedisperse(_dev(cuda, tfb), _dev(cuda, delays), maxd, ts,
                                           float(np.float32(math.sqrt(F * ts)))))
    assert got.shape == ((T - maxd) // ts, 5, B)
    assert np.all(got == int(math.sqrt(F * ts)))


def test_incoherent_dedispersion_char4_iquv(cuda, oracle):
    """char4 (IQUV) TFB: every component dedispersed and clamped on its own,
    like the reference's char4 instantiation (IncoherentDedisperser.cu:133-137)."""
    from skyweaver_b200 import stages, synthetic
    g = synthetic.rng(42)
    F, B, ts = 32, 16, 4
    freqs = synthetic.channel_frequencies(1284e6, 32 * 856e6 / 1024, F)
    dms = np.array([0, 50, 100], np.float32)
    delays, maxd = oracle.idd_delays(freqs, dms, ts * 16 / (856e6 / 1024))
    T = maxd + 32 * ts
    tfb = g.integers(-128, 128, size=(T, F, B, 4), dtype=np.int8)
    sf = np.float32(math.sqrt(F * ts))
    got = _np(stages.incoherent_dedisperse(_dev(cuda, tfb), _dev(cuda, delays), maxd, ts,
                                           float(sf)))
    assert got.shape == ((T - maxd) // ts, 3, B, 4)
    for c in range(4):
        ref = oracle.idd(np.ascontiguousarray(tfb[..., c]), delays, maxd, ts, sf)
        assert np.array_equal(got[..., c], ref)


def test_incoherent_dedispersion_pipeline_push_semantics(cuda, oracle):
    """AggregationBufferTester.cu:30-109 through the device pipeline. With one
    channel, one DM of delay 0, tscrunch 1 and scale 1 the dedisperser is the
    identity, so each dispatch hands back the buffer itself: one push of one
    dispatch (10 samples of 4 beams) fires one dispatch equal to it; a push
    of 100 samples fires 10, the last holding samples 90..99. With an overlap
    (two channels, delays {1, 0}: overlap 1) a 100-sample push fires
    (100 - 1) // 10 = 9 dispatches, the k-th covering samples
    [10 k, 10 k + 11). A push that is not whole samples raises."""
    from skyweaver_b200 import stages, synthetic
    g = synthetic.rng(47)
    B = 4
    got = []
    ident = [(np.zeros((1, 1), np.int32), 1, 1.0)]
    pipe = stages.IncoherentDedispersionPipeline(1, B, ident, lambda b, t: got.append(_np(t)),
                                                 dispatch=[10])
    one = g.integers(-128, 128, size=(10, 1, B), dtype=np.int8)
    pipe.push(0, _dev(cuda, one))
    cuda.cuda.synchronize()
    assert len(got) == 1 and np.array_equal(got[0][:, 0, :], one[:, 0, :])
    got.clear()
    many = g.integers(-128, 128, size=(100, 1, B), dtype=np.int8)
    pipe.push(0, _dev(cuda, many))
    cuda.cuda.synchronize()
    assert len(got) == 10 and np.array_equal(got[-1][:, 0, :], many[90:, 0, :])
    with pytest.raises(RuntimeError, match="slot size"):
        pipe.push(0, _dev(cuda, g.integers(-128, 128, size=101, dtype=np.int8)))
    pipe.close()

    got = []
    delays = np.array([[1, 0]], np.int32)
    pipe = stages.IncoherentDedispersionPipeline(2, B, [(delays, 1, 1.0)],
                                                 lambda b, t: got.append(_np(t)), dispatch=[10])
    assert pipe.geometry(0) == (10, 1, 10, 1)
    data = g.integers(-128, 128, size=(100, 2, B), dtype=np.int8)
    pipe.push(0, _dev(cuda, data))
    cuda.cuda.synchronize()
    pipe.close()
    assert len(got) == 9
    for k, tdb in enumerate(got):
        ref = oracle.idd(np.ascontiguousarray(data[10 * k:10 * k + 11]), delays, 1, 1,
                         np.float32(1.0))
        assert np.array_equal(tdb, ref), k


def test_incoherent_dedispersion_pipeline_aggregation(cuda, oracle):
    """Device AggregationBuffer semantics (AggregationBuffer.cu:23-117): with
    dispatch D and overlap O = max delay, dispatch k covers samples
    [k D, (k+1) D + O) of the pushed stream, whatever the push sizes."""
    from skyweaver_b200 import stages, synthetic
    g = synthetic.rng(43)
    F, B = 16, 8
    freqs = synthetic.channel_frequencies(1284e6, F * 856e6 / 1024, F)
    tsamp = 16 / (856e6 / 1024)
    blocks, refs = [], []
    for dms, ts in (([0.0, 40.0, 80.0], 2), ([250.0, 300.0], 4)):
        delays, maxd = oracle.idd_delays(freqs, np.array(dms, np.float32), tsamp)
        sf = np.float32(math.sqrt(F * ts))
        blocks.append((delays, ts, float(sf)))
        refs.append((delays, maxd, ts, sf))
    got = {0: [], 1: []}
    pipe = stages.IncoherentDedispersionPipeline(F, B, blocks, lambda b, t: got[b].append(t),
                                                 dispatch=[512, 1000])
    total = 6000
    stream = g.integers(-128, 128, size=(total, F, B), dtype=np.int8)
    for blk in (0, 1):
        pos = 0
        for n in (1, 700, 33, 2048, 1500, 1718):
            pipe.push(blk, _dev(cuda, stream[pos:pos + n]))
            pos += n
        assert pos == total
    geo = [pipe.geometry(b) for b in (0, 1)]
    pipe.close()
    for blk, (delays, maxd, ts, sf) in enumerate(refs):
        D, O, nout, nd = geo[blk]
        assert O == maxd and nout == D // ts
        nk = (total - O) // D
        assert len(got[blk]) == nk
        for k in range(nk):
            ref = oracle.idd(np.ascontiguousarray(stream[k * D:(k + 1) * D + O]), delays, maxd,
                             ts, sf)
            assert np.array_equal(_np(got[blk][k]), ref), (blk, k)
