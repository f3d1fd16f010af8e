"""End-to-end parity of the graph-captured BeamformerPipeline against the
oracle chain over consecutive gulps (overlap-save history carried across
gulps, scalings fixed from gulp 0 like BeamformerPipeline.cu:171-176).

The chain is checked stage by stage on the same inputs:
  * the dedispersed voltages against the FP64 oracle at the pipeline's own
    plan: DM 0 identical (its chirp is exactly 1), other DMs at most one LSB
    apart on at most 1e-5 of the values;
  * the incoherent and coherent beams of the pipeline's own voltages against
    the oracle's beams of those voltages: bit-identical;
  * the beams of the oracle's voltages: a beam sample can differ only in a
    (channel, time bin) where a voltage differs, and by at most one LSB.
"""
import math
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _run(cuda, oracle, use_graph, grouped, tones=False):
    torch = cuda
    from skyweaver_b200 import stages, synthetic
    g = synthetic.rng(77)
    A_in, A, F, B, T, ts = 13, 16, 4, 64, 4096, 4
    chbw = 856e6 / 1024
    centre, bw = 1284e6, F * chbw
    dms = [0.0, 10.0]
    mapping = np.zeros(B, np.int32)
    mapping[40:] = 1
    masks = np.ones((2, A), np.float32)
    masks[:, A_in:] = 0
    masks[1, :5] = 0
    delays = synthetic.delay_model(g, B, A)
    delays[..., 0] = masks[mapping]
    pipe = stages.BeamformerPipeline(nantennas=A, input_nantennas=A_in, nchans=F, nbeams=B,
                                     gulp_samples=T, tscrunch=ts, centre_frequency=centre,
                                     bandwidth=bw, dms=dms, beamset_weights=masks,
                                     beamset_mapping=mapping, use_graph=use_graph,
                                     grouped=grouped)
    epoch0, delay_epoch = 1.7e9, 1.7e9 - 3.0
    pipe.set_delays(delays, delay_epoch)
    fft_len, overlap, lag = pipe.cdd_plan()
    assert 0 < lag < overlap < fft_len
    freqs = synthetic.channel_frequencies(centre, bw, F)
    low = float(np.float32(centre - bw / 2))
    chirps = [oracle.chirp(F, fft_len, low, bw, d) for d in dms]
    history = np.zeros((F, overlap, 2, A, 2), np.int8)
    scl = None
    results = []
    for gulp in range(3):
        taftp = synthetic.voltages_taftp(g, T // 256, A_in, F, sigma=10)
        if tones:  # saturated channels: the incoherent beam takes them first
            synthetic.inject_tones(taftp, [1, 3], amplitude=160.0)
        epoch = epoch0 + gulp * T / chbw
        pipe.process_device(torch.from_numpy(taftp).cuda(), epoch)
        ftpa = oracle.transpose(taftp, A)
        stats_ref = oracle.statistics(ftpa)
        out0 = pipe.outputs(0)
        stats_gpu = pipe_stats(pipe, F, A)
        np.testing.assert_allclose(stats_gpu, stats_ref, rtol=1e-5, atol=1e-6)
        if scl is None:  # scalings come from gulp 0's statistics
            scl = oracle.scalings(stats_gpu, masks, 2, ts, ts, 24.0)
        w = oracle.weights(delays, freqs, epoch, delay_epoch)
        ext = np.concatenate([history, ftpa], axis=1)
        history = ext[:, -overlap:].copy() if overlap else history
        for d, dm in enumerate(dms):
            r = {"dm": dm, "out": out0 if d == 0 else pipe.outputs(d)}
            r["v_ref"] = oracle.cdd_ftpa(ext, T, chirps[d], overlap, lag=lag)
            r["v_gpu"] = np.ascontiguousarray(pipe.voltages(d).transpose(0, 4, 1, 2, 3))
            for key, v in (("ref", r["v_ref"]), ("own", r["v_gpu"])):
                r["raw_" + key], r["ib_" + key] = oracle.incoherent_beam(v, ts, scl[3], scl[2],
                                                                         masks, 2)
                r["cb_" + key] = oracle.coherent_beam(v, w, ts, scl[1], scl[0], masks, mapping)
            results.append(r)
    pipe.close()
    return results, ts


def pipe_stats(pipe, F, A):
    import ctypes
    from skyweaver_b200._lib import call
    from skyweaver_b200.stages import _device_view
    ptrs = [ctypes.c_void_p() for _ in range(4)]
    call("sw_pipeline_outputs", pipe.h, 0, *[ctypes.byref(p) for p in ptrs])
    n = F * 2 * A * 4
    return _device_view(ptrs[3].value, n * 4).cpu().numpy().view(np.float32).reshape(F, 2, A, 4)


@pytest.mark.parametrize("use_graph,grouped,tones",
                         [(True, True, False), (False, False, False), (True, True, True)])
def test_pipeline_matches_oracle_chain(cuda, oracle, use_graph, grouped, tones):
    results, ts = _run(cuda, oracle, use_graph, grouped, tones)
    for r in results:
        out = r["out"]
        # beams of the pipeline's own voltages: bit-identical
        assert np.array_equal(out["cb"], r["cb_own"])
        assert np.array_equal(out["ib_raw"], r["raw_own"])
        assert np.array_equal(out["ib"], r["ib_own"])
        # voltages against the FP64 oracle at the same plan
        dv = np.abs(r["v_gpu"].astype(int) - r["v_ref"].astype(int))
        dv = np.minimum(dv, 256 - dv)  # int8 wrap: -128 and 127 are one LSB apart
        nflip = int((dv > 0).sum())
        print(f"DM {r['dm']}: {nflip} of {dv.size} dedispersed values one LSB off")
        if r["dm"] == 0.0:
            assert nflip == 0
            assert np.array_equal(out["cb"], r["cb_ref"])
            assert np.array_equal(out["ib_raw"], r["raw_ref"])
            continue
        assert dv.max() <= 1 and nflip <= 1e-5 * dv.size, (int(dv.max()), nflip)
        # beams of the oracle's voltages: differences only where a voltage
        # differs, by at most one LSB
        flip_bins = (dv.any(axis=(2, 3, 4)).reshape(dv.shape[0], -1, ts).any(-1)).T  # [T'][F]
        dcb = np.abs(out["cb"].astype(int) - r["cb_ref"].astype(int))
        print(f"DM {r['dm']}: {(dcb > 0).sum()} of {dcb.size} coherent beams differ "
              f"(in {flip_bins.sum()} flipped (time, channel) bins)")
        assert dcb.max() <= 1
        assert not (dcb.any(-1) & ~flip_bins).any()
        draw = out["ib_raw"] != r["raw_ref"]
        assert not (draw.any(0) & ~flip_bins).any()


def test_ragged_beamsets_grouped_equals_plain_and_oracle(cuda, oracle):
    """Ragged (DM x beamset) problems: 8 beamsets with antenna masks of
    {64,57,48,40,32,24,16,8} antennas and {512,...,32} beams, 2 DMs.  The
    grouped launch (tiles packed across beamset boundaries) and the plain
    per-(DM, beamset) launches must agree bit for bit on every DM, and DM 0
    must equal the oracle chain."""
    torch = cuda
    from skyweaver_b200 import stages, synthetic
    g = synthetic.rng(2024)
    A, F, T, ts = 64, 2, 2048, 16
    ants = [64, 57, 48, 40, 32, 24, 16, 8]
    beams = [512, 256, 256, 128, 128, 64, 64, 32]
    B = sum(beams)
    masks = synthetic.beamset_masks(g, A, ants)
    mapping = np.repeat(np.arange(len(beams), dtype=np.int32), beams)
    delays = synthetic.delay_model(g, B, A)
    delays[..., 0] = masks[mapping]
    chbw = 856e6 / 1024
    centre, bw = 1284e6, F * chbw
    dms = [0.0, 50.0]
    taftp = synthetic.voltages_taftp(g, T // 256, A, F, sigma=8)
    outs = {}
    for name, kw in (("grouped", dict(grouped=True, use_graph=True)),
                     ("plain", dict(grouped=False, use_graph=False))):
        pipe = stages.BeamformerPipeline(nantennas=A, input_nantennas=A, nchans=F, nbeams=B,
                                         gulp_samples=T, tscrunch=ts, centre_frequency=centre,
                                         bandwidth=bw, dms=dms, beamset_weights=masks,
                                         beamset_mapping=mapping, **kw)
        pipe.set_delays(delays, 1.7e9)
        fft_len, overlap, lag = pipe.cdd_plan()
        pipe.process_device(torch.from_numpy(taftp).cuda(), 1.7e9)
        outs[name] = [pipe.outputs(d) for d in range(len(dms))]
        # the DescribedVector metadata of the outputs
        d = pipe.describe_cb(1)
        assert d["dims"] == "TFB" and d["extents"] == (T // ts, F, B)
        assert d["reference_dm"] == 50.0 and abs(d["tsamp"] - ts / chbw) < 1e-15
        assert abs(d["utc_offset"] - lag / chbw) < 1e-15
        assert pipe.describe_ib(0)["extents"] == (len(beams), T // ts, F)
        pipe.close()
    for a, b in zip(outs["grouped"], outs["plain"]):
        assert np.array_equal(a["cb"], b["cb"])
        assert np.array_equal(a["ib_raw"], b["ib_raw"])
    ftpa = oracle.transpose(taftp, A)
    scl = oracle.scalings(oracle.statistics(ftpa), masks, len(beams), ts, ts, 24.0)
    freqs = synthetic.channel_frequencies(centre, bw, F)
    w = oracle.weights(delays, freqs, 1.7e9, 1.7e9)
    # first gulp: zero history, DM 0 output delayed by the plan's lag
    ext = np.concatenate([np.zeros((F, overlap, 2, A, 2), np.int8), ftpa], axis=1)
    low = float(np.float32(centre - bw / 2))
    dd = oracle.cdd_ftpa(ext, T, oracle.chirp(F, fft_len, low, bw, 0.0), overlap, lag=lag)
    cb_ref = oracle.coherent_beam(dd, w, ts, scl[1], scl[0], masks, mapping)
    assert np.array_equal(outs["grouped"][0]["cb"], cb_ref)


def test_pipeline_full_stokes_iquv(cuda, oracle):
    """Stokes IQUV through the pipeline: char4 coherent beams, float4/char4
    incoherent beams, DM 0 bit-identical to the oracle chain."""
    torch = cuda
    from skyweaver_b200 import stages, synthetic
    g = synthetic.rng(78)
    A, F, B, T, ts = 32, 2, 128, 2048, 8
    chbw = 856e6 / 1024
    centre, bw = 1284e6, F * chbw
    mapping = np.zeros(B, np.int32)
    mapping[70:] = 1
    masks = synthetic.beamset_masks(g, A, [32, 20])
    delays = synthetic.delay_model(g, B, A)
    delays[..., 0] = masks[mapping]
    pipe = stages.BeamformerPipeline(nantennas=A, input_nantennas=A, nchans=F, nbeams=B,
                                     gulp_samples=T, tscrunch=ts, centre_frequency=centre,
                                     bandwidth=bw, dms=[0.0], beamset_weights=masks,
                                     beamset_mapping=mapping, stokes="IQUV")
    pipe.set_delays(delays, 1.7e9)
    taftp = synthetic.voltages_taftp(g, T // 256, A, F, sigma=8)
    pipe.process_device(torch.from_numpy(taftp).cuda(), 1.7e9)
    out = pipe.outputs(0)
    pipe.close()
    ftpa = oracle.transpose(taftp, A)
    scl = oracle.scalings(oracle.statistics(ftpa), masks, 2, ts, ts, 24.0)
    w = oracle.weights(delays, synthetic.channel_frequencies(centre, bw, F), 1.7e9, 1.7e9)
    raw_ref, ib_ref = oracle.incoherent_beam(ftpa, ts, scl[3], scl[2], masks, 2, "IQUV")
    cb_ref = oracle.coherent_beam(ftpa, w, ts, scl[1], scl[0], masks, mapping, "IQUV")
    assert out["cb"].shape == (T // ts, F, B, 4)
    assert np.array_equal(out["ib_raw"], raw_ref)
    assert np.array_equal(out["ib"], ib_ref)
    assert np.array_equal(out["cb"], cb_ref)


def test_dispersed_pulse_peaks_in_its_dm_fft65536(cuda, oracle):
    """Coherent dedispersion with 2^16-point FFTs in the pipeline: a burst
    dispersed within each channel at DM 150 (by the conjugate of the DM 150
    response, i.e. what the sky does) and arriving at boresight must come out
    strongest in the DM 150 coherent beam, and be re-compressed there."""
    torch = cuda
    from skyweaver_b200 import stages, synthetic
    g = synthetic.rng(150)
    A, F, B, T, ts, N = 16, 4, 32, 65536, 16, 65536
    dms = [0.0, 50.0, 150.0, 500.0]
    chbw = 856e6 / 1024
    bw = F * chbw
    centre = 1284e6 - 30 * chbw                  # bottom of the L-band subband
    low = float(np.float32(centre - bw / 2))
    # noise + a 32-sample burst at t0, dispersed per channel at DM 150
    v = g.normal(0, 8, size=(F, T, 2, A, 2))
    t0, W, amp = 30000, 32, 4.0
    H = oracle.chirp(F, N, low, bw, 150.0)       # DM 150 dedispersion response
    for c in range(F):
        burst = np.zeros(N, np.complex128)
        burst[t0 % N: t0 % N + W] = amp
        disp = np.fft.ifft(np.fft.fft(burst) * np.conj(H[c]))
        v[c, :N, :, :, 0] += disp.real[:, None, None]
        v[c, :N, :, :, 1] += disp.imag[:, None, None]
    ftpa = np.clip(np.rint(v), -127, 127).astype(np.int8)          # [F][T][P][A][2]
    taftp = ftpa.reshape(F, T // 256, 256, 2, A, 2).transpose(1, 4, 0, 2, 3, 5).copy()
    delays = synthetic.delay_model(g, B, A)
    delays[0] = [1.0, 0.0, 0.0]                  # beam 0 at boresight
    mapping = np.zeros(B, np.int32)
    pipe = stages.BeamformerPipeline(nantennas=A, input_nantennas=A, nchans=F, nbeams=B,
                                     gulp_samples=T, tscrunch=ts, centre_frequency=centre,
                                     bandwidth=bw, dms=dms, beamset_weights=np.ones((1, A)),
                                     beamset_mapping=mapping, fft_len=N)
    assert pipe.fft_plan()[0] == N
    pipe.set_delays(delays, 1.7e9)
    pipe.process_device(torch.from_numpy(taftp).cuda(), 1.7e9)
    series = []
    for d in range(len(dms)):
        cb = pipe.outputs(d)["cb"][:, :, 0].astype(np.float64).sum(axis=1)   # [T/ts]
        series.append(np.convolve(cb, np.ones(2), "valid"))                 # 2-bin boxcar
    pipe.close()
    peaks = [s.max() for s in series]
    print("boxcar peak per DM:", dict(zip(dms, peaks)))
    assert int(np.argmax(peaks)) == dms.index(150.0), peaks
    # re-compressed: the DM 150 peak stands well above its own noise
    s = series[2]
    assert (s.max() - np.median(s)) > 6 * s.std()


def test_autotune_choices_and_results(cuda, oracle):
    """sw_autotune picks a valid FFT length and beamformer work-item size for
    the shape, caches it, and a pipeline built with autotune gives the same
    beams as the default plan (DM 0 is exact for any FFT length; the
    work-item size never changes results)."""
    torch = cuda
    import time
    from skyweaver_b200 import stages, synthetic
    g = synthetic.rng(91)
    A, F, B, T, ts = 32, 4, 256, 8192, 16
    chbw = 856e6 / 1024
    centre, bw = 1284e6, F * chbw
    dms = [0.0, 150.0]
    t = stages.autotune(A, B, F, T, ts, dms, centre, bw)
    assert t["fft_len"] > t["overlap"] and t["fft_len"] & (t["fft_len"] - 1) == 0
    assert t["cb_tiles_per_item"] in (4, 8, 16, 32, 64, 128)
    assert (t["cb_voltage_stages"], t["cb_weight_stages"]) in (
        (4, 2), (2, 2), (3, 2), (6, 2), (8, 2), (4, 3), (6, 3))
    assert t["cdd_ms"] > 0 and t["cb_ms"] > 0
    t0 = time.perf_counter()
    assert stages.autotune(A, B, F, T, ts, dms, centre, bw) == t      # cached
    assert time.perf_counter() - t0 < 0.05
    taftp = synthetic.voltages_taftp(g, T // 256, A, F, sigma=8)
    delays = synthetic.delay_model(g, B, A)
    outs = []
    for tune in (False, True):
        pipe = stages.BeamformerPipeline(nantennas=A, input_nantennas=A, nchans=F, nbeams=B,
                                         gulp_samples=T, tscrunch=ts, centre_frequency=centre,
                                         bandwidth=bw, dms=dms, beamset_weights=np.ones((1, A)),
                                         beamset_mapping=np.zeros(B, np.int32), autotune=tune)
        if tune:
            assert pipe.fft_plan()[0] == t["fft_len"]
        pipe.set_delays(delays, 1.7e9)
        pipe.process_device(torch.from_numpy(taftp).cuda(), 1.7e9)
        outs.append(pipe.outputs(0)["cb"])
        pipe.close()
    assert np.array_equal(outs[0], outs[1])


def test_uhf_pipeline_with_incoherent_dedispersion_vs_oracle(cuda, oracle):
    """UHF end-to-end chain, reduced: 16 channels at the top of the 544-1088
    MHz band (1024-channel mode), 16 antennas, 32 beams, coherent DMs {0, 300},
    tscrunch 8, then the device incoherent-dedispersion pipeline with 9 trial
    DMs around each coherent DM.  A pulse dispersed at DM 300 (intra-channel
    by the conjugate DM 300 response, inter-channel by the incoherent delays)
    arrives at boresight.  The GPU TDB must match the oracle chain (exact for
    the DM 0 block, within one LSB on a small fraction for DM 300), and both
    must recover the pulse at the trial nearest DM 300 with the same S/N.
    Stage by stage: the dedispersed voltages are within one LSB of the FP64
    oracle on at most 1e-5 of the values, the coherent beams of the
    pipeline's own voltages and their incoherent dedispersion are
    bit-identical to the oracle's."""
    torch = cuda
    from skyweaver_b200 import stages, synthetic
    g = synthetic.rng(300)
    A, F, B, T, ts = 16, 16, 32, 32768, 8
    chbw = 0.53125e6
    top = 1088e6
    bw = F * chbw
    centre = top - bw / 2
    low = float(np.float32(centre - bw / 2))
    freqs = synthetic.channel_frequencies(centre, bw, F)
    coh = [0.0, 300.0]
    trials = [np.linspace(-10, 10, 9).astype(np.float32) + c for c in coh]
    trials[0] = np.abs(trials[0])
    cb_tsamp = ts / chbw
    idd = [oracle.idd_delays(freqs, tr, cb_tsamp) for tr in trials]
    # the pulse: 64 raw samples, lowest channel at raw time t_low
    maxd1 = idd[1][1]
    t_low = 8 * (maxd1 + 900)
    v = g.normal(0, 8, size=(F, T, 2, A, 2))
    H = oracle.chirp(F, T, low, bw, 300.0)
    k = 4.148806423e15
    for c in range(F):
        shift = int(round(k * 300.0 * (1 / freqs[0] ** 2 - 1 / freqs[c] ** 2) * chbw))
        burst = np.zeros(T, np.complex128)
        burst[t_low - shift: t_low - shift + 64] = 6.0
        disp = np.fft.ifft(np.fft.fft(burst) * np.conj(H[c]))
        v[c, :, :, :, 0] += disp.real[:, None, None]
        v[c, :, :, :, 1] += disp.imag[:, None, None]
    ftpa = np.clip(np.rint(v), -127, 127).astype(np.int8)
    taftp = ftpa.reshape(F, T // 256, 256, 2, A, 2).transpose(1, 4, 0, 2, 3, 5).copy()
    delays = synthetic.delay_model(g, B, A)
    delays[0] = [1.0, 0.0, 0.0]                  # beam 0 at boresight
    bw1 = np.ones((1, A), np.float32)
    mapping = np.zeros(B, np.int32)
    pipe = stages.BeamformerPipeline(nantennas=A, input_nantennas=A, nchans=F, nbeams=B,
                                     gulp_samples=T, tscrunch=ts, centre_frequency=centre,
                                     bandwidth=bw, dms=coh, beamset_weights=bw1,
                                     beamset_mapping=mapping)
    fft_len, overlap, lag = pipe.cdd_plan()
    pipe.set_delays(delays, 1.7e9)
    pipe.process_device(torch.from_numpy(taftp).cuda(), 1.7e9)
    cbs = [pipe.outputs(d)["cb"] for d in range(2)]
    volts = [np.ascontiguousarray(pipe.voltages(d).transpose(0, 4, 1, 2, 3)) for d in range(2)]
    pipe.close()
    sf = [float(np.float32(math.sqrt(F * 1))) for _ in coh]
    got = {0: [], 1: []}
    idp = stages.IncoherentDedispersionPipeline(
        F, B, [(idd[b][0], 1, sf[b]) for b in range(2)],
        lambda b, t: got[b].append(t.cpu().numpy()), dispatch=[2048, 2048])
    for d in range(2):
        idp.push(d, torch.from_numpy(np.ascontiguousarray(cbs[d])).cuda())
    idp.close()
    # oracle chain
    ext = np.concatenate([np.zeros((F, overlap, 2, A, 2), np.int8), ftpa], axis=1)
    scl = oracle.scalings(oracle.statistics(ftpa), bw1, 1, ts, ts, 24.0)
    w = oracle.weights(delays, freqs, 1.7e9, 1.7e9)
    snr = []
    for d, dm in enumerate(coh):
        dd = oracle.cdd_ftpa(ext, T, oracle.chirp(F, fft_len, low, bw, dm), overlap, lag=lag)
        dv = np.abs(volts[d].astype(int) - dd.astype(int))
        dv = np.minimum(dv, 256 - dv)
        print(f"UHF DM {dm}: {(dv > 0).sum()} of {dv.size} dedispersed values one LSB off")
        assert dv.max() <= 1 and (dv > 0).sum() <= 1e-5 * dv.size
        cb_own = oracle.coherent_beam(volts[d], w, ts, scl[1], scl[0], bw1, mapping)
        assert np.array_equal(cbs[d], cb_own)
        cb_ref = oracle.coherent_beam(dd, w, ts, scl[1], scl[0], bw1, mapping)
        if d == 0:
            assert np.array_equal(cbs[0], cb_ref)
        delays_d, maxd = idd[d]
        D = 2048
        assert len(got[d]) == 1
        tdb = got[d][0]
        own = oracle.idd(np.ascontiguousarray(cbs[d][:D + maxd]), delays_d, maxd, 1, sf[d])
        assert np.array_equal(tdb, own)
        ref = oracle.idd(np.ascontiguousarray(cb_ref[:D + maxd]), delays_d, maxd, 1, sf[d])
        dt = np.abs(tdb.astype(int) - ref.astype(int))
        print(f"UHF DM {dm}: {(dt > 0).sum()} of {dt.size} TDB values differ from the "
              f"oracle chain (max {dt.max()})")
        row = []
        for arr in (tdb, ref):
            # boresight beam, 8-sample boxcar (the pulse width): int8 outputs
            # saturate at 127, so single samples cap the S/N near 5
            s = arr[:, :, 0].astype(np.float64)          # [t][trial]
            s = np.stack([np.convolve(s[:, j], np.ones(8), "valid") for j in range(s.shape[1])], 1)
            base = np.median(s, axis=0)
            noise = s.std(axis=0)
            row.append(((s - base) / noise).max(axis=0))
        snr.append(row)
    gpu, cpu = snr[1]
    best = int(np.argmax(gpu))
    print("DM 300 block S/N per trial: gpu", np.round(gpu, 1), "cpu", np.round(cpu, 1))
    assert best == int(np.argmin(np.abs(trials[1] - 300.0)))
    assert gpu[best] > 8 and abs(gpu[best] - cpu[best]) < 0.05 * cpu[best]


def test_dada_files_through_pipeline_to_dada_outputs(cuda, tmp_path):
    """DADA ingest -> pipeline -> DADA output: TAFTP gulps read from two
    contiguous DADA files by the pinned double-buffered gulp reader, run
    through the host API, and each coherent DM's beams written as size-split
    DADA streams; the written payload equals the beams of the same gulps run
    from device memory."""
    torch = cuda
    from skyweaver_b200 import dada, stages, synthetic
    from test_dada_io import _header
    g = synthetic.rng(5150)
    A, F, B, T, ts = 32, 4, 64, 4096, 16
    chbw = 856e6 / 1024
    centre, bw = 1284e6, F * chbw
    dms = [0.0, 30.0]
    ngulps = 3
    gulps = [synthetic.voltages_taftp(g, T // 256, A, F, sigma=8) for _ in range(ngulps)]
    payload = np.concatenate([x.reshape(-1) for x in gulps])
    cut = payload.size // 2 + 123
    files = []
    for i, (a, b) in enumerate(((0, cut), (cut, payload.size))):
        p = tmp_path / f"in{i}.dada"
        p.write_bytes(_header(a, NCHAN=str(F), NANT=str(A)) + payload[a:b].tobytes())
        files.append(str(p))
    delays = synthetic.delay_model(g, B, A)
    kw = dict(nantennas=A, input_nantennas=A, nchans=F, nbeams=B, gulp_samples=T, tscrunch=ts,
              centre_frequency=centre, bandwidth=bw, dms=dms, beamset_weights=np.ones((1, A)),
              beamset_mapping=np.zeros(B, np.int32))
    # reference: the same gulps from device memory
    ref = [[] for _ in dms]
    pipe = stages.BeamformerPipeline(**kw)
    pipe.set_delays(delays, 1.7e9)
    for i, x in enumerate(gulps):
        pipe.process_device(torch.from_numpy(x).cuda(), 1.7e9 + i * T / chbw)
        for d in range(len(dms)):
            ref[d].append(pipe.outputs(d)["cb"])
    pipe.close()
    # DADA in -> host API -> DADA out
    reader = dada.MultiFileReader(files, check_contiguity=True)
    hdr = reader.header().as_dict()
    dada.validate_header(reader.header(), A, F, 2)
    pipe = stages.BeamformerPipeline(**kw)
    pipe.set_delays(delays, 1.7e9)
    per_dm = pipe.cb_bytes_per_dm()
    out = torch.empty(per_dm * len(dms), dtype=torch.int8, pin_memory=True)
    writers = []
    for d, dm in enumerate(dms):
        dr, base, ext = dada.output_paths(str(tmp_path / "out"), hdr, d, dm, "TFB")
        w = dada.FileStream(dr, base, ext, 2 * per_dm)
        w.set("NBEAM", B)
        w.set("COHERENT_DM", dm)
        writers.append((w, dr))
    gr = dada.GulpReader(reader, payload.size // ngulps)
    n = 0
    for buf, i in gr:
        pipe.process_host(buf, 1.7e9 + i * T / chbw, out)
        torch.cuda.synchronize()
        host = out.numpy()
        for d, (w, _) in enumerate(writers):
            w.write(host[d * per_dm:(d + 1) * per_dm])
        n += 1
    gr.close()
    reader.close()
    pipe.close()
    assert n == ngulps
    for d, (w, dr) in enumerate(writers):
        w.close()
        names = sorted(os.listdir(dr))
        assert len(names) == 2                       # 3 gulps in files of 2 gulps
        data = b"".join(open(os.path.join(dr, nm), "rb").read()[4096:] for nm in names)
        assert data == np.concatenate([r.reshape(-1) for r in ref[d]]).tobytes()


def test_host_path_several_gulps_in_flight_keep_their_epochs(cuda):
    """process_host with several gulps enqueued before one synchronisation:
    every gulp's weights must use that gulp's own epoch.  The delay model has
    non-zero rates, so the epochs (1000 s apart) change the weights; the
    beams of each gulp must equal those of a run that synchronises after
    every gulp."""
    torch = cuda
    from skyweaver_b200 import stages, synthetic
    g = synthetic.rng(4242)
    A, F, B, T, ts = 16, 2, 64, 2048, 16
    chbw = 856e6 / 1024
    delays = synthetic.delay_model(g, B, A)
    delays[..., 2] = g.uniform(-2e-9, 2e-9, size=(B, A))           # delay rates (s/s)
    kw = dict(nantennas=A, input_nantennas=A, nchans=F, nbeams=B, gulp_samples=T, tscrunch=ts,
              centre_frequency=1284e6, bandwidth=F * chbw, dms=[0.0],
              beamset_weights=np.ones((1, A)), beamset_mapping=np.zeros(B, np.int32))
    ngulp = 6
    # the same voltages every gulp: only the epochs tell the gulps apart
    x = torch.empty((T // 256, A, F, 256, 2, 2), dtype=torch.int8, pin_memory=True)
    x.copy_(torch.from_numpy(synthetic.voltages_taftp(g, T // 256, A, F, sigma=8)))
    ins = [x] * ngulp
    epochs = [1.7e9 + 1000.0 * i for i in range(ngulp)]
    res = {}
    for mode in ("sync_each", "all_in_flight"):
        pipe = stages.BeamformerPipeline(**kw)
        pipe.set_delays(delays, 1.7e9)
        outs = [torch.empty(pipe.cb_bytes_per_dm(), dtype=torch.int8, pin_memory=True)
                for _ in range(ngulp)]
        for i in range(ngulp):
            pipe.process_host(ins[i], epochs[i], outs[i])
            if mode == "sync_each":
                torch.cuda.synchronize()
        torch.cuda.synchronize()
        res[mode] = [o.numpy().copy() for o in outs]
        pipe.close()
    for i in range(ngulp):
        assert np.array_equal(res["sync_each"][i], res["all_in_flight"][i]), i
    # the epochs do change the beams
    assert not np.array_equal(res["sync_each"][0], res["sync_each"][2])
