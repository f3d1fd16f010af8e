"""The benchmark's own gulp through the pipeline, stage by stage against the
oracle on two of its channels: 64 antennas x 1024 beams x 64 channels x
65536 samples of the L-band subband at 1284 MHz, coherent DMs {0, 50, 150,
500}, Stokes I, tscrunch 16, the synthetic inputs of the benchmark (sigma-8
voltages, 20-sigma RFI tones in channels 9, 27 and 45), the autotuned plan.

Checked on channels 0 (the lowest, the largest smear) and 9 (an RFI channel):
  * statistics within 1e-5 relative;
  * dedispersed voltages of every DM within one LSB of the FP64 oracle at the
    pipeline's plan, on at most 1e-5 of the values;
  * the coherent beams (all 1024) and incoherent beam power of a 4096-sample
    slice, from the pipeline's own voltages: bit-identical to the oracle;
  * from the oracle's voltages: differences only in flipped (time, channel)
    bins, by at most one LSB.
"""
import os
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CHANS = [0, 9]


def _wrapdiff(a, b):
    d = np.abs(a.astype(np.int64) - b.astype(np.int64))
    return np.minimum(d, 256 - d)


def test_headline_gulp_two_channels_stage_by_stage(cuda, oracle):
    torch = cuda
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    from skyweaver_b200 import stages, synthetic
    W = bench.WORK
    A, B, F, T, ts, dms = W["nant"], W["nbeams"], W["nchans"], W["gulp"], W["tscrunch"], W["dms"]
    centre, bw = bench.rank_subband(0, 1)
    g = synthetic.rng(1000)
    delays = synthetic.delay_model(g, B, A)
    gen = torch.Generator(device="cuda").manual_seed(1234)
    taftp = bench.workload_gulp(torch, gen, centre, bw, pulse=False)
    mapping = np.zeros(B, np.int32)
    bwts = np.ones((1, A), np.float32)
    pipe = stages.BeamformerPipeline(nantennas=A, input_nantennas=A, nchans=F, nbeams=B,
                                     gulp_samples=T, tscrunch=ts, centre_frequency=centre,
                                     bandwidth=bw, dms=dms, beamset_weights=bwts,
                                     beamset_mapping=mapping, autotune=True)
    epoch = 1.7e9
    pipe.set_delays(delays, epoch)
    pipe.process_device(taftp, epoch)
    fft_len, overlap, lag = pipe.cdd_plan()
    outs = [pipe.outputs(d) for d in range(len(dms))]
    volts = [pipe.voltages(d, CHANS) for d in range(len(dms))]   # [C][P][A][2][T]
    pipe.close()
    sub = np.ascontiguousarray(taftp[:, :, CHANS].cpu().numpy())  # TAFTP of the two channels
    del taftp
    ftpa = oracle.transpose(sub, A)                               # [C][T][P][A][2]
    st = oracle.statistics(ftpa)
    np.testing.assert_allclose(outs[0]["stats"][CHANS], st, rtol=1e-5, atol=1e-6)
    scl = oracle.scalings(outs[0]["stats"][CHANS], bwts, 1, ts, ts, 24.0)
    freqs = synthetic.channel_frequencies(centre, bw, F)[CHANS]
    w = oracle.weights(delays, freqs, epoch, epoch)
    low = float(np.float32(centre - bw / 2))
    ext = np.concatenate([np.zeros((len(CHANS), overlap, 2, A, 2), np.int8), ftpa], axis=1)
    t0, nt = 30720, 4096                                          # the compared slice
    sl = slice(t0 // ts, (t0 + nt) // ts)
    for d, dm in enumerate(dms):
        chirps = oracle.chirp(F, fft_len, low, bw, dm)[CHANS]
        ref = oracle.cdd_ftpa(ext, T, chirps, overlap, lag=lag)
        got = np.ascontiguousarray(volts[d].transpose(0, 4, 1, 2, 3))
        dv = _wrapdiff(got, ref)
        nflip = int((dv > 0).sum())
        print(f"DM {dm}: {nflip} of {dv.size} dedispersed values one LSB off the FP64 oracle")
        assert dv.max() <= 1 and nflip <= 1e-5 * dv.size
        for name, v in (("own", got), ("oracle", ref)):
            vs = np.ascontiguousarray(v[:, t0:t0 + nt])
            raw, _ = oracle.incoherent_beam(vs, ts, scl[3], scl[2], bwts, 1)
            cb = oracle.coherent_beam(vs, w, ts, scl[1], scl[0], bwts, mapping)
            gcb = outs[d]["cb"][sl][:, CHANS]
            graw = outs[d]["ib_raw"][:, sl][:, :, CHANS]
            if name == "own":
                assert np.array_equal(gcb, cb)
                assert np.array_equal(graw, raw)
            else:
                dcb = np.abs(gcb.astype(int) - cb.astype(int))
                flips = dv[:, t0:t0 + nt].any(axis=(2, 3, 4)).reshape(len(CHANS), -1, ts).any(-1).T
                print(f"DM {dm}: {(dcb > 0).sum()} of {dcb.size} beams differ from the oracle "
                      f"chain, in {flips.sum()} flipped (time, channel) bins")
                assert dcb.max() <= 1
                assert not (dcb.any(-1) & ~flips).any()
