#!/usr/bin/env python3
"""Benchmark of the B200 skyweaver beamforming pipeline.

Workload (one "step" = one gulp through the whole stage chain):
  64 antennas x 1024 coherent beams (+ incoherent beam) x 64 channels of the
  MeerKAT L-band 1024-channel mode at 1284 MHz (0.8359375 MHz channels,
  1.196 us samples), 2 pols, 65536-sample gulps, 4 coherent DMs
  {0, 50, 150, 500} pc cm^-3, Stokes I, tscrunch 16, int8 TFB output.
  Synthetic seeded complex-Gaussian int8 voltages (sigma 8) and delays from a
  random 8 km array and beams within 0.5 deg (no recordings are available).

value  = real-time factor of the batched, graph-captured pipeline with the
         gulp already in HBM (data seconds processed per wall second, summed
         over ranks; every rank processes its own subband: weak scaling).
e2e    = the same through the public host API (pinned TAFTP H2D and the D2H
         of every DM's coherent-beam output inside the timed region).
Secondary lines in the same JSON object: the plain (eager, per-DM) pipeline,
the per-kernel breakdown, ragged beamsets (8 beamsets x 4 DMs, grouped vs
plain), long_fft (256 beams with 65536-point dedispersion windows) and uhf
(UHF band, 2048 beams, device incoherent dedispersion of 128 trial DMs).

python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

WORK = dict(nant=64, nbeams=1024, nchans=64, gulp=65536, tscrunch=16,
            dms=[0.0, 50.0, 150.0, 500.0], centre=1284e6, chbw=856e6 / 1024)
METRIC = "real-time factor & int8 TOPS, 64ant×1024beam×4DM: batched vs plain GPU"
# dram__bytes_read.sum + dram__bytes_write.sum of one cb_kernel<16,0> launch on
# the 16-channel, one-DM case of `bench.py --profile cb` (ncu --set full).
CB_NCU_BYTES_16CH_1DM = 273.172736e6 + 55.232512e6


def tsamp():
    return 1.0 / WORK["chbw"]


RFI_CHANNELS = (9, 27, 45)
UHF_RFI_CHANNELS = (40, 130, 200)
PULSE_EVERY = 20  # one gulp in 20 carries the DM-100 pulse (the step index = 10 mod 20)
INPUTS = ("complex Gaussian sigma 8 int8 voltages; narrowband RFI tones at 20 sigma in "
          "channels 9, 27 and 45; a DM-100 pulse (64 samples, +3 sigma) in every 20th gulp")


def add_rfi_tones(torch, v, channels, t0=0):
    """Narrowband RFI: a complex sinusoid of amplitude 160 per component (20
    sigma of the sigma-8 voltages, clipped by the int8 conversion) added to
    every antenna and pol of the given channels of a float TAFTP tensor
    [heap][antenna][channel][256][pol][re, im] whose first sample is sample
    `t0` of the stream."""
    t = torch.arange(v.shape[0] * 256, device=v.device, dtype=torch.float64) + t0
    t = t.reshape(v.shape[0], 256)
    for k, c in enumerate(channels):
        ph = torch.remainder((0.01 + 0.037 * k) * t, 1.0) * (2 * math.pi)
        tone = torch.stack([160.0 * torch.cos(ph), 160.0 * torch.sin(ph)], -1)  # [h][s][2]
        v[:, :, c] += tone[:, None, :, None, :].to(v.dtype)


def workload_gulp(torch, gen, centre, bwidth, pulse, device="cuda"):
    """One gulp of the benchmark workload on the device, TAFTP int8: complex
    Gaussian voltages (sigma 8 per component), three narrowband RFI tones at
    20 sigma and, when `pulse`, a DM-100 burst dispersed across the subband
    (arrival at the top channel a quarter into the gulp)."""
    from skyweaver_b200 import synthetic
    A, F, T = WORK["nant"], WORK["nchans"], WORK["gulp"]
    v = torch.randn((T // 256, A, F, 256, 2, 2), generator=gen, device=device) * 8.0
    add_rfi_tones(torch, v, RFI_CHANNELS)
    if pulse:
        freqs = synthetic.channel_frequencies(centre, bwidth, F)
        fref = freqs.max()
        for c, f in enumerate(freqs):
            s0 = T // 4 + int(round(synthetic.DM_CONST * 100.0 * (1 / f ** 2 - 1 / fref ** 2)
                                    / tsamp()))
            idx = torch.arange(s0, min(T, s0 + 64), device=device)
            if idx.numel():
                h, smp = idx // 256, idx % 256
                v[h, :, c, smp] += torch.randn((idx.numel(), A, 2, 2), generator=gen,
                                               device=device) * 24.0
    return v.round_().clamp_(-127, 127).to(torch.int8)


def config_block(extra=None):
    c = {"workload": "64ant x 1024beam x 64ch x 65536-sample gulps, 4 coherent DMs "
                     "{0,50,150,500}, Stokes I, tscrunch 16 (L-band 1284 MHz subband)",
         "nantennas": WORK["nant"], "nbeams": WORK["nbeams"], "nchans": WORK["nchans"],
         "gulp_samples": WORK["gulp"], "coherent_dms": WORK["dms"], "tscrunch": WORK["tscrunch"],
         "l2": "inputs larger than L2 (1.07 GB gulp per step)"}
    if extra:
        c.update(extra)
    return c


# ------------------------------------------------------------ CPU baseline
def cpu_baseline(threads=None, nsamp=2048):
    """Time the oracle (C restatement of the reference's CPU implementations)
    on a bounded sample: 1 channel x `nsamp` samples of a gulp through every
    stage of the chain (TAFTP -> FTPA transpose, statistics and scalings,
    weights of the 1024 beams, coherent dedispersion for 4 DMs, then per DM
    the incoherent beam and the coherent beamformer); RTF extrapolated
    linearly to 64 channels (every stage's cost is per channel)."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import concurrent.futures as cf

    import swb_oracle as O
    from skyweaver_b200 import synthetic
    O.build()
    threads = threads or os.cpu_count() or 1
    g = synthetic.rng(5)
    A, B, ts = WORK["nant"], WORK["nbeams"], WORK["tscrunch"]
    dms = WORK["dms"]
    chbw = WORK["chbw"]
    low = WORK["centre"] - 32 * chbw
    fft_len, ov, lag = O.cdd_plan(WORK["centre"], 64 * chbw, 64, dms)
    taftp = synthetic.voltages_taftp(g, nsamp // 256, A, 1)
    hist = np.clip(np.rint(g.normal(0, 8, size=(1, ov, 2, A, 2))), -127, 127).astype(np.int8)
    delays = synthetic.delay_model(g, B, A)
    freqs = np.array([low + chbw / 2])
    bw = np.ones((1, A), np.float32)
    mapping = np.zeros(B, np.int32)
    chirps = {d: O.chirp(1, fft_len, low, chbw, d) for d in dms}
    # tasks: (dm, stream) dedispersion, then (dm, time chunk) beamforming
    nchunk = max(1, min(threads, 16) // len(dms))
    stage = {}
    t0 = time.perf_counter()
    ftpa = O.transpose(taftp, A)
    t1 = time.perf_counter()
    scl = O.scalings(O.statistics(ftpa), bw, 1, ts, ts, 24.0)
    t2 = time.perf_counter()
    w = O.weights(delays, freqs, 0.0, 0.0)
    t3 = time.perf_counter()
    ext = np.concatenate([hist, ftpa], axis=1)
    dd = {}

    def cdd_task(d):
        return d, O.cdd_ftpa(ext, nsamp, chirps[d], ov, lag=lag)

    with cf.ThreadPoolExecutor(threads) as ex:
        for d, v in ex.map(cdd_task, dms):
            dd[d] = v
        t4 = time.perf_counter()

        def bf_task(args):
            d, c = args
            n = nsamp // nchunk
            x = np.ascontiguousarray(dd[d][:, c * n:(c + 1) * n])
            O.incoherent_beam(x, ts, scl[3], scl[2], bw, 1)
            return O.coherent_beam(x, w, ts, scl[1], scl[0], bw, mapping)

        list(ex.map(bf_task, [(d, c) for d in dms for c in range(nchunk)]))
    t5 = time.perf_counter()
    dt = t5 - t0
    stage = {"transpose": t1 - t0, "statistics_scalings": t2 - t1, "weights": t3 - t2,
             "coherent_dedispersion": t4 - t3, "beamformers": t5 - t4}
    data_s = nsamp * tsamp()
    rtf = data_s / (dt * WORK["nchans"])
    used = min(threads, len(dms) * nchunk)
    return {"value": rtf, "unit": "x real-time", "cores": used, "kind": "port",
            "sample": f"1 of 64 channels x {nsamp} samples through transpose, statistics, "
                      f"weights, 4-DM dedispersion and both beamformers (1024 beams): "
                      f"{dt:.2f} s on up to {used} threads, extrapolated x64 channels",
            "seconds": dt, "stage_seconds": {k: round(v, 4) for k, v in stage.items()}}


def cpu_baseline_median(threads=None, nsamp=2048, runs=3):
    """cpu_baseline after one untimed warm-up (thread pool, first-touch
    pages): the run with the median time of `runs`."""
    cpu_baseline(threads, nsamp=min(nsamp, 1024))
    vals = sorted((cpu_baseline(threads, nsamp) for _ in range(runs)), key=lambda x: x["seconds"])
    return vals[len(vals) // 2]


def cpu_baseline_bursts(bursts, threads=None):
    """The CPU side of C4's burst measurement: the oracle (C restatement of
    IncoherentDedisperser.cu:66-125, the reference's OpenMP host stage)
    dedisperses beam 0's coherent beams over each burst's window, and
    pulse_snr measures the burst on its output exactly as on the GPU's.
    Adds cpu_snr, cpu_trial and tdb_identical (the GPU's dedispersed window
    equals the oracle's byte for byte) to every measured burst."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import concurrent.futures as cf

    import swb_oracle as O
    O.build()
    tfb0, tdb0 = bursts["_tfb0"], bursts["_tdb0"]
    dl, maxd, sf = bursts["_delays"], bursts["_maxd"], bursts["_sf"]
    t0 = time.perf_counter()

    def one(r):
        if "gpu_snr" not in r:
            return
        lo, hi = r["centre"] - 16384, r["centre"] + 16384
        tdb = O.idd(np.ascontiguousarray(tfb0[lo:hi + maxd, :, None]), dl, maxd, 1, sf)[:, :, 0]
        snr, j, w, _ = pulse_snr(tdb, 16384)
        r.update(cpu_snr=round(snr, 3), cpu_trial=j, cpu_boxcar=w,
                 tdb_identical=bool(np.array_equal(tdb, tdb0[lo:hi])))

    with cf.ThreadPoolExecutor(threads or os.cpu_count() or 1) as ex:
        list(ex.map(one, bursts["pulses"]))
    bursts["cpu_seconds"] = round(time.perf_counter() - t0, 2)


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    for _ in range(args.warmup):
        cpu_baseline(nsamp=1024)
    vals = [cpu_baseline(nsamp=2048) for _ in range(args.steps)]
    v = float(np.median([x["value"] for x in vals]))
    ms = float(np.median([x["seconds"] for x in vals])) * 1e3
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "x real-time",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int8", "data": "synthetic",
            "config": config_block({"inputs": INPUTS}),
            "cpu_baseline": {"kind": vals[-1]["kind"], "cores": vals[-1]["cores"],
                             "sample": vals[-1]["sample"] + " (a Gaussian slice: the CPU path's "
                                       "cost does not depend on the values)",
                             "value": v, "unit": "x real-time"},
            "e2e": {"value": v, "unit": "x real-time", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- clocks
class Clocks:
    """SM clock, power and clock-event reasons sampled while the timed region
    runs: NVML every 10 ms from a thread (nvidia-smi -lms 200 if NVML is not
    importable).  summary() gives the median SM clock under load, the max
    clock and every slowdown reason seen."""

    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, index):
        self.index = index
        self.rows = []          # (sm_mhz, max_mhz, watts, reasons set)
        self.stop = threading.Event()
        self.thread = None
        self.p = None
        self.f = None

    def _nvml_handle(self, nv):
        try:
            import torch
            pr = torch.cuda.get_device_properties(self.index)
            bus = f"{pr.pci_domain_id:08X}:{pr.pci_bus_id:02X}:{pr.pci_device_id:02X}.0"
            return nv.nvmlDeviceGetHandleByPciBusId(bus.encode())
        except Exception:
            return nv.nvmlDeviceGetHandleByIndex(self.index)

    def _sample(self, nv, h):
        bits = {"hw_slowdown": nv.nvmlClocksEventReasonHwSlowdown,
                "hw_thermal_slowdown": nv.nvmlClocksEventReasonHwThermalSlowdown,
                "sw_thermal_slowdown": nv.nvmlClocksEventReasonSwThermalSlowdown,
                "sw_power_cap": nv.nvmlClocksEventReasonSwPowerCap}
        mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
        while not self.stop.is_set():
            try:
                sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                w = nv.nvmlDeviceGetPowerUsage(h) / 1000.0
                r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                self.rows.append((float(sm), float(mx), w, {n for n, b in bits.items() if r & b}))
            except Exception:
                pass
            self.stop.wait(0.01)

    def __enter__(self):
        try:
            import pynvml as nv
            nv.nvmlInit()
            h = self._nvml_handle(nv)
            self.thread = threading.Thread(target=self._sample, args=(nv, h), daemon=True)
            self.thread.start()
            return self
        except Exception:
            self.thread = None
        try:
            self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.p = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index),
                 "--query-gpu=clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None
        return self

    def __exit__(self, *a):
        if self.thread:
            self.stop.set()
            self.thread.join()
        if self.p:
            self.p.terminate()
            self.p.wait()

    def summary(self):
        rows = list(self.rows)
        if self.f is not None:
            self.f.flush()
            self.f.seek(0)
            for r in (r.split(",") for r in self.f.read().strip().splitlines() if r.strip()):
                try:
                    rows.append((float(r[0]), float(r[1]), float(r[2]),
                                 {n for n, v in zip(self.NAMES, r[4:8])
                                  if v.strip().lower() == "active"}))
                except (ValueError, IndexError):
                    pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        # the median under load: samples drawing more than half the peak power
        wmax = max(r[2] for r in rows)
        load = [r for r in rows if r[2] >= 0.5 * wmax] or rows
        return {"sm_mhz": float(np.median([r[0] for r in load])),
                "sm_max_mhz": float(max(r[1] for r in rows)),
                "reasons": sorted(set().union(*(r[3] for r in rows))),
                "samples": len(rows), "samples_under_load": len(load),
                "power_w_median": float(np.median([r[2] for r in load])),
                "source": "nvml 10 ms" if self.thread else "nvidia-smi 200 ms"}


# ------------------------------------------------------- rank decomposition
def rank_subband(rank, world):
    """Centre frequency and bandwidth of the subband that `rank` of `world`
    beamforms: adjacent, non-overlapping blocks of WORK["nchans"] channels
    centred on the band centre (weak scaling; subbands share no data, so
    no collective sits on the data path)."""
    bw = WORK["nchans"] * WORK["chbw"]
    return WORK["centre"] + (rank - (world - 1) / 2) * bw, bw


def max_over_ranks(value, world, device=None):
    """Max of a per-rank device time over the process group (the job takes
    as long as its slowest rank)."""
    if world == 1:
        return value
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ---------------------------------------------------------------- B200 arm
def main_b200(args):
    import torch
    import torch.distributed as dist

    from skyweaver_b200 import stages, synthetic
    from skyweaver_b200._lib import lib

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    A, B, F, T, ts = WORK["nant"], WORK["nbeams"], WORK["nchans"], WORK["gulp"], WORK["tscrunch"]
    dms = WORK["dms"]
    centre, bwidth = rank_subband(rank, world)
    g = synthetic.rng(1000 + rank)
    delays = synthetic.delay_model(g, B, A)
    gen = torch.Generator(device="cuda").manual_seed(1234 + rank)
    taftp = workload_gulp(torch, gen, centre, bwidth, pulse=False)
    taftp_pulse = workload_gulp(torch, gen, centre, bwidth, pulse=True)
    gulp = lambda i: taftp_pulse if i % PULSE_EVERY == 10 else taftp
    bwts = np.ones((1, A), np.float32)
    mapping = np.zeros(B, np.int32)
    common = dict(nantennas=A, input_nantennas=A, nchans=F, nbeams=B, gulp_samples=T,
                  tscrunch=ts, centre_frequency=centre, bandwidth=bwidth, dms=dms,
                  beamset_weights=bwts, beamset_mapping=mapping)
    # the autotuner picks the FFT length, the beamformer's work-item size and
    # its pipeline depths for this shape (cached for the process)
    if args.no_autotune:   # the cost model's FFT length and the kernel defaults
        tune = {"fft_len": 0, "cb_tiles_per_item": 0, "cb_voltage_stages": 0,
                "cb_weight_stages": 0}
    else:
        tune = stages.autotune(A, B, F, T, ts, dms, centre, bwidth)
    pipe = stages.BeamformerPipeline(**common, grouped=True, use_graph=True,
                                     autotune=not args.no_autotune)
    pipe.set_delays(delays, 1.7e9)
    fft_len, overlap, lag = pipe.cdd_plan()
    epoch0 = 1.7e9
    gulp_s = T * tsamp()
    stream = torch.cuda.current_stream()

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()

    def time_steps(fn, K, W):
        for i in range(W):
            fn(i)
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for i in range(K):
            fn(W + i)
        e1.record(stream)
        barrier()
        return max_over_ranks(e0.elapsed_time(e1), world, "cuda") / K

    # ---- headline: batched grouped CB + CUDA graph, input resident in HBM
    with Clocks(local) as clk:
        ms_graph = time_steps(lambda i: pipe.process_device(gulp(i), epoch0 + i * gulp_s),
                              args.steps, args.warmup)
    clocks = clk.summary()
    rtf = gulp_s / (ms_graph * 1e-3)
    value = rtf * world

    # ---- plain GPU form: one CB launch per (DM, beamset), no graph
    plain = stages.BeamformerPipeline(**common, grouped=False, use_graph=False,
                                      autotune=not args.no_autotune)
    plain.set_delays(delays, 1.7e9)
    ms_plain = time_steps(lambda i: plain.process_device(gulp(i), epoch0 + i * gulp_s),
                          max(3, args.steps // 2), 2)
    plain.close()
    del plain

    # ---- per-kernel timings (CUDA events on the launching stream)
    kern = kernel_breakdown(torch, stages, taftp, delays, fft_len, overlap, lag, centre,
                            bwidth, args.steps, tune)
    # ---- the plan's deviation from 65536-point (= gulp) windows, the
    # reference's FFT length
    plan_dev = cdd_window_deviation(torch, stages, taftp, centre, bwidth, fft_len, overlap, lag)

    # ---- ragged (DM x beamset) problems: grouped vs plain
    ragged = ragged_case(torch, stages, synthetic, args.steps)

    # ---- 65536-point dedispersion windows, 256 beams (precision configuration)
    long_fft = long_fft_case(torch, stages, synthetic, taftp, common, args.steps)

    # ---- end to end through the host API (pinned H2D + D2H inside the timing)
    h_ins = []
    for g_dev in (taftp, taftp_pulse):
        h_ins.append(torch.empty(taftp.shape, dtype=torch.int8, pin_memory=True))
        h_ins[-1].copy_(g_dev)
    h_in = h_ins[0]
    cb_bytes = pipe.cb_bytes_per_dm() * len(dms)
    h_out = torch.empty(cb_bytes, dtype=torch.int8, pin_memory=True)
    # at least 30 steps: the first gulp's upload and the last one's download
    # cannot overlap other work, and over 10 steps they add ~3.9 ms per step
    k_e2e = max(args.steps, 30)
    ms_e2e = time_steps(lambda i: pipe.process_host(h_ins[i % PULSE_EVERY == 10],
                                                    epoch0 + i * gulp_s, h_out),
                        k_e2e, args.warmup)
    # the transfer bound: the same bytes copied both ways at once (pinned host
    # buffers, one stream per direction), with no compute
    d_out_copy = torch.empty(cb_bytes, dtype=torch.int8, device="cuda")
    d_in_copy = torch.empty(h_in.shape, dtype=torch.int8, device="cuda")
    s_up, s_dn = torch.cuda.Stream(), torch.cuda.Stream()

    def both_ways():
        with torch.cuda.stream(s_up):
            d_in_copy.copy_(h_in, non_blocking=True)
        with torch.cuda.stream(s_dn):
            h_out.copy_(d_out_copy, non_blocking=True)

    both_ways()
    torch.cuda.synchronize()
    t_copy = time.perf_counter()
    for _ in range(5):
        both_ways()
    torch.cuda.synchronize()
    ms_copy = (time.perf_counter() - t_copy) / 5 * 1e3
    del d_out_copy, d_in_copy
    e2e = {"value": gulp_s / (ms_e2e * 1e-3) * world, "unit": "x real-time",
           "h2d_bytes_per_step": int(h_in.numel()), "d2h_bytes_per_step": int(cb_bytes),
           "ms_per_step": ms_e2e, "steps": k_e2e,
           "transfer_bound_ms": ms_copy, "frac_of_transfer_bound": ms_copy / ms_e2e}

    peaks = {}
    pk = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(pk):
        with open(pk) as f:
            peaks = json.load(f)
    int8_peak = 2.0 * peaks.get("bf16_tflops", 1590.0)      # dense int8 = 2x dense bf16
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    cb = kern["coherent_beamformer"]
    # DRAM bytes of one cb_kernel launch from the ncu capture of the 16-channel,
    # one-DM profile case (dram__bytes_read.sum 273.2 MB + write 55.2 MB),
    # scaled by the channels x DMs one grouped launch processes.
    traffic = CB_NCU_BYTES_16CH_1DM * (F / 16.0) * len(dms)
    algo_bytes = len(dms) * (F * 2 * A * 2 * T + (T // WORK["tscrunch"]) * F * B)
    roof = {"bound": "tensor", "kernel": "coherent_beamformer (tcgen05 kind::i8, grouped)",
            "achieved": cb["tops"], "peak": int8_peak, "unit": "TOPS (int8)",
            "frac": cb["tops"] / int8_peak, "traffic": traffic,
            "traffic_unit": "DRAM bytes per launch (ncu, 16-channel case scaled)",
            "algorithmic_bytes": algo_bytes,
            "peak_source": "2x measured bf16 cuBLAS burst (MEASURED_PEAKS.json)"
            if peaks else "2x fallback bf16 1.59 PFLOP/s"}
    # the other stages against their own bounds: HBM (measured copy) for the
    # byte-moving stages, the CUDA cores' FP32 rate for the FFT dedisperser
    # (148 SMs x 128 lanes x 2 flop at the timed region's median SM clock; no
    # measured FP32 peak exists)
    fp32_peak = 148 * 128 * 2 * (clocks.get("sm_mhz") or 1965.0) * 1e6 / 1e12
    rooflines = {
        "transpose_statistics": {"bound": "hbm", "achieved": kern["transpose_statistics"]["gbs"],
                                 "peak": hbm_peak, "unit": "GB/s",
                                 "frac": kern["transpose_statistics"]["gbs"] / hbm_peak},
        "incoherent_beamformer": {"bound": "hbm", "achieved": kern["incoherent_beamformer"]["gbs"],
                                  "peak": hbm_peak, "unit": "GB/s",
                                  "frac": kern["incoherent_beamformer"]["gbs"] / hbm_peak},
        "coherent_dedispersion": {"bound": "fp32 (CUDA cores); measured limit: shared-memory pipe",
                                  "achieved": kern["coherent_dedispersion"]["gflops"] / 1e3,
                                  "peak": fp32_peak, "unit": "TFLOP/s",
                                  "frac": kern["coherent_dedispersion"]["gflops"] / 1e3 / fp32_peak,
                                  "peak_source": "nominal at the median SM clock"}}
    ops_gulp = 8.0 * A * B * 2 * F * T * len(dms)
    # weights, history copy, transpose + statistics and its finalize, IB channel
    # order, CDD, IB per DM, CB
    launches = 1 + 1 + 2 + (1 if F <= 1024 else 0) + 1 + len(dms) + 1
    line = {"metric": METRIC, "value": value, "unit": "x real-time", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_graph,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int8",
            "data": "synthetic", "impl": "b200",
            "config": config_block({"inputs": INPUTS}),
            "parallelism": f"{world} independent subbands",
            "int8_tops_pipeline": ops_gulp / (ms_graph * 1e-3) / 1e12,
            "cb_int8_tops": cb["tops"],
            "plain": {"value": gulp_s / (ms_plain * 1e-3) * world, "ms_per_step": ms_plain},
            "batched_vs_plain": ms_plain / ms_graph, "ragged": ragged,
            "kernels": kern, "roofline": roof, "rooflines": rooflines, "hbm_peak_gbs": hbm_peak,
            "e2e": e2e,
            "cdd_plan": plan_dev,
            "autotune": {k: tune[k] for k in ("fft_len", "cb_tiles_per_item", "cb_voltage_stages",
                                              "cb_weight_stages")},
            "gpu_launches": launches * args.steps, "clocks": clocks}
    pipe_out_tfb = pipe.cb_device(0).clone() if world > 1 else None
    pipe.close()
    line["long_fft"] = long_fft
    if world > 1:
        try:   # every rank takes the same steps; a failure is reported, not fatal
            line["chain"] = chain_case(torch, stages, pipe_out_tfb, rank, world, args.steps)
        except Exception as e:  # noqa: BLE001
            line["chain"] = {"error": f"{type(e).__name__}: {e}"}
    if not args.no_uhf:
        free, _ = torch.cuda.mem_get_info()
        if free >= 120e9:   # the UHF chain holds ~100 GB (aggregation buffers included)
            # the burst stream (C4's S/N measurement) runs on one GPU only
            line["uhf"] = uhf_case(torch, stages, synthetic, max(8, (args.steps + 3) // 4 * 4), 8,
                                   pulses=(world == 1))
        else:
            line["uhf"] = {"skipped": f"needs ~120 GB free device memory, {free / 1e9:.0f} GB free"}
    if rank == 0 and world == 1 and not args.no_cpu:
        line["cpu_baseline"] = {k: v for k, v in cpu_baseline_median().items()
                                if k != "seconds"}
        if "bursts" in line.get("uhf", {}):
            cpu_baseline_bursts(line["uhf"]["bursts"])
    if "bursts" in line.get("uhf", {}):
        b = line["uhf"]["bursts"]
        for k in [k for k in b if k.startswith("_")]:
            del b[k]
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def kernel_breakdown(torch, stages, taftp, delays, fft_len, overlap, lag, centre, bwidth, K,
                     tune):
    """Each stage timed standalone with CUDA events over K launches."""
    A, B, F, T, ts = WORK["nant"], WORK["nbeams"], WORK["nchans"], WORK["gulp"], WORK["tscrunch"]
    dms = WORK["dms"]
    stream = torch.cuda.current_stream()
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()

    def timeit(fn, reps=K, warm=2):
        for _ in range(warm):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    out = {}
    vbytes = T * F * 2 * A * 2
    ext = torch.zeros((F, 2, A, 2, overlap + T), dtype=torch.int8, device="cuda")
    ms = timeit(lambda: stages.transpose_fpact(taftp, A, overlap + T, overlap, out=ext))
    out["transpose"] = {"ms": ms, "gbs": 2 * vbytes / (ms * 1e-3) / 1e9}
    ms = timeit(lambda: stages.statistics(ext, T, overlap))
    out["statistics"] = {"ms": ms, "gbs": vbytes / (ms * 1e-3) / 1e9}
    # the pipeline's form: both in one pass over the gulp
    ms = timeit(lambda: stages.transpose_fpact_statistics(taftp, A, overlap + T, overlap,
                                                          out=ext))
    out["transpose_statistics"] = {"ms": ms, "gbs": 2 * vbytes / (ms * 1e-3) / 1e9}
    low = centre - bwidth / 2
    cdd = stages.CoherentDedisperser(F, A, fft_len, overlap, float(np.float32(low)), bwidth, dms,
                                     lag=lag)
    outs = [torch.empty((F, 2, A, 2, T), dtype=torch.int8, device="cuda") for _ in dms]
    ms = timeit(lambda: cdd.dedisperse(ext, T, outs))
    nseg = -(-T // (fft_len - overlap))
    nstream = F * 2 * A
    # one forward transform per window, one inverse per non-zero DM (the DM-0
    # output is the window itself)
    flops = 5.0 * fft_len * np.log2(fft_len) * nseg * nstream * (1 + sum(d != 0 for d in dms))
    out["coherent_dedispersion"] = {"ms": ms, "fft_len": fft_len, "overlap": overlap,
                                    "gflops": flops / (ms * 1e-3) / 1e9,
                                    "gbs": vbytes * (1 + len(dms)) / (ms * 1e-3) / 1e9}
    bw = dev(np.ones((1, A), np.float32))
    sc = dev(np.full(F, 1e3, np.float32))
    raws = [stages.incoherent_beamform(o, T, ts, sc, sc, bw)[0] for o in outs]
    ms_ib = timeit(lambda: [stages.incoherent_beamform(o, T, ts, sc, sc, bw) for o in outs])
    out["incoherent_beamformer"] = {"ms": ms_ib, "gbs": vbytes * len(dms) / (ms_ib * 1e-3) / 1e9}
    freqs = stages.channel_frequencies(centre, bwidth, F)
    _, gemm = stages.generate_weights(dev(delays), dev(freqs), 0.0, 0.0, want_fba=False)
    mapping = dev(np.zeros(B, np.int32))
    scl = dev(np.full(F, 1e9, np.float32))
    cbo = [torch.empty((T // ts, F, B), dtype=torch.int8, device="cuda") for _ in dms]
    probs = [(o, c, r, 0, B) for o, c, r in zip(outs, cbo, raws[:len(dms)])]
    cbt = dict(tiles_per_item=tune["cb_tiles_per_item"], voltage_stages=tune["cb_voltage_stages"],
               weight_stages=tune["cb_weight_stages"])
    ms = timeit(lambda: stages.coherent_beamform_grouped(probs, gemm, scl, scl, mapping, T, ts,
                                                         **cbt))
    ops = 8.0 * A * B * 2 * F * T * len(dms)
    out["coherent_beamformer"] = {"ms": ms, "tops": ops / (ms * 1e-3) / 1e12,
                                  "ops_per_launch": ops}
    ms1 = timeit(lambda: [stages.coherent_beamform(o, gemm, scl, scl, mapping, r, T, ts, out=c)
                          for o, c, r in zip(outs, cbo, raws)])
    out["coherent_beamformer_plain"] = {"ms": ms1, "tops": ops / (ms1 * 1e-3) / 1e12}
    # shares of the pipeline's own stages (the fused transpose + statistics
    # stands in for the two separate ones)
    chain = ("transpose_statistics", "coherent_dedispersion", "incoherent_beamformer",
             "coherent_beamformer")
    total = sum(out[k]["ms"] for k in chain)
    for k in chain:
        out[k]["share"] = out[k]["ms"] / total
    return out


def cdd_window_deviation(torch, stages, taftp, centre, bwidth, fft_len, overlap, lag,
                         chans=(0, 32)):
    """How far the pipeline's overlap-save plan lies from one with 65536-point
    windows (the reference's FFT length = its gulp length,
    CoherentDedisperser.cu:47-57) and the same trims, on two channels of the
    benchmark gulp (lowest and middle), every DM: the fraction of int8
    dedispersed values that differ and the largest difference (LSB, int8
    wrap-aware).  Both plans run on this GPU; the test suite pins each of them
    to the FP64 oracle at its own geometry.  The reference chirp's phase jump
    at the bin wrap gives its response 1/n tails, so any two window
    geometries differ by about this much."""
    A, F, T = WORK["nant"], WORK["nchans"], WORK["gulp"]
    dms = WORK["dms"]
    chbw = bwidth / F
    low = float(np.float32(centre - bwidth / 2))
    ext = torch.zeros((F, 2, A, 2, overlap + T), dtype=torch.int8, device="cuda")
    stages.transpose_fpact(taftp, A, overlap + T, overlap, out=ext)
    res = {"fft_len": fft_len, "overlap": overlap, "lag": lag, "reference_fft_len": 65536,
           "channels": list(chans), "per_dm": {}}
    for dm in dms:
        fr, mx = [], 0
        for c in chans:
            x = ext[c:c + 1].contiguous()
            o = []
            for n in (fft_len, 65536):
                cdd = stages.CoherentDedisperser(1, A, n, overlap, low + c * chbw, chbw, [dm],
                                                 lag=lag)
                o.append(cdd.dedisperse(x, T)[0].to(torch.int32))
            d = (o[0] - o[1]).abs()
            d = torch.minimum(d, 256 - d)
            fr.append(float((d > 0).float().mean()))
            mx = max(mx, int(d.max()))
        res["per_dm"][str(dm)] = {"mismatch_fraction": float(np.mean(fr)), "max_lsb": mx}
    torch.cuda.synchronize()
    return res


def chain_case(torch, stages, tfb, rank, world, K):
    """The channel-partitioned chain after beamforming (N > 1): this rank's
    DM-0 coherent beams of its subband, TFB [4096][64][1024], go through one
    NCCL all-to-all (subbands.channels_to_beams: device tensors, no TMA) to
    [4096][64 x world][1024 / world], then the device incoherent dedisperser
    sums this rank's beam block over the whole band for 32 trial DMs 0-10.
    Timed with CUDA events, max over ranks."""
    from skyweaver_b200 import subbands
    import torch.distributed as dist
    F, ts = WORK["nchans"], WORK["tscrunch"]
    Ftot = F * world
    bw = Ftot * WORK["chbw"]
    freqs = stages.channel_frequencies(WORK["centre"], bw, Ftot)
    trials = np.linspace(0.0, 10.0, 32).astype(np.float32)
    tsamp_cb = ts / WORK["chbw"]
    k = 4.148806423e15
    delays = np.array([[int(k * (1 / freqs[0] ** 2 - 1 / f ** 2) * d / tsamp_cb + 0.5)
                        for f in freqs] for d in trials], np.int32)
    maxd = int(delays.max())
    n = tfb.shape[0]
    if maxd >= n:
        return {"skipped": f"max delay {maxd} exceeds the {n} samples of a gulp"}
    d_delays = torch.from_numpy(delays).cuda()
    scale = float(np.float32(np.sqrt(Ftot)))
    stream = torch.cuda.current_stream()

    def step():
        blk = subbands.channels_to_beams(tfb)
        return blk, stages.incoherent_dedisperse(blk[:n], d_delays, maxd, 1, scale)

    for _ in range(2):
        step()
    torch.cuda.synchronize()
    dist.barrier()
    e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
    xs, ids = 0.0, 0.0
    for _ in range(K):
        e0.record(stream)
        blk = subbands.channels_to_beams(tfb)
        e1.record(stream)
        stages.incoherent_dedisperse(blk[:n], d_delays, maxd, 1, scale)
        e2.record(stream)
        torch.cuda.synchronize()
        xs += e0.elapsed_time(e1)
        ids += e1.elapsed_time(e2)
    xs = max_over_ranks(xs / K, world, "cuda")
    ids = max_over_ranks(ids / K, world, "cuda")
    return {"workload": f"DM-0 beams of {world} subbands: all-to-all to beam blocks, then "
                        f"incoherent dedispersion over {Ftot} channels, 32 trial DMs 0-10",
            "exchange_ms": xs, "exchange_bytes_per_rank": int(tfb.numel()),
            "idd_ms": ids, "max_delay_samples": maxd}


RAGGED = dict(nant=64, nchans=64, gulp=32768, tscrunch=16, dms=[0.0, 50.0, 150.0, 500.0],
              ants=[64, 57, 48, 40, 32, 24, 16, 8], beams=[512, 256, 256, 128, 128, 64, 64, 32])


def long_fft_case(torch, stages, synthetic, taftp, common, K):
    """The benchmark gulp with 256 beams and 65536-point overlap-save
    windows (the precision configuration: one window per channel and gulp,
    four-step split FFT through a workspace), DMs {0, 50, 150, 500}; graph +
    grouped beamformer, input resident in HBM.  Its precision against the FP64
    oracle and the DM-150 pulse are checked by the GPU tests."""
    B = 256
    cfg = dict(common, nbeams=B, beamset_mapping=np.zeros(B, np.int32))
    pipe = stages.BeamformerPipeline(**cfg, fft_len=65536, grouped=True, use_graph=True)
    pipe.set_delays(synthetic.delay_model(synthetic.rng(256), B, cfg["nantennas"]), 1.7e9)
    fft_len, overlap, lag = pipe.cdd_plan()
    gulp_s = cfg["gulp_samples"] * tsamp()
    for i in range(3):
        pipe.process_device(taftp, 1.7e9 + i * gulp_s)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for i in range(K):
        pipe.process_device(taftp, 1.7e9 + (3 + i) * gulp_s)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / K
    pipe.close()
    return {"workload": f"{cfg['nantennas']}ant x {B}beam x {cfg['nchans']}ch x "
                        f"{cfg['gulp_samples']}-sample gulps, DMs {list(cfg['dms'])}, "
                        f"{fft_len}-point windows (overlap {overlap}, lag {lag})",
            "fft_len": fft_len, "overlap": overlap, "lag": lag, "ms_per_gulp": ms,
            "rtf": gulp_s / (ms * 1e-3), "timed_gulps": K, "warmup_gulps": 3}


def ragged_case(torch, stages, synthetic, K):
    """Ragged batched beamforming: 8 beamsets with antenna masks of
    {64..8} antennas and {512..32} beams, x 4 coherent DMs = 32 (DM, beamset)
    GEMM problems, 64 channels, 32768-sample gulps.  The grouped form is one
    persistent launch over all of them (128-beam tiles pack across beamset
    boundaries); the plain form is one launch per (DM, beamset).  Credited
    int8 ops count active antennas only: 8 * sum(A_s * B_s) * P * F * T per DM.
    Also times the whole pipeline both ways (graph + grouped vs eager + plain)."""
    R = RAGGED
    A, F, T, ts, dms = R["nant"], R["nchans"], R["gulp"], R["tscrunch"], R["dms"]
    B = sum(R["beams"])
    g = synthetic.rng(31)
    masks = synthetic.beamset_masks(g, A, R["ants"])
    mapping = np.repeat(np.arange(len(R["beams"]), dtype=np.int32), R["beams"])
    delays = synthetic.delay_model(g, B, A)
    delays[..., 0] = masks[mapping]
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    stream = torch.cuda.current_stream()

    def timeit(fn, reps=K, warm=3):
        for _ in range(warm):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    gen = torch.Generator(device="cuda").manual_seed(99)
    fps = [(torch.randn((F, 2, A, 2, T), generator=gen, device="cuda") * 8).round_()
           .clamp_(-127, 127).to(torch.int8) for _ in dms]
    freqs = stages.channel_frequencies(WORK["centre"], F * WORK["chbw"], F)
    _, gemm = stages.generate_weights(dev(delays), dev(freqs), 0.0, 0.0, want_fba=False)
    S = len(R["beams"])
    scl = dev(np.full(S * F, 1e9, np.float32))
    d_map = dev(mapping)
    raws = [torch.rand((S, T // ts, F), device="cuda") for _ in dms]
    outs = [torch.empty((T // ts, F, B), dtype=torch.int8, device="cuda") for _ in dms]
    starts = np.concatenate([[0], np.cumsum(R["beams"])[:-1]])
    grouped = [(fp, o, r, 0, B) for fp, o, r in zip(fps, outs, raws)]
    plain = [(fp, o, r, int(b0), int(nb)) for fp, o, r in zip(fps, outs, raws)
             for b0, nb in zip(starts, R["beams"])]
    ms_g = timeit(lambda: stages.coherent_beamform_grouped(grouped, gemm, scl, scl, d_map, T, ts))
    ref = [o.clone() for o in outs]
    ms_p = timeit(lambda: [stages.coherent_beamform(p[0], gemm, scl, scl, d_map, p[2], T, ts,
                                                    beam_start=p[3], beam_count=p[4], out=p[1])
                           for p in plain])
    same = all(torch.equal(a, b) for a, b in zip(ref, outs))
    credited = 8.0 * float(np.dot(R["ants"], R["beams"])) * 2 * F * T * len(dms)
    del fps, outs, raws
    # whole pipeline, both forms
    bw = F * WORK["chbw"]
    common = dict(nantennas=A, input_nantennas=A, nchans=F, nbeams=B, gulp_samples=T,
                  tscrunch=ts, centre_frequency=WORK["centre"], bandwidth=bw, dms=dms,
                  beamset_weights=masks, beamset_mapping=mapping)
    taftp = (torch.randn((T // 256, A, F, 256, 2, 2), generator=gen, device="cuda") * 8.0)
    taftp = taftp.round_().clamp_(-127, 127).to(torch.int8)
    gulp_s = T / WORK["chbw"]
    res = {}
    for name, kw in (("grouped_graph", dict(grouped=True, use_graph=True)),
                     ("plain_eager", dict(grouped=False, use_graph=False))):
        p = stages.BeamformerPipeline(**common, **kw)
        p.set_delays(delays, 1.7e9)
        res[name] = timeit(lambda: p.process_device(taftp, 1.7e9), reps=max(3, K // 2))
        p.close()
    return {"workload": "8 beamsets, antennas {64,57,48,40,32,24,16,8}, beams "
                        "{512,256,256,128,128,64,64,32}, x4 DMs = 32 problems, 64 ch, "
                        "32768-sample gulps",
            "cb_grouped_ms": ms_g, "cb_plain_ms": ms_p, "cb_grouped_vs_plain": ms_p / ms_g,
            "cb_grouped_tops_credited": credited / (ms_g * 1e-3) / 1e12,
            "cb_plain_tops_credited": credited / (ms_p * 1e-3) / 1e12,
            "cb_outputs_identical": bool(same),
            "pipeline_grouped_graph_rtf": gulp_s / (res["grouped_graph"] * 1e-3),
            "pipeline_plain_eager_rtf": gulp_s / (res["plain_eager"] * 1e-3),
            "pipeline_grouped_vs_plain": res["plain_eager"] / res["grouped_graph"]}


UHF = dict(nant=64, nchans=256, nbeams=2048, gulp=65536, tscrunch=8, coherent_dms=[0.0, 300.0],
           ntrials=128, trial_span=50.0, chbw=856e6 / 1024 * 544 / 856, top=1088e6,
           idd_dispatch=32768)


UHF_STREAM_S = 30.0   # seconds of voltages in the UHF pulse stream
UHF_NPULSES = 10


def pulse_snr(series, centre, guard=2000, half_window=16384):
    """Recovered S/N of one burst in a dedispersed series float [T][ntrials]
    (one beam): boxcars of 16..1024 samples (steps of sqrt 2) ending within
    `guard` samples of `centre`; the noise mean and per-sample standard
    deviation of each trial come from the samples of [centre - half_window,
    centre + half_window) farther than `guard` from `centre` (the standard
    deviation of a W-sample boxcar is taken as sqrt(W) times it: the
    dedispersed samples are independent).  Returns (S/N, trial index,
    boxcar width, start sample)."""
    lo = max(0, centre - half_window)
    hi = min(series.shape[0], centre + half_window)
    x = np.asarray(series[lo:hi], np.float64)
    idx = np.arange(lo, hi)
    off = np.abs(idx - centre) > guard
    mu = x[off].mean(axis=0)
    sd = x[off].std(axis=0)
    sd[sd == 0] = np.inf
    cs = np.concatenate([np.zeros((1, x.shape[1])), np.cumsum(x - mu, axis=0)])
    best = (-np.inf, 0, 0, 0)
    for k in range(13):
        w = int(round(16 * 2 ** (k / 2)))
        s = (cs[w:] - cs[:-w]) / (sd * math.sqrt(w))     # s[i] = boxcar over x[i:i+w]
        start = np.arange(s.shape[0]) + lo
        on = np.abs(start + w // 2 - centre) <= guard
        if not on.any():
            continue
        so = s[on]
        i, j = np.unravel_index(int(np.argmax(so)), so.shape)
        if so[i, j] > best[0]:
            best = (float(so[i, j]), int(j), w, int(start[on][i]))
    return best


def uhf_pulse_stream(torch, stages, synthetic, pipe, freqs, trial_dms, trial_delays, maxd, sf,
                     chbw, lag):
    """C4's stream: UHF_STREAM_S seconds of fresh sigma-8 voltages with the
    RFI tones and UHF_NPULSES bursts (DM 250-350, width 1-10 ms, target S/N
    8-30, at boresight) through the UHF pipeline and the DM-300 block's
    incoherent dedispersion (trial DMs 250-350).  Beam 0 (boresight) of the
    coherent beams and of the dedispersed output is kept on the host; the
    S/N of each burst is measured on the dedispersed output with pulse_snr.
    Returns the burst list with the recovered S/N and the beam-0 data for
    the CPU leg."""
    U = UHF
    A, F, B, T, ts = U["nant"], U["nchans"], U["nbeams"], U["gulp"], U["tscrunch"]
    tsamp_raw = 1.0 / chbw
    ngulps = int(math.ceil(UHF_STREAM_S / (T * tsamp_raw)))
    g = synthetic.rng(3030)
    pulses = synthetic.pulse_train(g, UHF_NPULSES, ngulps * T * tsamp_raw)
    bw = F * chbw
    low = float(np.float32(U["top"] - bw))
    inj = synthetic.BurstInjector(torch, pulses, freqs, tsamp_raw, low, bw, A, seed=77)
    nt = T // ts
    tfb0 = np.empty((ngulps * nt, F), np.int8)
    tdb0 = []
    idp = stages.IncoherentDedispersionPipeline(
        F, B, [(trial_delays, 1, sf)], lambda b, t: tdb0.append(t[:, :, 0].cpu().numpy()),
        dispatch=[U["idd_dispatch"]])
    gen = torch.Generator(device="cuda").manual_seed(8080)
    taftp = torch.empty((T // 256, A, F, 256, 2, 2), dtype=torch.int8, device="cuda")
    hc = 32   # heaps per noise chunk (2.1 GB of float noise)
    for gi in range(ngulps):
        for h0 in range(0, T // 256, hc):
            v = torch.empty((hc, A, F, 256, 2, 2), device="cuda").normal_(0.0, 8.0, generator=gen)
            add_rfi_tones(torch, v, UHF_RFI_CHANNELS, t0=gi * T + h0 * 256)
            taftp[h0:h0 + hc] = v.round_().clamp_(-127, 127).to(torch.int8)
            del v
        inj.inject(taftp, gi * T)
        pipe.process_device(taftp, 1.7e9 + gi * T * tsamp_raw)
        cb = pipe.cb_device(1)
        tfb0[gi * nt:(gi + 1) * nt] = cb[:, :, 0].cpu().numpy()
        idp.push(0, cb)
    torch.cuda.synchronize()
    idp.close()
    tdb = np.concatenate(tdb0) if tdb0 else np.zeros((0, trial_delays.shape[0]), np.int8)
    cb_tsamp = ts * tsamp_raw
    k = synthetic.DM_CONST
    out = []
    for p in pulses:
        # dedispersed sample of the burst: output o sums coherent-beam rows
        # o + maxd - delay, the burst reaches the top channel at raw sample
        # t_top / tsamp + lag (the dedisperser's output delay)
        top = k * p["dm"] * (1 / freqs[0] ** 2 - 1 / freqs[-1] ** 2) / cb_tsamp
        centre = int(round((p["t_top"] / tsamp_raw + lag) / ts + top - maxd
                           + 0.5 * p["width"] / cb_tsamp))
        r = {"t_top_s": round(p["t_top"], 4), "dm": round(p["dm"], 2),
             "width_ms": round(p["width"] * 1e3, 3), "target_snr": round(p["snr"], 2),
             "centre": centre}
        if centre + 16384 > tdb.shape[0]:
            r["skipped"] = "outside the dispatched output"
        else:
            snr, j, w, st = pulse_snr(tdb, centre)
            # the same trial's float sum of the int8 beams (no division, no
            # truncation): what the int8 dedispersed output can recover
            o = np.arange(centre - 16384, centre + 16384)
            rows = o[:, None] + maxd - trial_delays[j][None, :]
            flt = tfb0[rows, np.arange(F)[None, :]].astype(np.float64).sum(axis=1)
            fsnr = pulse_snr(flt[:, None], 16384)[0]
            r.update(gpu_snr=round(snr, 3), gpu_trial=j,
                     gpu_trial_dm=round(float(trial_dms[j]), 3), gpu_boxcar=w,
                     gpu_start=st, beam_float_snr=round(fsnr, 3))
        out.append(r)
    return {"stream_s": round(ngulps * T * tsamp_raw, 3), "gulps": ngulps, "beam": 0,
            "coherent_dm": 300.0, "pulses": out, "_tfb0": tfb0, "_tdb0": tdb,
            "_delays": trial_delays, "_maxd": maxd, "_sf": sf}


def uhf_case(torch, stages, synthetic, K, W, pulses=True):
    """End-to-end UHF chain: 64 antennas x 256 channels (the top of the
    544-1088 MHz band in 1024-channel mode, 0.53125 MHz channels), 2048
    coherent beams + incoherent beam, coherent DMs {0, 300}, tscrunch 8,
    then on the device the incoherent-dedispersion pipeline with 128 trial
    DMs over +-50 around each coherent DM (non-negative), dispatching every
    32768 beamformed samples (4 gulps; the dispatch must cover the 24837-sample
    overlap of the DM 250-350 block).  Times W + K gulps of synthetic voltages
    and reports the steady-state real-time factor of the K timed gulps (a
    multiple of 4, so each block dispatches K / 4 times inside them)."""
    U = UHF
    A, F, B, T, ts = U["nant"], U["nchans"], U["nbeams"], U["gulp"], U["tscrunch"]
    chbw = U["chbw"]
    bw = F * chbw
    centre = U["top"] - bw / 2
    freqs = stages.channel_frequencies(centre, bw, F)
    g = synthetic.rng(1088)
    delays = synthetic.delay_model(g, B, A)
    delays[0] = [1.0, 0.0, 0.0]   # beam 0 at boresight (the bursts' direction)
    pipe = stages.BeamformerPipeline(nantennas=A, input_nantennas=A, nchans=F, nbeams=B,
                                     gulp_samples=T, tscrunch=ts, centre_frequency=centre,
                                     bandwidth=bw, dms=U["coherent_dms"],
                                     beamset_weights=np.ones((1, A), np.float32),
                                     beamset_mapping=np.zeros(B, np.int32), autotune=True)
    pipe.set_delays(delays, 1.7e9)
    cb_tsamp = ts / chbw
    k = 4.148806423e15
    blocks, trials_of = [], []
    for dm in U["coherent_dms"]:
        trials = np.abs(np.linspace(dm - U["trial_span"], dm + U["trial_span"], U["ntrials"]))
        trials_of.append(trials.astype(np.float32))
        dl = np.array([[int(k * (1 / freqs[0] ** 2 - 1 / f ** 2) * d / cb_tsamp + 0.5)
                        for f in freqs] for d in trials.astype(np.float32)], np.int32)
        blocks.append((dl, 1, float(np.float32(math.sqrt(F)))))
    idp = stages.IncoherentDedispersionPipeline(F, B, blocks, None,
                                                dispatch=[U["idd_dispatch"]] * len(blocks))
    gen = torch.Generator(device="cuda").manual_seed(4321)
    taftp = (torch.randn((T // 256, A, F, 256, 2, 2), generator=gen, device="cuda") * 8.0)
    add_rfi_tones(torch, taftp, UHF_RFI_CHANNELS)
    taftp = taftp.round_().clamp_(-127, 127).to(torch.int8)
    stream = torch.cuda.current_stream()

    def gulp(i, mark=None):
        pipe.process_device(taftp, 1.7e9 + i * T / chbw)
        if mark is not None:  # end of the beamforming pipeline's part
            mark.record(stream)
        for d in range(len(blocks)):
            idp.push(d, pipe.cb_device(d))

    for i in range(W):
        gulp(i)
    torch.cuda.synchronize()
    ev = lambda: torch.cuda.Event(enable_timing=True)
    e0, e1 = ev(), ev()
    starts, mids = [ev() for _ in range(K)], [ev() for _ in range(K)]
    e0.record(stream)
    for i in range(K):
        starts[i].record(stream)
        gulp(W + i, mids[i])
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / K
    # per gulp: the beamforming pipeline, then the incoherent-dedispersion
    # pipeline (pushes into its aggregation buffers and, every dispatch
    # samples, the dedispersion and its overlap copy)
    ends = starts[1:] + [e1]
    ms_bf = sum(a.elapsed_time(b) for a, b in zip(starts, mids)) / K
    ms_idd = sum(b.elapsed_time(c) for b, c in zip(mids, ends)) / K
    geo = [idp.geometry(b) for b in range(len(blocks))]
    idp.close()
    del taftp
    torch.cuda.empty_cache()
    gulp_s = T / chbw
    adds = sum(U["ntrials"] * (T // ts) * B * F for _ in blocks)
    res = {"workload": "UHF 544-1088 MHz (top 256 of 1024 channels), 64 ant x 2048 beams, "
                       "coherent DMs {0,300}, tscrunch 8, 128 incoherent trials per coherent "
                       "DM over +-50, device aggregation (dispatch 32768); sigma-8 voltages "
                       "with RFI tones at 20 sigma in channels 40, 130 and 200",
           "ms_per_gulp": ms, "rtf": gulp_s / (ms * 1e-3),
           "idd_adds_per_gulp": adds, "idd_overlap_samples": [g[1] for g in geo],
           "cdd_plan": list(pipe.cdd_plan()), "timed_gulps": K, "warmup_gulps": W,
           "ms_per_gulp_split": {"beamforming_pipeline": ms_bf,
                                 "incoherent_dedispersion_pipeline": ms_idd}}
    if pulses:
        _, lag = pipe.cdd_plan()[1:]
        dl, _, sf = blocks[1]
        res["bursts"] = uhf_pulse_stream(torch, stages, synthetic, pipe, freqs, trials_of[1],
                                         dl, int(dl.max()), sf, chbw, lag)
    pipe.close()
    torch.cuda.empty_cache()
    return res


def profile_case(which, nchans=16, reps=3):
    """Small single-kernel case for ncu captures: `nchans` channels of the
    benchmark workload (268 MB of voltages for 16 channels, above L2), one
    warm-up launch and `reps` profiled launches of one kernel.  `cb8`: the
    `cb` case at tscrunch 8.  `idd`: the UHF incoherent-dedispersion trials
    (128 DMs over 0-100, 256 channels) for 1024 of the 2048 beams on 4096
    output samples, a 2.9 GB beam buffer.  `bw`: the
    transpose, statistics, fused transpose + statistics and incoherent-beam
    kernels on the same channels.  `uhf`: the UHF leg's chain (C4) without
    its burst stream, 4 warm-up + 4 timed gulps, for the launch list (one-pass
    `gpu__time_duration.sum` only: it holds tens of GB)."""
    import torch

    from skyweaver_b200 import stages, synthetic
    if which == "uhf":
        r = uhf_case(torch, stages, synthetic, 4, 4, pulses=False)
        print(json.dumps({"profile case uhf": r}))
        return
    if which == "idd":
        U = UHF
        F, B, D = U["nchans"], U["nbeams"] // 2, 4096   # 2.9 GB of beams
        freqs = U["top"] - F * U["chbw"] + U["chbw"] * (np.arange(F) + 0.5)
        cb_tsamp = U["tscrunch"] / U["chbw"]
        trials = np.linspace(0.0, 2 * U["trial_span"], U["ntrials"]).astype(np.float32)
        k = 4.148806423e15
        dl = np.array([[int(k * (1 / freqs[0] ** 2 - 1 / f ** 2) * d / cb_tsamp + 0.5)
                        for f in freqs] for d in trials], np.int32)
        maxd = int(dl.max())
        tfb = torch.randint(-128, 128, (D + maxd, F, B), dtype=torch.int8, device="cuda")
        delays = torch.from_numpy(dl).cuda()
        sf = float(np.float32(math.sqrt(F)))
        fn = lambda: stages.incoherent_dedisperse(tfb, delays, maxd, 1, sf)
        for _ in range(1 + reps):
            fn()
        torch.cuda.synchronize()
        print(f"profile case idd: {U['ntrials']} DMs, {D} samples, {1 + reps} launches ok")
        return
    A, B, T, ts = WORK["nant"], WORK["nbeams"], WORK["gulp"], WORK["tscrunch"]
    F = nchans
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    gen = torch.Generator(device="cuda").manual_seed(7)
    if which == "bw":
        # the HBM-bound stages of one gulp: TAFTP -> FPACT transpose, statistics,
        # and the incoherent beam of one DM
        # complex-Gaussian sigma = 8 voltages, as in the workload (full-range
        # uniform bytes would push the incoherent beam's integer sums past 2^24
        # and onto its reference-order float path)
        taftp = (torch.randn((T // 256, A, F, 256, 2, 2), generator=gen, device="cuda") * 8)
        taftp = taftp.round_().clamp_(-127, 127).to(torch.int8)
        fpact = stages.transpose_fpact(taftp, A)
        bw = dev(np.ones((1, A), np.float32))
        scl = dev(np.full(F, 1e4, np.float32))
        for _ in range(1 + reps):
            stages.transpose_fpact(taftp, A, out=fpact)
            stages.statistics(fpact, T)
            stages.transpose_fpact_statistics(taftp, A, out=fpact)  # the pipeline's form
            stages.incoherent_beamform(fpact, T, ts, scl, scl, bw)
        torch.cuda.synchronize()
        print(f"profile case bw: {nchans} channels, {1 + reps} launches of each stage ok")
        return
    fp = (torch.randn((F, 2, A, 2, T), generator=gen, device="cuda") * 8).round_().clamp_(-127, 127)
    fp = fp.to(torch.int8)
    if which in ("cb", "cb8"):
        ts = 8 if which == "cb8" else ts
        g = synthetic.rng(3)
        freqs = stages.channel_frequencies(WORK["centre"], F * WORK["chbw"], F)
        _, gemm = stages.generate_weights(dev(synthetic.delay_model(g, B, A)), dev(freqs),
                                          0.0, 0.0, want_fba=False)
        mapping = dev(np.zeros(B, np.int32))
        scl = dev(np.full(F, 1e9, np.float32))
        ib = torch.rand((1, T // ts, F), device="cuda")
        out = torch.empty((T // ts, F, B), dtype=torch.int8, device="cuda")
        fn = lambda: stages.coherent_beamform_grouped([(fp, out, ib, 0, B)], gemm, scl, scl,
                                                      mapping, T, ts)
    else:
        n, ov, lag = stages.cdd_plan(WORK["centre"], 64 * WORK["chbw"], 64, WORK["dms"])
        ext = torch.zeros((F, 2, A, 2, ov + T), dtype=torch.int8, device="cuda")
        ext[..., ov:] = fp
        low = WORK["centre"] - 32 * WORK["chbw"]
        cdd = stages.CoherentDedisperser(F, A, n, ov, low, F * WORK["chbw"], WORK["dms"],
                                         lag=lag)
        outs = [torch.empty((F, 2, A, 2, T), dtype=torch.int8, device="cuda") for _ in WORK["dms"]]
        fn = lambda: cdd.dedisperse(ext, T, outs)
    for _ in range(1 + reps):
        fn()
    torch.cuda.synchronize()
    print(f"profile case {which}: {nchans} channels, {1 + reps} launches ok")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--profile", choices=["cb", "cb8", "cdd", "idd", "bw", "uhf"], default=None,
                    help="run a small single-kernel case for ncu and exit")
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-uhf", action="store_true",
                    help="skip the UHF beamforming + incoherent dedispersion measurement")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-autotune", action="store_true",
                    help="run the cost model's plan and the kernel defaults instead of "
                         "the autotuned ones (for profiling captures)")
    args = ap.parse_args()
    if args.profile:
        profile_case(args.profile)
    elif args.impl == "reference":
        run_reference(args)
    else:
        main_b200(args)


if __name__ == "__main__":
    main()
