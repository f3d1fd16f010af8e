"""CPU ORACLE for the skyweaver beamforming hot path -- test infrastructure only.

numpy/ctypes face of ``swb_oracle.c`` (a plain-C restatement of the skyweaver
reference's CPU test implementations; see that file's header for the reference
file:line each function follows).  Only ``tests/``, ``__graft_entry__.smoke()``
and ``bench.py``'s CPU-baseline leg import this module, and only as a checker:
the product library never routes through it.

Array conventions (all C-contiguous numpy arrays):
  voltages  int8 [..., 2]  (re, im) pairs, i.e. char2
  TAFTP     [heaps][ant][chan][256][pol][2]
  FTPA      [chan][sample][pol][ant][2]
  weights   [chan][beam][ant][2]
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libswb_oracle.so")
_lib = None

STOKES = {"I": 0, "Q": 1, "U": 2, "V": 3}


def build() -> str:
    """Compile the oracle shared library (gcc) if it is missing or stale."""
    src = os.path.join(_HERE, "swb_oracle.c")
    if (not os.path.exists(_LIB_PATH)
            or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src)):
        subprocess.check_call(["make", "-s", "-C", _HERE, "-B", "libswb_oracle.so"])
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        _lib = ctypes.CDLL(_LIB_PATH)
        _lib.swo_dm_delay.restype = ctypes.c_double
        _lib.swo_dm_delay.argtypes = [ctypes.c_double] * 3
        _lib.swo_dm_sample_delay.restype = ctypes.c_int
        _lib.swo_dm_sample_delay.argtypes = [ctypes.c_double] * 4
        _lib.swo_idd_delays.restype = ctypes.c_int
        _lib.swo_idd.restype = ctypes.c_int
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


def _c(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)


# ---------------------------------------------------------------- transpose
def transpose(taftp: np.ndarray, out_nant: int) -> np.ndarray:
    """TAFTP -> FTPA with zero-padded antennas (TransposerTester.cu:30-72)."""
    taftp = _c(taftp, np.int8)
    nheaps, in_nant, nchans, nsph, npol, _ = taftp.shape
    out = np.empty((nchans, nheaps * nsph, npol, out_nant, 2), np.int8)
    lib().swo_transpose(_p(taftp), _p(out), in_nant, out_nant, nchans, nheaps,
                        nsph, npol)
    return out


# --------------------------------------------------------------- statistics
def statistics(ftpa: np.ndarray) -> np.ndarray:
    """RunningStats per (F,P,A) -> float32 [F][P][A][4] = mean,std,skew,kurt."""
    ftpa = _c(ftpa, np.int8)
    nchans, nsamp, npol, nant, _ = ftpa.shape
    out = np.empty((nchans, npol, nant, 4), np.float32)
    lib().swo_statistics(_p(ftpa), _p(out), nchans, nsamp, npol, nant)
    return out


def scalings(stats, beamset_weights, nbeamsets, cb_tscrunch, ib_tscrunch,
             output_level):
    """Per-(beamset, channel) CB/IB offsets and scalings
    (StatisticsCalculator.cu:132-239, per-beamset index)."""
    stats = _c(stats, np.float32)
    bw = _c(beamset_weights, np.float32)
    nchans, npol, nant, _ = stats.shape
    outs = [np.empty(nbeamsets * nchans, np.float32) for _ in range(4)]
    lib().swo_scalings(_p(stats), _p(bw), nbeamsets, nchans, npol, nant,
                       cb_tscrunch, ib_tscrunch, ctypes.c_float(output_level),
                       *[_p(o) for o in outs])
    return tuple(outs)  # cb_offsets, cb_scaling, ib_offsets, ib_scaling


# ---------------------------------------------------------------- IB and CB
def incoherent_beam(ftpa, tscrunch, scale, offset, beamset_weights, nbeamsets,
                    stokes="I"):
    """IncoherentBeamformerTester.cu:41-103 -> (raw float BTF, int8 BTF).

    stokes="IQUV" follows FullStokesBeamformerTraits (beamformer_utils.cuh:
    198-278): every member (integrate, ib_subtract, rescale, clamp) applies
    the single-Stokes trait of its component, so component c of the float4 /
    char4 result is the single-Stokes result for c; the arrays gain a last
    axis of 4."""
    if stokes == "IQUV":
        parts = [incoherent_beam(ftpa, tscrunch, scale, offset, beamset_weights, nbeamsets, c)
                 for c in "IQUV"]
        return (np.stack([p[0] for p in parts], -1), np.stack([p[1] for p in parts], -1))
    ftpa = _c(ftpa, np.int8)
    nchans, nsamp, npol, nant, _ = ftpa.shape
    raw = np.empty((nbeamsets, nsamp // tscrunch, nchans), np.float32)
    out = np.empty((nbeamsets, nsamp // tscrunch, nchans), np.int8)
    lib().swo_ib(_p(ftpa), _p(raw), _p(out), nchans, tscrunch, nsamp, nant,
                 _p(_c(scale, np.float32)), _p(_c(offset, np.float32)),
                 _p(_c(beamset_weights, np.float32)), nbeamsets, STOKES[stokes])
    return raw, out


def coherent_beam(ftpa, weights, tscrunch, scales, offsets, beamset_weights,
                  mapping, stokes="I", ib_subtract=True, want_voltages=False):
    """CoherentBeamformerTester.cu:43-152 -> int8 TFB [T/ts][F][B]
    (and optionally the exact int32 beam voltages [F][T][P][B][2]).
    stokes="IQUV": char4 TFB [T/ts][F][B][4], component c equal to the
    single-Stokes result for c (FullStokesBeamformerTraits)."""
    if stokes == "IQUV":
        parts = [coherent_beam(ftpa, weights, tscrunch, scales, offsets, beamset_weights,
                               mapping, c, ib_subtract, want_voltages) for c in "IQUV"]
        if want_voltages:
            return np.stack([p[0] for p in parts], -1), parts[0][1]
        return np.stack(parts, -1)
    ftpa = _c(ftpa, np.int8)
    weights = _c(weights, np.int8)
    nchans, nsamp, npol, nant, _ = ftpa.shape
    nbeams = weights.shape[1]
    out = np.empty((nsamp // tscrunch, nchans, nbeams), np.int8)
    volts = (np.empty((nchans, nsamp, npol, nbeams, 2), np.int32)
             if want_voltages else None)
    lib().swo_cb(_p(ftpa), _p(weights), _p(out), nchans, tscrunch, nsamp,
                 nbeams, nant, _p(_c(scales, np.float32)),
                 _p(_c(offsets, np.float32)), _p(_c(beamset_weights, np.float32)),
                 _p(_c(mapping, np.int32)), STOKES[stokes], int(ib_subtract),
                 _p(volts))
    return (out, volts) if want_voltages else out


# ------------------------------------------------------------------ weights
def weights(delays, freqs, current_epoch, delay_epoch):
    """WeightsManagerTester.cu:33-71: float3 [B][A] -> char2 [F][B][A]."""
    delays = _c(delays, np.float32)
    freqs = _c(freqs, np.float64)
    nbeams, nant, _ = delays.shape
    out = np.empty((len(freqs), nbeams, nant, 2), np.int8)
    lib().swo_weights(_p(delays), _p(out), _p(freqs), nant, nbeams, len(freqs),
                      ctypes.c_double(current_epoch), ctypes.c_double(delay_epoch),
                      ctypes.c_double(0.0), 1)
    return out


# -------------------------------------------------------- coherent dedisp.
def dm_delay(f_ref, f, dm):
    return lib().swo_dm_delay(f_ref, f, dm)


def dm_sample_delay(dm, f_ref, tsamp, f):
    return lib().swo_dm_sample_delay(dm, f_ref, tsamp, f)


def chirp(nchans, fft_len, low_freq, bw, dm):
    """FP64 DMResponse table [nchans][fft_len] complex128
    (CoherentDedisperser.cu:293-336)."""
    out = np.empty((nchans, fft_len), np.complex128)
    lib().swo_chirp(_p(out), nchans, fft_len, ctypes.c_double(low_freq),
                    ctypes.c_double(bw), ctypes.c_float(dm))
    return out


def cdd_segment(stream, chirp_row, overlap, want_f64=False, lag=None):
    """One FFT -> chirp -> IFFT -> trim -> /N -> round -> int8-wrap segment.
    stream: int8 [fft_len][2]; chirp_row: complex128 [fft_len].  `lag`
    samples are trimmed at the end of the window and overlap - lag at its
    start; None is the reference's overlap / 2 at each end
    (CoherentDedisperser.cu:196-223)."""
    stream = _c(stream, np.int8)
    n = stream.shape[0]
    lag = overlap // 2 if lag is None else int(lag)
    if not 0 <= lag <= overlap:
        raise ValueError("lag must lie in [0, overlap]")
    ch = _c(chirp_row, np.complex128)
    out = np.empty((n - overlap, 2), np.int8)
    f64 = np.empty(n - overlap, np.complex128) if want_f64 else None
    lib().swo_cdd_segment(_p(stream), _p(ch), n, overlap, lag, _p(out), _p(f64))
    return (out, f64) if want_f64 else out


def cdd_stream(stream, nsamples, chirp_row, overlap, want_f64=False, lag=None):
    """Overlap-save over a gulp for one stream: stream int8 [overlap+T][2]
    (history then gulp) -> int8 [T][2] (and FP64 values [T]); output m is
    the dedispersed voltage at gulp position m - lag."""
    stream = _c(stream, np.int8)
    lag = overlap // 2 if lag is None else int(lag)
    if not 0 <= lag <= overlap:
        raise ValueError("lag must lie in [0, overlap]")
    ch = _c(chirp_row, np.complex128)
    out = np.empty((nsamples, 2), np.int8)
    f64 = np.empty(nsamples, np.complex128) if want_f64 else None
    lib().swo_cdd_stream(_p(stream), nsamples, _p(ch), len(ch), overlap, lag,
                         _p(out), _p(f64))
    return (out, f64) if want_f64 else out


def cdd_ftpa(ftpa_ext, nsamples, chirps, overlap, want_f64=False, lag=None):
    """Coherent dedispersion of a whole FTPA gulp for one DM.
    ftpa_ext: int8 [F][overlap+T][P][A][2] (history + gulp);
    chirps: complex128 [F][fft_len].  Returns int8 FTPA [F][T][P][A][2]."""
    F, _, P, A, _ = ftpa_ext.shape
    out = np.empty((F, nsamples, P, A, 2), np.int8)
    f64 = np.empty((F, nsamples, P, A), np.complex128) if want_f64 else None
    for f in range(F):
        for p in range(P):
            for a in range(A):
                r = cdd_stream(ftpa_ext[f, :, p, a], nsamples, chirps[f], overlap,
                               want_f64, lag)
                if want_f64:
                    out[f, :, p, a], f64[f, :, p, a] = r
                else:
                    out[f, :, p, a] = r
    return (out, f64) if want_f64 else out


def cdd_plan(centre_frequency, bandwidth, nchans, dms, fft_len=0, lag=128):
    """The pipeline's overlap-save plan restated: (fft_len, overlap, lag).

    The reference's chirp (CoherentDedisperser.cu:313-335) has a one-sided
    impulse response: nearly all of it lies at lags 0 .. the intra-channel
    smear of the lowest channel at the largest DM.  The window therefore
    trims that smear (rounded up to 16) at its start and a margin `lag`
    (rounded up to 16) at its end, which holds the response's short
    anti-causal part; the output is delayed by `lag` samples.  With every DM
    0 the response is a unit impulse and nothing is trimmed."""
    chbw = bandwidth / nchans
    f_low = float(np.float32(centre_frequency - bandwidth / 2.0))
    smear = 4.148806423e15 * (1.0 / f_low ** 2 - 1.0 / (f_low + chbw) ** 2) * max(dms)
    head = (int(np.ceil(smear * chbw)) + 15) // 16 * 16
    lag = (int(lag) + 15) // 16 * 16 if head else 0   # every DM 0: a unit impulse
    overlap = head + lag
    if not fft_len:
        best = None
        for n in (1024, 2048, 4096, 8192):
            if n <= overlap:
                continue
            cost = np.log2(n) / (1.0 - overlap / n)
            if best is None or cost < best[0] - 1e-9:
                best = (cost, n)
        if best is None:
            best = (0.0, next(n for n in (16384, 32768, 65536) if n > overlap))
        fft_len = best[1]
    return fft_len, overlap, lag


# -------------------------------------------------------- incoherent dedisp.
def idd_delays(freqs, dms, tsamp):
    freqs = _c(freqs, np.float64)
    dms = _c(dms, np.float32)
    delays = np.empty((len(dms), len(freqs)), np.int32)
    maxd = lib().swo_idd_delays(_p(freqs), len(freqs), _p(dms), len(dms),
                                ctypes.c_double(tsamp), _p(delays))
    return delays, maxd


def idd(tfb, delays, max_delay, tscrunch, scale_factor):
    """IncoherentDedisperser.cu:66-125: int8 TFB -> int8 TDB."""
    tfb = _c(tfb, np.int8)
    nsamp, nchans, nbeams = tfb.shape
    ndms = delays.shape[0]
    if nsamp <= max_delay or (nsamp - max_delay) % tscrunch:
        raise RuntimeError("invalid number of samples for incoherent dedispersion")
    out = np.empty(((nsamp - max_delay) // tscrunch, ndms, nbeams), np.int8)
    rc = lib().swo_idd(_p(tfb), _p(out), nsamp, nchans, nbeams,
                       _p(_c(delays, np.int32)), ndms, max_delay, tscrunch,
                       ctypes.c_float(scale_factor))
    if rc != 0:
        raise RuntimeError("swo_idd failed")
    return out
