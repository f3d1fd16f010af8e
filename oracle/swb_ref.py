"""ctypes access to oracle/_ref/libswref.so: the reference's own stage
implementations built from its sources (oracle/Makefile, target `ref`; see
ref_driver.cu).  Test infrastructure only: the GPU parity tests use it to
pin the oracle restatement and the B200 kernels to the reference itself.
Shapes are the build's compile-time constants (shape())."""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_ref", "libswref.so")
_lib = None


def available() -> bool:
    return os.path.exists(LIB)


def lib():
    global _lib
    if _lib is None:
        _lib = ctypes.CDLL(LIB)
        _lib.swref_error.restype = ctypes.c_char_p
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def _check(rc):
    if rc != 0:
        raise RuntimeError(lib().swref_error().decode())


def shape():
    v = [ctypes.c_int() for _ in range(5)]
    lib().swref_shape(*[ctypes.byref(x) for x in v])
    return dict(zip(("nant", "nchans", "nbeams", "cb_ts", "ib_ts"), (x.value for x in v)))


def transpose(taftp, input_nant):
    s = shape()
    H = taftp.shape[0]
    out = np.empty((s["nchans"], H * 256, 2, s["nant"], 2), np.int8)
    _check(lib().swref_transpose(_p(np.ascontiguousarray(taftp)), H, input_nant, _p(out)))
    return out


def statistics(ftpa):
    s = shape()
    T = ftpa.shape[1]
    out = np.empty((s["nchans"], 2, s["nant"], 4), np.float32)
    _check(lib().swref_statistics(_p(np.ascontiguousarray(ftpa)), T, _p(out)))
    return out


def beamform(ftpa, weights, cb_scale, cb_offset, ib_scale, ib_offset, beamset_weights, mapping):
    s = shape()
    F, T, B = s["nchans"], ftpa.shape[1], s["nbeams"]
    S = beamset_weights.shape[0]
    ts = s["cb_ts"]
    raw = np.empty((S, T // ts, F), np.float32)
    ib = np.empty((S, T // ts, F), np.int8)
    cb = np.empty((T // ts, F, B), np.int8)
    f32 = lambda a: np.ascontiguousarray(a, np.float32)
    _check(lib().swref_beamform(_p(np.ascontiguousarray(ftpa)), T, _p(np.ascontiguousarray(weights)),
                                _p(f32(cb_scale)), _p(f32(cb_offset)), _p(f32(ib_scale)),
                                _p(f32(ib_offset)), _p(f32(beamset_weights)),
                                _p(np.ascontiguousarray(mapping, np.int32)), S, _p(raw), _p(ib),
                                _p(cb)))
    return raw, ib, cb


def weights(delays, current_epoch, delay_epoch, centre, bw):
    s = shape()
    out = np.empty((s["nchans"], s["nbeams"], s["nant"], 2), np.int8)
    lib().swref_weights.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_double,
                                    ctypes.c_double, ctypes.c_double, ctypes.c_void_p]
    _check(lib().swref_weights(_p(np.ascontiguousarray(delays, np.float32)), current_epoch,
                               delay_epoch, centre, bw, _p(out)))
    return out


def idd(tfb, dms, tscrunch, centre, bw):
    s = shape()
    T = tfb.shape[0]
    dms = np.ascontiguousarray(dms, np.float32)
    delays = np.empty((len(dms), s["nchans"]), np.int32)
    maxd = ctypes.c_int()
    lib().swref_idd.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int,
                                ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_void_p,
                                ctypes.c_void_p, ctypes.c_void_p]
    # TDB rows: (T - max_delay) / tscrunch; allocate for the largest case
    out = np.empty((T // tscrunch + 1) * len(dms) * s["nbeams"], np.int8)
    _check(lib().swref_idd(_p(np.ascontiguousarray(tfb)), T, _p(dms), len(dms), tscrunch, centre,
                           bw, _p(out), _p(delays), ctypes.byref(maxd)))
    n = (T - maxd.value) // tscrunch
    return out[:n * len(dms) * s["nbeams"]].reshape(n, len(dms), s["nbeams"]), delays, maxd.value


def cdd(tpa, overlap, dms, dm_idx, chan, low, bw):
    """One overlap-save window of channel `chan` through the reference's
    CoherentDedisperser (cuFFT): int8 TPA [fft_length][2][A][2] in, the
    trimmed [fft_length - overlap][2][A][2] int8 for DM `dm_idx` out.  The
    band [low, low + bw) spans the build's channels."""
    tpa = np.ascontiguousarray(tpa, np.int8)
    n = tpa.shape[0]
    dms = np.ascontiguousarray(dms, np.float32)
    out = np.empty((n - overlap,) + tpa.shape[1:], np.int8)
    lib().swref_cdd.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_int,
                                ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                ctypes.c_void_p, ctypes.c_void_p]
    _check(lib().swref_cdd(n, overlap, _p(dms), len(dms), low, bw, chan, dm_idx, _p(tpa),
                           _p(out)))
    return out


LIB_C1 = os.path.join(HERE, "_ref", "c1", "libswref_c1.so")


def time_beamform_c1(nsamples=65536, reps=3):
    """Device ms of the reference's own IncoherentBeamformer and
    CoherentBeamformer (Stokes I) at 64 antennas x 64 channels x 1024 beams,
    tscrunch 16, one call each (oracle/_ref/c1)."""
    lc = ctypes.CDLL(LIB_C1)
    lc.swref_error.restype = ctypes.c_char_p
    ib, cb = ctypes.c_float(), ctypes.c_float()
    if lc.swref_time_beamform(nsamples, reps, ctypes.byref(ib), ctypes.byref(cb)) != 0:
        raise RuntimeError(lc.swref_error().decode())
    return ib.value, cb.value


def time_cdd_c1(dms, fft_length=65536, overlap=1472, centre=1284e6, bw=64 * 856e6 / 1024,
                reps=2):
    """Device ms per gulp of the reference's own coherent dedispersion: one
    CoherentDedisperser::dedisperse call per (channel, DM) at 64 channels x
    2 pols x 64 antennas (oracle/_ref/c1)."""
    lc = ctypes.CDLL(LIB_C1)
    lc.swref_error.restype = ctypes.c_char_p
    lc.swref_time_cdd.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_int,
                                  ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_void_p]
    d = np.ascontiguousarray(dms, np.float32)
    ms = ctypes.c_float()
    if lc.swref_time_cdd(fft_length, overlap, _p(d), len(d), centre, bw, reps,
                         ctypes.byref(ms)) != 0:
        raise RuntimeError(lc.swref_error().decode())
    return ms.value
