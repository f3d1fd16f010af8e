"""Python face of the skyweaver_b200 C ABI, shaped like the reference's stage
classes (Transposer, StatisticsCalculator, WeightsManager, CoherentDedisperser,
IncoherentBeamformer, CoherentBeamformer, IncoherentDedisperser,
BeamformerPipeline).  Device memory is torch CUDA tensors; every call goes
through libskyweaver_b200.so (there is no other implementation).
"""
from __future__ import annotations

import ctypes
import math

import numpy as np
import torch

from . import _lib
from ._lib import STOKES, CbProblem, CbShape, call, lib

DM_CONST = 4.148806423e15


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def _stream(stream=None):
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


def device_error() -> int:
    """The device error word that kernels with bounded waits set when a wait
    gives up (0 = clean); it stays set until reset_device_error()."""
    code = ctypes.c_int()
    call("sw_read_device_error", ctypes.byref(code))
    return code.value


def reset_device_error() -> None:
    call("sw_reset_device_error")


def check_device_error() -> None:
    """Raise SkyweaverError(SW_ERR_TIMEOUT) if a bounded device-side wait gave
    up since the last reset, clearing the word."""
    code = device_error()
    if code:
        reset_device_error()
        raise _lib.SkyweaverError(_lib.SW_ERR_TIMEOUT,
                                  f"a bounded device-side wait gave up (device error {code})")


def cb_timeout_selftest(timeout_us: int = 20000, stream=None) -> int:
    """Run the coherent beamformer's bounded-wait self-test; returns its
    status (SW_ERR_TIMEOUT when the kernel timed out and returned)."""
    return lib().sw_cb_timeout_selftest(int(timeout_us), _stream(stream))


def channel_frequencies(centre, bandwidth, nchans):
    chbw = bandwidth / nchans
    return centre - bandwidth / 2.0 + chbw / 2.0 + chbw * np.arange(nchans)


# ------------------------------------------------------------------ layouts
def transpose_ftpa(taftp: torch.Tensor, out_nant: int, stream=None) -> torch.Tensor:
    """Transposer::transpose: TAFTP [H][A_in][F][256][2][2] -> FTPA."""
    H, A_in, F = taftp.shape[:3]
    out = torch.empty((F, H * 256, 2, out_nant, 2), dtype=torch.int8, device=taftp.device)
    call("sw_transpose_ftpa", _ptr(taftp), _ptr(out), H, A_in, out_nant, F, _stream(stream))
    return out


def transpose_fpact(taftp, out_nant, row_stride=None, offset=0, out=None, stream=None):
    H, A_in, F = taftp.shape[:3]
    T = H * 256
    row_stride = row_stride or (offset + T)
    if out is None:
        out = torch.zeros((F, 2, out_nant, 2, row_stride), dtype=torch.int8, device=taftp.device)
    call("sw_transpose_fpact", _ptr(taftp), _ptr(out), H, A_in, out_nant, F, row_stride,
         offset, _stream(stream))
    return out


def ftpa_to_fpact(ftpa, row_stride=None, offset=0, stream=None):
    F, T, P, A, _ = ftpa.shape
    row_stride = row_stride or (offset + T)
    out = torch.zeros((F, P, A, 2, row_stride), dtype=torch.int8, device=ftpa.device)
    call("sw_ftpa_to_fpact", _ptr(ftpa), _ptr(out), F, T, A, row_stride, offset,
         _stream(stream))
    return out


def fpact_to_ftpa(fpact, nsamples, offset=0, stream=None):
    F, P, A, _, stride = fpact.shape
    out = torch.empty((F, nsamples, P, A, 2), dtype=torch.int8, device=fpact.device)
    call("sw_fpact_to_ftpa", _ptr(fpact), _ptr(out), F, nsamples, A, stride, offset,
         _stream(stream))
    return out


# --------------------------------------------------------------- statistics
def statistics(fpact, nsamples, offset=0, stream=None):
    """StatisticsCalculator::calculate_statistics -> float [F][P][A][4]."""
    F, P, A, _, stride = fpact.shape
    scratch = torch.empty(lib().sw_statistics_scratch_bytes(F, P, A), dtype=torch.uint8,
                          device=fpact.device)
    stats = torch.empty((F, P, A, 4), dtype=torch.float32, device=fpact.device)
    call("sw_statistics", _ptr(fpact), stride, offset, F, P, A, nsamples, _ptr(scratch),
         _ptr(stats), _stream(stream))
    return stats


def transpose_fpact_statistics(taftp, out_nant, row_stride=None, offset=0, out=None,
                               stream=None):
    """The TAFTP -> FPACT transpose and the statistics of the gulp in one pass
    over the voltages: (fpact, float [F][2][out_nant][4]), equal to
    transpose_fpact followed by statistics."""
    H, A_in, F = taftp.shape[:3]
    T = H * 256
    row_stride = row_stride or (offset + T)
    if out is None:
        out = torch.zeros((F, 2, out_nant, 2, row_stride), dtype=torch.int8, device=taftp.device)
    scratch = torch.empty(lib().sw_statistics_scratch_bytes(F, 2, out_nant), dtype=torch.uint8,
                          device=taftp.device)
    stats = torch.empty((F, 2, out_nant, 4), dtype=torch.float32, device=taftp.device)
    call("sw_transpose_fpact_statistics", _ptr(taftp), _ptr(out), H, A_in, out_nant, F,
         row_stride, offset, _ptr(scratch), _ptr(stats), _stream(stream))
    return out, stats


def update_scalings(stats, beamset_weights, cb_tscrunch, ib_tscrunch, output_level,
                    stream=None):
    """StatisticsCalculator::update_scalings -> (cb_off, cb_scl, ib_off, ib_scl)."""
    F, P, A, _ = stats.shape
    S = beamset_weights.shape[0]
    outs = [torch.empty(S * F, dtype=torch.float32, device=stats.device) for _ in range(4)]
    call("sw_update_scalings", _ptr(stats), _ptr(beamset_weights), S, F, P, A, cb_tscrunch,
         ib_tscrunch, ctypes.c_float(output_level), *[_ptr(o) for o in outs], _stream(stream))
    return tuple(outs)


# ------------------------------------------------------------------ weights
def generate_weights(delays, freqs, current_epoch, delay_epoch, want_fba=True,
                     want_gemm=True, stream=None):
    """WeightsManager::weights: float3 [B][A] -> (char2 [F][B][A], GEMM layout)."""
    B, A, _ = delays.shape
    F = freqs.shape[0]
    fba = torch.empty((F, B, A, 2), dtype=torch.int8, device=delays.device) if want_fba else None
    gemm = (torch.empty((F, 2, B, A, 2), dtype=torch.int8, device=delays.device)
            if want_gemm else None)
    call("sw_generate_weights", _ptr(delays), _ptr(freqs), A, B, F,
         ctypes.c_double(current_epoch), ctypes.c_double(delay_epoch), _ptr(fba), _ptr(gemm),
         _stream(stream))
    return fba, gemm


def pack_weights(fba, stream=None):
    F, B, A, _ = fba.shape
    gemm = torch.empty((F, 2, B, A, 2), dtype=torch.int8, device=fba.device)
    call("sw_pack_weights", _ptr(fba), _ptr(gemm), F, B, A, _stream(stream))
    return gemm


# --------------------------------------------------------------------- beams
def incoherent_beamform(fpact, nsamples, tscrunch, scale, offset, beamset_weights,
                        offset_samples=0, stokes="I", stream=None):
    F, P, A, _, stride = fpact.shape
    S = beamset_weights.shape[0]
    shape = (S, nsamples // tscrunch, F) + ((4,) if stokes == "IQUV" else ())
    raw = torch.empty(shape, dtype=torch.float32, device=fpact.device)
    out = torch.empty(shape, dtype=torch.int8, device=fpact.device)
    call("sw_incoherent_beamform", _ptr(fpact), stride, offset_samples, F, nsamples, A,
         tscrunch, _ptr(scale), _ptr(offset), _ptr(beamset_weights), S, STOKES[stokes],
         _ptr(raw), _ptr(out), _stream(stream))
    return raw, out


def cb_shape(fpact, nsamples, nbeams, tscrunch, stokes="I", ib_subtract=True,
             offset_samples=0, tiles_per_item=0, voltage_stages=0, weight_stages=0):
    F, P, A, _, stride = fpact.shape
    return CbShape(F, nsamples, A, nbeams, tscrunch, STOKES[stokes], int(ib_subtract),
                   stride, offset_samples, tiles_per_item, voltage_stages, weight_stages)


def coherent_beamform(fpact, weights_gemm, scale, offset, mapping, ib_raw, nsamples,
                      tscrunch, stokes="I", ib_subtract=True, beam_start=0, beam_count=None,
                      out=None, debug=False, offset_samples=0, tiles_per_item=0, stream=None):
    """CoherentBeamformer::beamform (plain: one problem) -> int8 TFB.
    tiles_per_item: 64-sample tiles per work item (0: the library default)."""
    F = fpact.shape[0]
    nbeams = weights_gemm.shape[2]
    beam_count = nbeams if beam_count is None else beam_count
    if out is None:
        out = torch.zeros((nsamples // tscrunch, F, nbeams) + ((4,) if stokes == "IQUV" else ()),
                          dtype=torch.int8, device=fpact.device)
    dbg = (torch.zeros((F, nsamples, 2, nbeams, 2), dtype=torch.int32, device=fpact.device)
           if debug else None)
    shape = cb_shape(fpact, nsamples, nbeams, tscrunch, stokes, ib_subtract, offset_samples,
                     tiles_per_item)
    prob = CbProblem(fpact.data_ptr(), out.data_ptr(),
                     ib_raw.data_ptr() if ib_raw is not None else None, beam_start, beam_count)
    call("sw_coherent_beamform", ctypes.byref(shape), ctypes.byref(prob), _ptr(weights_gemm),
         _ptr(scale), _ptr(offset), _ptr(mapping), _ptr(dbg), _stream(stream))
    return (out, dbg) if debug else out


def coherent_beamform_grouped(problems, weights_gemm, scale, offset, mapping, nsamples,
                              tscrunch, stokes="I", ib_subtract=True, offset_samples=0,
                              tiles_per_item=0, voltage_stages=0, weight_stages=0, stream=None):
    """problems: list of (fpact, out, ib_raw, beam_start, beam_count).
    voltage_stages / weight_stages: copies in flight (0: library defaults)."""
    fp0 = problems[0][0]
    nbeams = weights_gemm.shape[2]
    shape = cb_shape(fp0, nsamples, nbeams, tscrunch, stokes, ib_subtract, offset_samples,
                     tiles_per_item, voltage_stages, weight_stages)
    arr = (CbProblem * len(problems))(*[
        CbProblem(p[0].data_ptr(), p[1].data_ptr(), p[2].data_ptr() if p[2] is not None else None,
                  p[3], p[4]) for p in problems])
    call("sw_coherent_beamform_grouped", ctypes.byref(shape), arr, len(problems),
         _ptr(weights_gemm), _ptr(scale), _ptr(offset), _ptr(mapping), _stream(stream))


# ------------------------------------------------------- coherent dedisp.
def dm_delay(f_ref, f, dm):
    return DM_CONST * (1 / (f_ref * f_ref) - 1 / (f * f)) * dm


def cdd_plan(centre_frequency, bandwidth, nchans, dms, fft_len=0, lag=0):
    """sw_cdd_plan (host only): the pipeline's overlap-save plan
    (fft_len, overlap, lag) for this band and DM set."""
    d = (ctypes.c_float * len(dms))(*[float(x) for x in dms])
    n, o, g = ctypes.c_int(int(fft_len)), ctypes.c_int(), ctypes.c_int()
    call("sw_cdd_plan", ctypes.c_double(centre_frequency), ctypes.c_double(bandwidth), nchans,
         d, len(dms), int(lag), ctypes.byref(n), ctypes.byref(o), ctypes.byref(g))
    return n.value, o.value, g.value


class CoherentDedisperser:
    """create_coherent_dedisperser_config + CoherentDedisperser::dedisperse for
    all channels/antennas/pols and DMs of a gulp (overlap-save with history).

    Every window trims overlap - lag samples at its start and lag at its end,
    and the output is delayed by lag samples; lag=None is the reference's
    overlap / 2 at each end (CoherentDedisperser.cu:196-223)."""

    def __init__(self, nchans, nant, fft_len, overlap, low_freq, bw, dms, device="cuda",
                 lag=None):
        self.nchans, self.nant, self.fft_len, self.overlap = nchans, nant, fft_len, overlap
        self.lag = overlap // 2 if lag is None else int(lag)
        if not 0 <= self.lag <= overlap:
            raise ValueError("lag must lie in [0, overlap]")
        self.dms = np.asarray(dms, np.float32)
        nbytes = lib().sw_cdd_setup_bytes(len(dms), nchans, fft_len)
        if nbytes == 0:
            raise ValueError(f"unsupported fft_len {fft_len}")
        self.setup = torch.empty(nbytes, dtype=torch.uint8, device=device)
        dms_c = (ctypes.c_float * len(dms))(*self.dms)
        call("sw_cdd_chirps", dms_c, len(dms), nchans, fft_len, ctypes.c_double(low_freq),
             ctypes.c_double(bw), _ptr(self.setup), _stream())

    def dedisperse(self, fpact_ext, nsamples, outs=None, stream=None, debug=False,
                   workspace_limit=2 << 30):
        """fpact_ext rows hold `overlap` history samples then the gulp.
        fft_len > 8192 runs the split transform through a device workspace of
        at most `workspace_limit` bytes (segments are processed in chunks).
        debug=True also returns the float dedispersed voltages before
        rounding, [ndms][F][P][A][nsamples][re|im]."""
        F, P, A, _, stride = fpact_ext.shape
        if F != self.nchans:
            raise ValueError(f"voltages have {F} channels but the chirp tables {self.nchans}")
        nd = len(self.dms)
        if outs is None:
            outs = [torch.empty((F, P, A, 2, nsamples), dtype=torch.int8,
                                device=fpact_ext.device) for _ in range(nd)]
        arr = (ctypes.c_void_p * nd)(*[o.data_ptr() for o in outs])
        need = lib().sw_cdd_workspace_bytes(F, P, A, nsamples, self.fft_len, self.overlap, nd)
        ws = None
        if need:
            per_seg = nd * self.fft_len * 8
            nbytes = max(per_seg, min(need, workspace_limit) // per_seg * per_seg)
            ws = torch.empty(nbytes, dtype=torch.uint8, device=fpact_ext.device)
        dbg = (torch.empty((nd, F, P, A, nsamples, 2), dtype=torch.float32,
                           device=fpact_ext.device) if debug else None)
        call("sw_coherent_dedisperse_ws", _ptr(fpact_ext), stride, F, P, A, nsamples,
             self.fft_len, self.overlap, self.lag, _ptr(self.setup), nd, arr, outs[0].shape[-1],
             _ptr(ws), ws.numel() if ws is not None else 0, _ptr(dbg), _stream(stream))
        return (outs, dbg) if debug else outs


# ----------------------------------------------------- incoherent dedisp.
def incoherent_dedisperse(tfb, delays, max_delay, tscrunch, scale_factor, stream=None):
    """IncoherentDedisperser::dedisperse: int8 TFB [T][F][B] -> TDB
    [(T - max_delay) / tscrunch][D][B].  A char4 (IQUV) TFB [T][F][B][4] is
    dedispersed per component (the reference's char4 instantiation,
    IncoherentDedisperser.cu:133-137, sums and clamps each component
    independently), i.e. as 4B int8 beams."""
    T, F, B = tfb.shape[:3]
    C = tfb.shape[3] if tfb.dim() == 4 else 1
    ndms = delays.shape[0]
    out = torch.empty(((T - max_delay) // tscrunch, ndms, B) + ((C,) if tfb.dim() == 4 else ()),
                      dtype=torch.int8, device=tfb.device)
    call("sw_incoherent_dedisperse", _ptr(tfb), T, F, B * C, _ptr(delays), ndms, max_delay,
         tscrunch, ctypes.c_float(scale_factor), _ptr(out), _stream(stream))
    return out


def autotune(nantennas, nbeams, nchans, nsamples, tscrunch, dms, centre_frequency, bandwidth,
             stream=None):
    """sw_autotune: the fastest FFT length and beamformer work-item size for
    this shape, measured on the device (cached per shape for the process)."""
    t = _lib.Tuning()
    d = (ctypes.c_float * len(dms))(*[float(x) for x in dms])
    call("sw_autotune", nantennas, nbeams, nchans, nsamples, tscrunch, len(dms), d,
         ctypes.c_double(centre_frequency), ctypes.c_double(bandwidth), ctypes.byref(t),
         _stream(stream))
    return {"fft_len": t.fft_len, "overlap": t.overlap, "lag": t.lag,
            "cb_tiles_per_item": t.cb_tiles_per_item, "cb_voltage_stages": t.cb_voltage_stages,
            "cb_weight_stages": t.cb_weight_stages,
            "cdd_ms": t.cdd_ms, "cb_ms": t.cb_ms}


class IncoherentDedispersionPipeline:
    """IncoherentDedispersionPipeline (detail/IncoherentDedispersionPipeline.cu:
    6-113) with its AggregationBuffer (detail/AggregationBuffer.cu:23-117) in
    device memory.  blocks: one (delays int [ndms][F], tscrunch, scale_factor)
    per coherent DM.  push(block, tfb) appends int8 TFB [T][F][nbeams]
    (nbeams counting Stokes components); each dispatch calls
    handler(block, tdb) with a device copy of the TDB
    [dispatch / tscrunch][ndms][nbeams]."""

    def __init__(self, nchans, nbeams, blocks, handler, dispatch=None):
        self.handler = handler
        self.nchans, self.nbeams = int(nchans), int(nbeams)
        nb = len(blocks)
        self._delays = [np.ascontiguousarray(b[0], np.int32) for b in blocks]
        ndms = (ctypes.c_int * nb)(*[d.shape[0] for d in self._delays])
        dptr = (ctypes.c_void_p * nb)(*[d.ctypes.data for d in self._delays])
        ts = (ctypes.c_int * nb)(*[int(b[1]) for b in blocks])
        sc = (ctypes.c_float * nb)(*[float(b[2]) for b in blocks])
        disp = (ctypes.c_int * nb)(*dispatch) if dispatch is not None else None
        self._cb = _lib.IDD_HANDLER(self._on_dispatch) if handler is not None else None
        h = ctypes.c_void_p()
        call("sw_idd_pipeline_create", nchans, nbeams, nb, ndms, dptr, ts, sc, disp,
             ctypes.cast(self._cb, ctypes.c_void_p) if self._cb is not None else None, None,
             ctypes.byref(h))
        self.h = h

    def _on_dispatch(self, user, block, ptr, nout, ndms, nbeams, stream):
        # runs on the pushing thread, ordered on the pushing stream
        tdb = _device_view(ptr, nout * ndms * nbeams).clone().view(torch.int8)
        self.handler(block, tdb.reshape(nout, ndms, nbeams))

    def push(self, block, tfb, stream=None):
        """Append whole time samples: like AggregationBuffer::push_back
        (AggregationBuffer.cu:53-56), a length that is not a multiple of one
        sample (nchans x nbeams bytes) raises RuntimeError."""
        row = self.nchans * self.nbeams
        n = tfb.numel()
        if tfb.dtype != torch.int8 or not tfb.is_contiguous() or n % row:
            raise RuntimeError(f"input size is not a multiple of the slot size ({n} int8 values, "
                               f"slots of {self.nchans} x {self.nbeams})")
        call("sw_idd_pipeline_push", self.h, block, _ptr(tfb), n // row, _stream(stream))

    def geometry(self, block):
        v = [ctypes.c_int() for _ in range(4)]
        call("sw_idd_pipeline_geometry", self.h, block, *[ctypes.byref(x) for x in v])
        return tuple(x.value for x in v)  # dispatch, overlap, nsamples_out, ndms

    def close(self):
        if self.h:
            lib().sw_idd_pipeline_destroy(self.h)
            self.h = None


# ------------------------------------------------------------------ pipeline
def describe(dims, sizes, centre_frequency, bandwidth, nchans, tscrunch, lag, dm):
    """The metadata the reference's DescribedVector carries beside its data
    (DescribedVector.hpp:96-573) for one pipeline output: dimension order and
    extents, channel centre frequencies (PipelineConfig.cpp:188-203), tsamp =
    tscrunch x channel sample (CoherentBeamformer.cu:235), utc_offset = the
    coherent dedisperser's filter delay, i.e. the delay of its output: `lag`
    channel samples (the reference's symmetric trim makes it tsamp * overlap / 2,
    CoherentDedisperser.cu:82) and reference_dm = the coherent DM
    (CoherentDedisperser.cu:224)."""
    chbw = bandwidth / nchans
    bottom = centre_frequency - bandwidth / 2.0
    chan_tsamp = nchans / bandwidth
    return {"dims": dims, "extents": tuple(int(x) for x in sizes),
            "frequencies": [bottom + chbw / 2.0 + chbw * i for i in range(nchans)],
            "tsamp": chan_tsamp * tscrunch, "utc_offset": chan_tsamp * lag,
            "dms": [], "reference_dm": float(dm)}


class BeamformerPipeline:
    """sw_pipeline_*: the graph-captured per-gulp chain (BeamformerPipeline)."""

    def __init__(self, *, nantennas, input_nantennas, nchans, nbeams, gulp_samples,
                 tscrunch, centre_frequency, bandwidth, dms, beamset_weights,
                 beamset_mapping, stokes="I", ib_subtract=True, output_level=24.0,
                 fft_len=0, coherent_dedispersion=True, grouped=True, use_graph=True,
                 autotune=False, cdd_lag=0):
        self._dms = (ctypes.c_float * len(dms))(*[float(d) for d in dms])
        bw = np.ascontiguousarray(beamset_weights, np.float32)
        mp = np.ascontiguousarray(beamset_mapping, np.int32)
        self._bw = bw.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
        self._mp = mp.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
        self._keep = (bw, mp)
        cfg = _lib.PipelineConfig(
            nantennas, input_nantennas, nchans, nbeams, gulp_samples, tscrunch,
            STOKES[stokes], int(ib_subtract), output_level, centre_frequency, bandwidth,
            len(dms), self._dms, fft_len, int(coherent_dedispersion), int(grouped),
            int(use_graph), bw.shape[0], self._bw, self._mp, int(autotune), int(cdd_lag))
        h = ctypes.c_void_p()
        call("sw_pipeline_create", ctypes.byref(cfg), ctypes.byref(h))
        self.h = h
        self.ndms = len(dms)
        self.nchans, self.nbeams, self.tscrunch, self.gulp = nchans, nbeams, tscrunch, gulp_samples
        self.nbeamsets = bw.shape[0]
        self._nant = nantennas
        self.stokes = stokes
        self._centre, self._bandwidth = float(centre_frequency), float(bandwidth)
        self._dm_list = [float(d) for d in dms]
        self._ib_tscrunch = tscrunch

    def close(self):
        if self.h:
            lib().sw_pipeline_destroy(self.h)
            self.h = None

    def _describe(self, dm_idx, dims, sizes, tscrunch):
        if not 0 <= dm_idx < self.ndms:
            raise IndexError(f"DM index {dm_idx} out of range")
        lag = self.cdd_plan()[2]
        return describe(dims, sizes, self._centre, self._bandwidth, self.nchans, tscrunch,
                        lag, self._dm_list[dm_idx])

    def describe_cb(self, dm_idx: int) -> dict:
        """DescribedVector metadata of one DM's coherent beams (TFB): the
        description the reference's CB handler finds on its TFBPowersD."""
        return self._describe(dm_idx, "TFB", (self.gulp // self.tscrunch, self.nchans,
                                              self.nbeams), self.tscrunch)

    def describe_ib(self, dm_idx: int) -> dict:
        """The same for the incoherent beams (BTF over beamsets)."""
        return self._describe(dm_idx, "BTF", (self.nbeamsets, self.gulp // self._ib_tscrunch,
                                              self.nchans), self._ib_tscrunch)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_delays(self, delays: np.ndarray, delay_epoch: float):
        d = np.ascontiguousarray(delays, np.float32)
        call("sw_pipeline_set_delays", self.h, d.ctypes.data_as(ctypes.c_void_p),
             ctypes.c_double(delay_epoch))

    def process_device(self, taftp: torch.Tensor, epoch: float, stream=None):
        call("sw_pipeline_process_device", self.h, _ptr(taftp), ctypes.c_double(epoch),
             _stream(stream))

    def process_host(self, taftp_pinned: torch.Tensor, epoch: float, cb_out_pinned=None,
                     stream=None):
        call("sw_pipeline_process_host", self.h, _ptr(taftp_pinned), ctypes.c_double(epoch),
             _ptr(cb_out_pinned), _stream(stream))

    def fft_plan(self):
        """(fft_len, overlap) of the coherent dedisperser."""
        return self.cdd_plan()[:2]

    def cdd_plan(self):
        """(fft_len, overlap, lag): every window trims overlap - lag samples at
        its start and lag at its end; the dedispersed voltages are delayed by
        lag samples."""
        n, o, g = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        call("sw_pipeline_fft_len", self.h, ctypes.byref(n), ctypes.byref(o), ctypes.byref(g))
        return n.value, o.value, g.value

    def cb_device(self, dm_idx: int):
        """The last gulp's coherent beams of one DM as a device tensor view
        (int8 TFB, owned by the pipeline, overwritten by the next gulp)."""
        pcb = ctypes.c_void_p()
        call("sw_pipeline_outputs", self.h, dm_idx, ctypes.byref(pcb), None, None, None)
        T = self.gulp // self.tscrunch
        shape = (T, self.nchans, self.nbeams) + ((4,) if self.stokes == "IQUV" else ())
        return _device_view(pcb.value, int(np.prod(shape))).view(torch.int8).reshape(shape)

    def voltages(self, dm_idx: int, channels=None):
        """A copy of the last gulp's voltages that fed the beamformers for one
        DM, as FPACT int8 [F][P][A][re|im][gulp] (dedispersed and delayed by the
        plan's lag, or as transposed without coherent dedispersion); only the
        given channels when `channels` is a list."""
        p, stride = ctypes.c_void_p(), ctypes.c_size_t()
        call("sw_pipeline_voltages", self.h, dm_idx, ctypes.byref(p), ctypes.byref(stride))
        torch.cuda.synchronize()
        rows = self.nchans * 2 * self._nant * 2
        v = _device_view(p.value, (rows - 1) * stride.value + self.gulp).view(torch.int8)
        v = v.as_strided((self.nchans, 4 * self._nant, self.gulp), (4 * self._nant * stride.value,
                                                                     stride.value, 1))
        if channels is not None:
            v = v[list(channels)]
        return v.cpu().numpy().reshape(v.shape[0], 2, self._nant, 2, self.gulp)

    def cb_bytes_per_dm(self):
        return lib().sw_pipeline_cb_bytes_per_dm(self.h)

    def outputs(self, dm_idx: int):
        """Copies of the last gulp's outputs for one DM (numpy)."""
        pcb, praw, pib, pst = (ctypes.c_void_p() for _ in range(4))
        call("sw_pipeline_outputs", self.h, dm_idx, ctypes.byref(pcb), ctypes.byref(praw),
             ctypes.byref(pib), ctypes.byref(pst))
        torch.cuda.synchronize()
        check_device_error()
        T = self.gulp // self.tscrunch
        S, F, B = self.nbeamsets, self.nchans, self.nbeams
        C = (4,) if self.stokes == "IQUV" else ()
        res = {}
        for name, p, dt, shape in (("cb", pcb, np.int8, (T, F, B) + C),
                                   ("ib_raw", praw, np.float32, (S, T, F) + C),
                                   ("ib", pib, np.int8, (S, T, F) + C),
                                   ("stats", pst, np.float32, (F, 2, -1, 4))):
            n = int(np.prod([x for x in shape if x > 0]))
            if name == "stats":
                n = F * 2 * (self._nant if hasattr(self, "_nant") else 0) * 4
                if n == 0:
                    continue
            nbytes = n * np.dtype(dt).itemsize
            res[name] = _device_view(p.value, nbytes).cpu().numpy().view(dt).reshape(shape)
        return res


def _device_view(ptr, nbytes):
    # Build a uint8 CUDA tensor aliasing `ptr` (owned by the pipeline).
    class _Arr:
        __cuda_array_interface__ = {"shape": (nbytes,), "typestr": "|u1",
                                    "data": (ptr, False), "version": 3}
    return torch.as_tensor(_Arr(), device="cuda")
