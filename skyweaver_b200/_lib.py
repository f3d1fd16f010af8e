"""ctypes binding of libskyweaver_b200.so (the C ABI in include/skyweaver_b200.h).

The library is built in-tree by ``skyweaver_b200.build``.  Loading fails
loudly when it is missing: there is no CPU fallback for any stage.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libskyweaver_b200.so")

c_int, c_size_t, c_double, c_float = ctypes.c_int, ctypes.c_size_t, ctypes.c_double, ctypes.c_float
c_void_p = ctypes.c_void_p
c_float_p = ctypes.POINTER(ctypes.c_float)

SW_OK = 0
SW_ERR_TIMEOUT = 4  # a bounded device-side wait gave up
IDD_HANDLER = ctypes.CFUNCTYPE(None, c_void_p, c_int, c_void_p, c_int, c_int, c_int, c_void_p)
STOKES = {"I": 0, "Q": 1, "U": 2, "V": 3, "IQUV": 4}


class SkyweaverError(RuntimeError):
    """Raised for a non-zero status from the C ABI (the reference throws
    std::runtime_error in the same situations)."""

    def __init__(self, status: int, message: str):
        super().__init__(f"[status {status}] {message}")
        self.status = status


class CbProblem(ctypes.Structure):
    _fields_ = [("d_fpact", c_void_p), ("d_out", c_void_p), ("d_ib_raw", c_void_p),
                ("beam_start", c_int), ("beam_count", c_int)]


class CbShape(ctypes.Structure):
    _fields_ = [("nchans", c_int), ("nsamples", c_int), ("nantennas", c_int),
                ("nbeams", c_int), ("tscrunch", c_int), ("stokes", c_int),
                ("ib_subtract", c_int), ("row_stride", c_size_t),
                ("sample_offset", c_size_t), ("tiles_per_item", c_int),
                ("voltage_stages", c_int), ("weight_stages", c_int)]


class PipelineConfig(ctypes.Structure):
    _fields_ = [("nantennas", c_int), ("input_nantennas", c_int), ("nchans", c_int),
                ("nbeams", c_int), ("gulp_samples", c_int), ("tscrunch", c_int),
                ("stokes", c_int), ("ib_subtract", c_int), ("output_level", c_float),
                ("centre_frequency", c_double), ("bandwidth", c_double),
                ("ndms", c_int), ("dms", c_float_p), ("fft_len", c_int),
                ("enable_coherent_dedispersion", c_int), ("grouped", c_int),
                ("use_graph", c_int), ("nbeamsets", c_int),
                ("beamset_weights", c_float_p), ("beamset_mapping", ctypes.POINTER(c_int)),
                ("autotune", c_int), ("cdd_lag", c_int)]


class Tuning(ctypes.Structure):
    _fields_ = [("fft_len", c_int), ("overlap", c_int), ("lag", c_int), ("cb_tiles_per_item", c_int),
                ("cdd_ms", c_float), ("cb_ms", c_float), ("cb_voltage_stages", c_int),
                ("cb_weight_stages", c_int)]


_SIGS = {
    "sw_version": (c_int, []),
    "sw_last_error": (ctypes.c_char_p, []),
    "sw_read_device_error": (c_int, [ctypes.POINTER(c_int)]),
    "sw_reset_device_error": (c_int, []),
    "sw_cb_timeout_selftest": (c_int, [c_int, c_void_p]),
    "sw_transpose_ftpa": (c_int, [c_void_p, c_void_p, c_int, c_int, c_int, c_int, c_void_p]),
    "sw_transpose_fpact": (c_int, [c_void_p, c_void_p, c_int, c_int, c_int, c_int,
                                   c_size_t, c_size_t, c_void_p]),
    "sw_ftpa_to_fpact": (c_int, [c_void_p, c_void_p, c_int, c_int, c_int, c_size_t,
                                 c_size_t, c_void_p]),
    "sw_fpact_to_ftpa": (c_int, [c_void_p, c_void_p, c_int, c_int, c_int, c_size_t,
                                 c_size_t, c_void_p]),
    "sw_fpact_keep_history": (c_int, [c_void_p, c_size_t, c_size_t, c_size_t, c_void_p]),
    "sw_fpact_copy_history": (c_int, [c_void_p, c_void_p, c_size_t, c_size_t, c_size_t,
                                      c_void_p]),
    "sw_statistics_scratch_bytes": (c_size_t, [c_int, c_int, c_int]),
    "sw_statistics": (c_int, [c_void_p, c_size_t, c_size_t, c_int, c_int, c_int, c_int,
                              c_void_p, c_void_p, c_void_p]),
    "sw_transpose_fpact_statistics": (c_int, [c_void_p, c_void_p, c_int, c_int, c_int, c_int,
                                              c_size_t, c_size_t, c_void_p, c_void_p,
                                              c_void_p]),
    "sw_statistics_noalloc": (c_int, [c_void_p, c_size_t, c_size_t, c_int, c_int, c_int, c_int,
                                      c_void_p, c_void_p]),
    "sw_update_scalings": (c_int, [c_void_p, c_void_p, c_int, c_int, c_int, c_int, c_int,
                                   c_int, c_float, c_void_p, c_void_p, c_void_p, c_void_p,
                                   c_void_p]),
    "sw_generate_weights": (c_int, [c_void_p, c_void_p, c_int, c_int, c_int, c_double,
                                    c_double, c_void_p, c_void_p, c_void_p]),
    "sw_pack_weights": (c_int, [c_void_p, c_void_p, c_int, c_int, c_int, c_void_p]),
    "sw_incoherent_beamform": (c_int, [c_void_p, c_size_t, c_size_t, c_int, c_int, c_int,
                                       c_int, c_void_p, c_void_p, c_void_p, c_int, c_int,
                                       c_void_p, c_void_p, c_void_p]),
    "sw_coherent_beamform": (c_int, [ctypes.POINTER(CbShape), ctypes.POINTER(CbProblem),
                                     c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                                     c_void_p]),
    "sw_coherent_beamform_grouped": (c_int, [ctypes.POINTER(CbShape),
                                             ctypes.POINTER(CbProblem), c_int, c_void_p,
                                             c_void_p, c_void_p, c_void_p, c_void_p]),
    "sw_cdd_setup_bytes": (c_size_t, [c_int, c_int, c_int]),
    "sw_cdd_chirps": (c_int, [c_float_p, c_int, c_int, c_int, c_double, c_double, c_void_p,
                              c_void_p]),
    "sw_coherent_dedisperse": (c_int, [c_void_p, c_size_t, c_int, c_int, c_int, c_int, c_int,
                                       c_int, c_int, c_void_p, c_int, ctypes.POINTER(c_void_p),
                                       c_size_t, c_void_p]),
    "sw_cdd_workspace_bytes": (c_size_t, [c_int, c_int, c_int, c_int, c_int, c_int, c_int]),
    "sw_coherent_dedisperse_ws": (c_int, [c_void_p, c_size_t, c_int, c_int, c_int, c_int, c_int,
                                          c_int, c_int, c_void_p, c_int, ctypes.POINTER(c_void_p),
                                          c_size_t, c_void_p, c_size_t, c_void_p, c_void_p]),
    "sw_coherent_dedisperse_channel": (c_int, [c_void_p, c_size_t, c_int, c_int, c_int, c_int,
                                               c_int, c_int, c_void_p, c_int, c_int, c_int,
                                               c_int, c_void_p, c_size_t, c_void_p, c_size_t,
                                               c_void_p]),
    "sw_idd_pipeline_create": (c_int, [c_int, c_int, c_int, ctypes.POINTER(c_int),
                                       ctypes.POINTER(c_void_p), ctypes.POINTER(c_int),
                                       c_float_p, ctypes.POINTER(c_int), c_void_p, c_void_p,
                                       ctypes.POINTER(c_void_p)]),
    "sw_idd_pipeline_destroy": (None, [c_void_p]),
    "sw_idd_pipeline_push": (c_int, [c_void_p, c_int, c_void_p, c_size_t, c_void_p]),
    "sw_idd_pipeline_geometry": (c_int, [c_void_p, c_int, ctypes.POINTER(c_int),
                                         ctypes.POINTER(c_int), ctypes.POINTER(c_int),
                                         ctypes.POINTER(c_int)]),
    "sw_autotune": (c_int, [c_int, c_int, c_int, c_int, c_int, c_int, c_float_p, c_double,
                            c_double, ctypes.POINTER(Tuning), c_void_p]),
    "sw_incoherent_dedisperse": (c_int, [c_void_p, c_int, c_int, c_int, c_void_p, c_int,
                                         c_int, c_int, c_float, c_void_p, c_void_p]),
    "sw_pipeline_create": (c_int, [ctypes.POINTER(PipelineConfig), ctypes.POINTER(c_void_p)]),
    "sw_pipeline_destroy": (c_int, [c_void_p]),
    "sw_pipeline_set_delays": (c_int, [c_void_p, c_void_p, c_double]),
    "sw_pipeline_process_device": (c_int, [c_void_p, c_void_p, c_double, c_void_p]),
    "sw_pipeline_process_host": (c_int, [c_void_p, c_void_p, c_double, c_void_p, c_void_p]),
    "sw_pipeline_outputs": (c_int, [c_void_p, c_int, ctypes.POINTER(c_void_p),
                                    ctypes.POINTER(c_void_p), ctypes.POINTER(c_void_p),
                                    ctypes.POINTER(c_void_p)]),
    "sw_pipeline_cb_bytes_per_dm": (c_size_t, [c_void_p]),
    "sw_cdd_plan": (c_int, [c_double, c_double, c_int, c_float_p, c_int, c_int,
                            ctypes.POINTER(c_int), ctypes.POINTER(c_int), ctypes.POINTER(c_int)]),
    "sw_pipeline_gulp_count": (ctypes.c_long, [c_void_p]),
    "sw_pipeline_gulp_outputs": (c_int, [c_void_p, ctypes.c_long, c_int,
                                         ctypes.POINTER(c_void_p), ctypes.POINTER(c_void_p),
                                         ctypes.POINTER(c_void_p), ctypes.POINTER(c_void_p)]),
    "sw_pipeline_wait_input": (c_int, [c_void_p]),
    "sw_pipeline_order_after": (c_int, [c_void_p, c_void_p]),
    "sw_pipeline_voltages": (c_int, [c_void_p, c_int, ctypes.POINTER(c_void_p),
                                     ctypes.POINTER(c_size_t)]),
    "sw_pipeline_fft_len": (c_int, [c_void_p, ctypes.POINTER(c_int), ctypes.POINTER(c_int),
                                    ctypes.POINTER(c_int)]),
}

_lib = None


def lib():
    """Load the shared library once; raise if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -m skyweaver_b200.build` "
                "(the beamforming path has no CPU fallback)")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            fn = getattr(L, name, None)
            if fn is None:
                continue
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def exported_symbols():
    return list(_SIGS)


def check(status: int) -> None:
    if status != SW_OK:
        msg = lib().sw_last_error()
        raise SkyweaverError(status, msg.decode() if msg else "unknown error")


def call(name: str, *args) -> None:
    check(getattr(lib(), name)(*args))
