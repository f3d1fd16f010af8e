"""DADA ingest and output around the pipeline (ctypes over sw_dada_*).

Reference: cpp/skyweaver/src/ObservationHeader.cpp:6-62,
cpp/skyweaver/src/MultiFileReader.cu:34-303,
cpp/skyweaver/detail/MultiFileWriter.cu:74-243 and
cpp/skyweaver/src/FileOutputStream.cpp:80-150.
"""
from __future__ import annotations

import ctypes
import datetime
import os
import threading

import numpy as np

from ._lib import call, lib

_c = ctypes


class ObservationHeader(_c.Structure):
    _fields_ = [(k, _c.c_size_t) for k in ("nchans", "npol", "nbits", "nantennas",
                                            "sample_clock_start", "chan0_idx", "obs_nchans",
                                            "obs_offset")] + \
               [(k, _c.c_double) for k in ("bandwidth", "obs_bandwidth", "frequency",
                                           "obs_frequency", "tsamp", "sample_clock", "sync_time",
                                           "utc_start", "mjd_start")] + \
               [("source_name", _c.c_char * 64), ("ra", _c.c_char * 32), ("dec", _c.c_char * 32),
                ("telescope", _c.c_char * 32), ("instrument", _c.c_char * 32)]

    def as_dict(self):
        return {k: (getattr(self, k).decode() if isinstance(getattr(self, k), bytes)
                    else getattr(self, k)) for k, _ in self._fields_}


def _sigs():
    L = lib()
    P = _c.POINTER
    for name, res, args in (
            ("sw_dada_header_get", _c.c_int, [_c.c_char_p, _c.c_size_t, _c.c_char_p, _c.c_char_p,
                                              _c.c_size_t]),
            ("sw_dada_parse_header", _c.c_int, [_c.c_char_p, _c.c_size_t, P(ObservationHeader)]),
            ("sw_dada_validate_header", _c.c_int, [P(ObservationHeader), _c.c_int, _c.c_int,
                                                   _c.c_int]),
            ("sw_dada_reader_open", _c.c_int, [P(_c.c_char_p), _c.c_int, _c.c_size_t, _c.c_int,
                                               P(_c.c_void_p)]),
            ("sw_dada_reader_close", None, [_c.c_void_p]),
            ("sw_dada_reader_header", _c.c_int, [_c.c_void_p, _c.c_int, P(ObservationHeader)]),
            ("sw_dada_reader_total_bytes", _c.c_size_t, [_c.c_void_p]),
            ("sw_dada_reader_tell", _c.c_size_t, [_c.c_void_p]),
            ("sw_dada_reader_seek", _c.c_int, [_c.c_void_p, _c.c_size_t]),
            ("sw_dada_reader_read", _c.c_int, [_c.c_void_p, _c.c_void_p, _c.c_size_t,
                                               P(_c.c_size_t)]),
            ("sw_dada_writer_open", _c.c_int, [_c.c_char_p, _c.c_char_p, _c.c_char_p, _c.c_size_t,
                                               _c.c_char_p, _c.c_size_t, P(_c.c_void_p)]),
            ("sw_dada_writer_set", _c.c_int, [_c.c_void_p, _c.c_char_p, _c.c_char_p]),
            ("sw_dada_writer_write", _c.c_int, [_c.c_void_p, _c.c_void_p, _c.c_size_t]),
            ("sw_dada_writer_close", _c.c_int, [_c.c_void_p])):
        fn = getattr(L, name)
        fn.restype, fn.argtypes = res, args


_ready = False


def _init():
    global _ready
    if not _ready:
        _sigs()
        _ready = True


def header_get(header: bytes, key: str) -> str:
    _init()
    buf = _c.create_string_buffer(1024)
    call("sw_dada_header_get", header, len(header), key.encode(), buf, len(buf))
    return buf.value.decode()


def parse_header(header: bytes) -> ObservationHeader:
    _init()
    h = ObservationHeader()
    call("sw_dada_parse_header", header, len(header), _c.byref(h))
    return h


def validate_header(h: ObservationHeader, nantennas: int, nchans: int, npol: int = 2):
    _init()
    call("sw_dada_validate_header", _c.byref(h), nantennas, nchans, npol)


class MultiFileReader:
    """MultiFileReader: DADA files as one contiguous payload."""

    def __init__(self, files, header_size=4096, check_contiguity=False):
        _init()
        arr = (_c.c_char_p * len(files))(*[os.fsencode(f) for f in files])
        h = _c.c_void_p()
        call("sw_dada_reader_open", arr, len(files), header_size, int(check_contiguity),
             _c.byref(h))
        self.h = h
        self.nfiles = len(files)

    def header(self, file_idx=0) -> ObservationHeader:
        out = ObservationHeader()
        call("sw_dada_reader_header", self.h, file_idx, _c.byref(out))
        return out

    def total_bytes(self):
        return lib().sw_dada_reader_total_bytes(self.h)

    def tell(self):
        return lib().sw_dada_reader_tell(self.h)

    def seek(self, offset):
        call("sw_dada_reader_seek", self.h, offset)

    def read_into(self, ptr, nbytes):
        got = _c.c_size_t()
        call("sw_dada_reader_read", self.h, _c.c_void_p(ptr), nbytes, _c.byref(got))
        return got.value

    def read(self, nbytes) -> np.ndarray:
        buf = np.empty(nbytes, np.int8)
        n = self.read_into(buf.ctypes.data, nbytes)
        return buf[:n]

    def close(self):
        if self.h:
            lib().sw_dada_reader_close(self.h)
            self.h = None


class GulpReader:
    """Reads fixed-size gulps into two pinned host buffers on a background
    thread, so that the file read of gulp g+1 overlaps the processing of
    gulp g (the reference CLI's std::thread reader, skyweaver_cli.cu:186-237).
    Iterating yields (pinned uint8 tensor, gulp index); the buffer is reused
    two gulps later."""

    def __init__(self, reader: MultiFileReader, gulp_bytes: int):
        import torch
        self.reader, self.gulp_bytes = reader, gulp_bytes
        self.bufs = [torch.empty(gulp_bytes, dtype=torch.int8, pin_memory=True) for _ in range(2)]
        self._ready = [threading.Event(), threading.Event()]
        self._free = [threading.Event(), threading.Event()]
        for e in self._free:
            e.set()
        self._n = [0, 0]
        self._stop = False
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()

    def _run(self):
        i = 0
        while not self._stop:
            k = i & 1
            self._free[k].wait()
            self._free[k].clear()
            n = self.reader.read_into(self.bufs[k].data_ptr(), self.gulp_bytes)
            self._n[k] = n
            self._ready[k].set()
            if n < self.gulp_bytes:
                return
            i += 1

    def __iter__(self):
        i = 0
        while True:
            k = i & 1
            self._ready[k].wait()
            self._ready[k].clear()
            if self._n[k] < self.gulp_bytes:
                return
            yield self.bufs[k], i
            self._free[k].set()
            i += 1

    def close(self):
        self._stop = True
        for e in self._free:
            e.set()
        self._t.join(timeout=5)


DEFAULT_HEADER = """HEADER       DADA
HDR_VERSION  1.0
HDR_SIZE     4096
DADA_VERSION 1.0
FILE_SIZE    0
FILE_NUMBER  0
NBIT         8
NDIM         1
NPOL         1
"""


class FileStream:
    """FileStream: a payload split over DADA files of bytes_per_file."""

    def __init__(self, directory, base_filename, extension, bytes_per_file,
                 header_template=DEFAULT_HEADER, header_size=4096):
        _init()
        h = _c.c_void_p()
        call("sw_dada_writer_open", os.fsencode(directory), base_filename.encode(),
             extension.encode(), bytes_per_file, header_template.encode(), header_size,
             _c.byref(h))
        self.h = h

    def set(self, key, value):
        call("sw_dada_writer_set", self.h, key.encode(), str(value).encode())

    def write(self, array: np.ndarray):
        a = np.ascontiguousarray(array)
        call("sw_dada_writer_write", self.h, _c.c_void_p(a.ctypes.data), a.nbytes)

    def close(self):
        if self.h:
            lib().sw_dada_writer_close(self.h)
            self.h = None


def formatted_time(unix_timestamp: float) -> str:
    """get_formatted_time (MultiFileWriter.cu:64-71): %Y-%m-%d-%H:%M:%S, UTC."""
    return datetime.datetime.fromtimestamp(int(unix_timestamp), datetime.timezone.utc) \
        .strftime("%Y-%m-%d-%H:%M:%S")


def output_paths(output_dir, header: dict, stream_idx, reference_dm, dims, prefix="", tag=""):
    """MultiFileWriter's output directory, base file name and extension
    (MultiFileWriter.cu:170-221):
    <out>/<utc>/<stream>/<freq %09d> and
    [<prefix>_]<utc>_<stream>_<dm %09.3f>_<freq %09.0f>[_<tag>], .<dims lower>."""
    utc = formatted_time(header["utc_start"])
    d = f"{output_dir}/{utc}/{stream_idx}/{int(header['frequency']):09d}"
    base = (f"{prefix}_" if prefix else "") + \
        f"{utc}_{stream_idx}_{reference_dm:09.3f}_{header['frequency']:09.0f}"
    if tag:
        base += f"_{tag}"
    return d, base, "." + dims.lower()
