"""DADA ingest and output (host I/O, no GPU): header parsing like
read_dada_header (ObservationHeader.cpp:6-33), the multi-file reader's
contiguous payload, seek and OBS_OFFSET contiguity check
(MultiFileReader.cu:34-303), and the size-split writer's files and headers
(FileOutputStream.cpp:80-150), read back by the reader."""
import os

import numpy as np
import pytest

from conftest import REPO  # noqa: F401  (puts the repository on sys.path)

HEADER_KEYS = {
    "NCHAN": "64", "OBS_NCHAN": "4096", "NPOL": "2", "NBIT": "8", "NANT": "57",
    "SAMPLE_CLOCK_START": "12345678", "BW": "13375000.0", "OBS_BW": "856000000.0",
    "FREQ": "1284000000.0", "OBS_FREQ": "1284000000.0", "TSAMP": "4.785046728971962",
    "SAMPLE_CLOCK": "1712000000.0", "SYNC_TIME": "1708039531.0",
    "UTC_START": "1708082229.000020336", "MJD_START": "60356.47024305579093",
    "SOURCE": "J1644-4559", "RA": "16:44:49.27", "DEC": "-45:59:09.7",
    "TELESCOPE": "MeerKAT", "INSTRUMENT": "CBF-Feng", "CHAN0_IDX": "2688",
}


def _header(obs_offset, size=4096, **over):
    keys = dict(HEADER_KEYS, OBS_OFFSET=str(obs_offset), **over)
    text = "HEADER DADA\nHDR_SIZE 4096\n" + "".join(f"{k} {v}\n" for k, v in keys.items())
    return text.encode().ljust(size, b"\0")


def _write_files(tmp_path, payload, splits, gap=0):
    files, off = [], 0
    for i, n in enumerate(splits):
        p = tmp_path / f"f{i}.dada"
        p.write_bytes(_header(off + (gap if i == len(splits) - 1 and i else 0))
                      + payload[off:off + n].tobytes())
        files.append(str(p))
        off += n
    return files


def test_parse_header_and_validate():
    from skyweaver_b200 import dada
    h = dada.parse_header(_header(0))
    d = h.as_dict()
    assert d["nchans"] == 64 and d["nantennas"] == 57 and d["chan0_idx"] == 2688
    assert d["frequency"] == 1284e6 and d["source_name"] == "J1644-4559"
    assert abs(d["utc_start"] - 1708082229.000020336) < 1e-6
    assert dada.header_get(_header(0), "MJD_START") == "60356.47024305579093"
    dada.validate_header(h, 64, 64, 2)
    with pytest.raises(Exception, match="too many antennas"):
        dada.validate_header(h, 32, 64, 2)
    with pytest.raises(Exception, match="NANT"):
        bad = _header(0).replace(b"NANT 57", b"XANT 57")
        dada.parse_header(bad)
    with pytest.raises(Exception, match="unset"):
        dada.parse_header(_header(0, SOURCE="unset"))


def test_reader_spans_files_and_seeks(tmp_path):
    from skyweaver_b200 import dada
    rng = np.random.default_rng(1)
    payload = rng.integers(-128, 128, 30000, dtype=np.int8)
    files = _write_files(tmp_path, payload, [10000, 7000, 13000])
    r = dada.MultiFileReader(files, check_contiguity=True)
    assert r.total_bytes() == 30000
    got = np.concatenate([r.read(4096) for _ in range(8)])
    assert np.array_equal(got, payload)            # last read is short
    r.seek(9990)
    assert np.array_equal(r.read(20), payload[9990:10010])
    assert r.tell() == 10010
    r.seek(17000)
    assert np.array_equal(r.read(5), payload[17000:17005])
    r.close()
    gap_files = _write_files(tmp_path, payload, [10000, 20000], gap=5)
    with pytest.raises(Exception, match="not contiguous"):
        dada.MultiFileReader(gap_files, check_contiguity=True)


def test_writer_splits_and_reads_back(tmp_path):
    from skyweaver_b200 import dada
    rng = np.random.default_rng(2)
    data = rng.integers(-128, 128, (5, 3000), dtype=np.int8)
    out = tmp_path / "out"
    w = dada.FileStream(str(out), "beams", ".tfb", 4096)
    w.set("NBEAM", 64)
    w.set("ORDER", "TFB")
    for row in data:
        w.write(row)
    w.close()
    names = sorted(os.listdir(out))
    assert names == [f"beams_{k * 4096:016d}.tfb" for k in range(4)]
    files = [str(out / n) for n in names]
    hdrs = [open(f, "rb").read(4096) for f in files]
    for k, h in enumerate(hdrs):
        assert dada.header_get(h, "FILE_NUMBER") == str(k)
        assert dada.header_get(h, "OBS_OFFSET") == str(k * 4096)
        assert dada.header_get(h, "FILE_SIZE") == "4096"
        assert dada.header_get(h, "NBEAM") == "64"
        assert dada.header_get(h, "HDR_SIZE") == "4096"
    payload = b"".join(open(f, "rb").read()[4096:] for f in files)
    assert payload == data.tobytes()


def test_output_paths_follow_multifilewriter():
    from skyweaver_b200 import dada
    d, base, ext = dada.output_paths("/data", {"utc_start": 1708082229.0, "frequency": 1284e6},
                                     3, 150.0, "TDB", prefix="sw", tag="cb")
    assert d == "/data/2024-02-16-11:17:09/3/1284000000"
    assert base == "sw_2024-02-16-11:17:09_3_00150.000_1284000000_cb"
    assert ext == ".tdb"


def test_reader_eof_zero_size_and_missing_file(tmp_path):
    """MultiFileReaderTester.cu:97-130: seeking to the payload's end is legal
    and leaves nothing to read, one byte past it raises, a read of 0 bytes
    returns 0, and a file that does not exist raises when the reader opens."""
    from skyweaver_b200 import dada
    payload = np.arange(3000, dtype=np.int64).astype(np.int8)
    r = dada.MultiFileReader(_write_files(tmp_path, payload, [1000, 2000]))
    r.seek(r.total_bytes())
    assert r.tell() == r.total_bytes() == 3000
    assert len(r.read(10)) == 0
    with pytest.raises(Exception, match="Invalid seek position"):
        r.seek(r.total_bytes() + 1)
    r.seek(0)
    assert len(r.read(0)) == 0 and r.tell() == 0
    r.close()
    with pytest.raises(Exception, match="Could not open file"):
        dada.MultiFileReader([str(tmp_path / "non_existent_file.dada")])
