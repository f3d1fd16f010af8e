"""bench.py host logic that needs no GPU: the clock summary that goes into
the JSON line (median SM clock under load, every slowdown reason seen)."""
import os
import sys

from conftest import REPO

sys.path.insert(0, REPO)
import bench  # noqa: E402


def _clocks(rows):
    c = bench.Clocks(0)
    c.rows = rows
    return c.summary()


def test_clock_summary_median_under_load_and_reasons():
    idle = [(1965.0, 1965.0, 120.0, set())] * 5
    load = [(1965.0, 1965.0, 900.0, set()), (1860.0, 1965.0, 990.0, {"sw_power_cap"}),
            (1965.0, 1965.0, 950.0, set())]
    s = _clocks(idle + load)
    assert s["samples"] == 8 and s["samples_under_load"] == 3
    assert s["sm_mhz"] == 1965.0 and s["sm_max_mhz"] == 1965.0
    assert s["reasons"] == ["sw_power_cap"]
    assert s["power_w_median"] == 950.0


def test_clock_summary_without_samples():
    s = _clocks([])
    assert s == {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}


def test_clock_summary_reads_nvidia_smi_rows(tmp_path):
    c = bench.Clocks(0)
    c.f = open(os.path.join(tmp_path, "clk.csv"), "w+")
    c.f.write("1965, 1965, 800.5, 0x0, Not Active, Not Active, Not Active, Not Active\n"
              "1900, 1965, 990.1, 0x4, Not Active, Not Active, Not Active, Active\n")
    s = c.summary()
    assert s["samples"] == 2 and s["reasons"] == ["sw_power_cap"]
    assert s["source"] == "nvidia-smi 200 ms"


def test_workload_gulp_tones_and_pulse(monkeypatch):
    """The benchmark gulp (here 2 antennas): sigma-8 voltages, the three RFI
    channels saturated by their tones, and the DM-100 pulse a quarter into the
    gulp at the top channel, arriving later in lower channels."""
    import torch
    monkeypatch.setitem(bench.WORK, "nant", 2)
    centre, bw = bench.WORK["centre"], bench.WORK["nchans"] * bench.WORK["chbw"]
    gen = torch.Generator().manual_seed(1)
    v = bench.workload_gulp(torch, gen, centre, bw, pulse=True, device="cpu")
    T, F = bench.WORK["gulp"], bench.WORK["nchans"]
    assert v.shape == (T // 256, 2, F, 256, 2, 2) and v.dtype == torch.int8
    level = v.float().abs().mean(dim=(0, 1, 3, 4, 5))           # per channel
    quiet = [c for c in range(F) if c not in bench.RFI_CHANNELS]
    assert level[quiet].max() < 8 and level[list(bench.RFI_CHANNELS)].min() > 80
    power = (v.float() ** 2).sum(dim=(1, 4, 5)).permute(1, 0, 2).reshape(F, T)
    peak = power.argmax(dim=1)
    assert abs(int(peak[F - 1]) - T // 4) < 64
    assert int(peak[0]) > int(peak[F // 2]) > int(peak[F - 1])
    plain = bench.workload_gulp(torch, gen, centre, bw, pulse=False, device="cpu")
    assert (plain.float() ** 2).sum(dim=(1, 4, 5)).permute(1, 0, 2).reshape(F, T)[0].max() < \
        power[0].max()
