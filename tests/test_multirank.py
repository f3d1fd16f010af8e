"""The N>1 path of bench.py on CPU: two gloo ranks, each beamforming its own
subband through the oracle, with the max-over-ranks timing reduction.

The beamforming path partitions by channel with no exchange, so what needs
checking is the decomposition itself: adjacent, disjoint subbands that tile
the band, per-rank results equal to a single-process run over the same
subbands, and the timing reduction returning the slowest rank."""
import os
import socket
import subprocess
import sys

import numpy as np
import pytest

from conftest import REPO

torch = pytest.importorskip("torch")


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _subband_beams(oracle, centre, bw, seed):
    """Oracle coherent beams of a tiny seeded case on one rank's subband."""
    from skyweaver_b200 import synthetic
    F, A, B, T, ts = 4, 8, 16, 256, 4
    g = synthetic.rng(seed)
    freqs = centre - bw / 2 + (bw / F) * (np.arange(F) + 0.5)
    ftpa = np.clip(np.rint(g.normal(0, 8, size=(F, T, 2, A, 2))), -127, 127).astype(np.int8)
    w = oracle.weights(synthetic.delay_model(g, B, A), freqs, 0.0, 0.0)
    one = np.ones(F, np.float32)
    return oracle.coherent_beam(ftpa, w, ts, one * 1e4, one * 0, np.ones((1, A), np.float32),
                                np.zeros(B, np.int32))


def _rank_main(rank, world, port, out_dir):
    import torch.distributed as dist
    sys.path.insert(0, REPO)
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import bench
    import swb_oracle as oracle
    oracle.build()
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world)
    try:
        centre, bw = bench.rank_subband(rank, world)
        got = torch.zeros(world, dtype=torch.float64)
        got[rank] = centre
        dist.all_reduce(got)
        slowest = bench.max_over_ranks(10.0 + rank, world)
        beams = _subband_beams(oracle, centre, bw, 100 + rank)
        np.save(os.path.join(out_dir, f"rank{rank}.npy"), beams)
        np.save(os.path.join(out_dir, f"meta{rank}.npy"),
                np.array([centre, bw, slowest] + got.tolist()))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks(tmp_path, oracle):
    import torch.multiprocessing as mp
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world,
                       join=True, start_method="spawn")
    sys.path.insert(0, REPO)
    import bench
    F, chbw = bench.WORK["nchans"], bench.WORK["chbw"]
    metas = [np.load(tmp_path / f"meta{r}.npy") for r in range(world)]
    for r, m in enumerate(metas):
        centre, bw, slowest = m[:3]
        assert slowest == 10.0 + world - 1             # max over ranks
        assert np.allclose(m[3:], [x[0] for x in metas])  # every rank saw every centre
        assert bw == F * chbw
    # adjacent, disjoint subbands tiling [centre - world*bw/2, centre + world*bw/2]
    lo = [m[0] - m[1] / 2 for m in metas]
    hi = [m[0] + m[1] / 2 for m in metas]
    assert np.isclose(hi[0], lo[1])
    assert np.isclose((lo[0] + hi[-1]) / 2, bench.WORK["centre"])
    # each rank's output equals the same subband computed in one process
    for r, m in enumerate(metas):
        ref = _subband_beams(oracle, m[0], m[1], 100 + r)
        assert np.array_equal(np.load(tmp_path / f"rank{r}.npy"), ref)


def test_reference_arm_nonzero_rank_does_no_work():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(REPO, "bench.py"), "--impl", "reference",
                        "--gpus", "2", "--steps", "1", "--warmup", "0"],
                       capture_output=True, text=True, timeout=120, env=env)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""


def _exchange_main(rank, world, port, out_dir):
    import torch
    import torch.distributed as dist
    sys.path.insert(0, REPO)
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    from skyweaver_b200 import subbands
    import swb_oracle as oracle
    oracle.build()
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world)
    try:
        T, F, B = 600, 16, 24
        full = np.random.default_rng(7).integers(-128, 128, size=(T, F, B), dtype=np.int8)
        mine = torch.from_numpy(np.ascontiguousarray(full[:, subbands.rank_channels(F, world, rank)]))
        got = subbands.channels_to_beams(mine).numpy()
        np.save(os.path.join(out_dir, f"beams{rank}.npy"), got)
        # incoherent dedispersion of this rank's beams over the whole band
        freqs = 1284e6 + (np.arange(F) - F / 2) * 0.8359375e6
        delays, maxd = oracle.idd_delays(freqs, np.array([0, 40, 80], np.float32), 1.9e-5)
        n = T - (T - maxd) % 2
        tdb = oracle.idd(np.ascontiguousarray(got[:n]), delays, maxd, 2, np.float32(4.0))
        np.save(os.path.join(out_dir, f"tdb{rank}.npy"), tdb)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_channel_partition_exchange_to_beam_blocks(tmp_path, oracle):
    """Channel-partitioned ranks + one all-to-all give each rank every
    channel of its beam block, and the incoherent dedispersion of those
    blocks equals that of the single-process array."""
    import torch.multiprocessing as mp
    world = 2
    mp.start_processes(_exchange_main, args=(world, _free_port(), str(tmp_path)), nprocs=world,
                       join=True, start_method="spawn")
    sys.path.insert(0, REPO)
    from skyweaver_b200 import subbands
    T, F, B = 600, 16, 24
    full = np.random.default_rng(7).integers(-128, 128, size=(T, F, B), dtype=np.int8)
    freqs = 1284e6 + (np.arange(F) - F / 2) * 0.8359375e6
    delays, maxd = oracle.idd_delays(freqs, np.array([0, 40, 80], np.float32), 1.9e-5)
    n = T - (T - maxd) % 2
    ref = oracle.idd(np.ascontiguousarray(full[:n]), delays, maxd, 2, np.float32(4.0))
    for r in range(world):
        bs = subbands.rank_beams(B, world, r)
        assert np.array_equal(np.load(tmp_path / f"beams{r}.npy"), full[:, :, bs])
        assert np.array_equal(np.load(tmp_path / f"tdb{r}.npy"), ref[:, :, bs])


def _chain_case(oracle, F=8, A=8, B=12, T=2048, ts=4, seed=33):
    """A small seeded gulp, its weights and the whole band's incoherent
    dedispersion delays (the same on every rank)."""
    from skyweaver_b200 import synthetic
    g = synthetic.rng(seed)
    chbw = 856e6 / 1024
    freqs = 1284e6 + (np.arange(F) - F / 2 + 0.5) * chbw
    ftpa = np.clip(np.rint(g.normal(0, 8, size=(F, T, 2, A, 2))), -127, 127).astype(np.int8)
    w = oracle.weights(synthetic.delay_model(g, B, A), freqs, 0.0, 0.0)
    delays, maxd = oracle.idd_delays(freqs, np.array([0, 20, 40], np.float32), ts / chbw)
    assert 0 < maxd < T // ts
    return ftpa, w, delays, maxd


def _beams(oracle, ftpa, w, ts):
    F, A = ftpa.shape[0], ftpa.shape[3]
    one = np.ones(F, np.float32)
    return oracle.coherent_beam(ftpa, w, ts, one * 1e4, one * 0, np.ones((1, A), np.float32),
                                np.zeros(w.shape[1], np.int32))


def _chain_main(rank, world, port, out_dir):
    import torch
    import torch.distributed as dist
    sys.path.insert(0, REPO)
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    from skyweaver_b200 import subbands
    import swb_oracle as oracle
    oracle.build()
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world)
    try:
        ftpa, w, delays, maxd = _chain_case(oracle)
        F, ts = ftpa.shape[0], 4
        ch = subbands.rank_channels(F, world, rank)
        # each rank holds only its channels' voltages and weights
        mine = np.ascontiguousarray(ftpa[ch])
        w_mine = np.ascontiguousarray(w[ch])

        def beamform(v):
            return torch.from_numpy(_beams(oracle, v, w_mine, ts))

        def dedisperse(tfb):
            x = tfb.numpy()
            n = x.shape[0]
            return oracle.idd(np.ascontiguousarray(x[:n]), delays, maxd, 1, np.float32(3.0))

        chain = subbands.ChannelChain(beamform, dedisperse)
        np.save(os.path.join(out_dir, f"chain{rank}.npy"), chain(mine))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_channel_partitioned_chain_equals_single_process(tmp_path, oracle):
    """The whole chain on two gloo ranks (beamform own channels -> all-to-all
    -> incoherent dedispersion of own beams over the whole band) equals the
    single-process chain (beamform every channel -> dedisperse) sliced by
    beam block."""
    import torch.multiprocessing as mp
    world = 2
    mp.start_processes(_chain_main, args=(world, _free_port(), str(tmp_path)), nprocs=world,
                       join=True, start_method="spawn")
    sys.path.insert(0, REPO)
    from skyweaver_b200 import subbands
    ftpa, w, delays, maxd = _chain_case(oracle)
    full = _beams(oracle, ftpa, w, 4)
    ref = oracle.idd(np.ascontiguousarray(full), delays, maxd, 1, np.float32(3.0))
    B = w.shape[1]
    for r in range(world):
        got = np.load(tmp_path / f"chain{r}.npy")
        assert np.array_equal(got, ref[:, :, subbands.rank_beams(B, world, r)])
