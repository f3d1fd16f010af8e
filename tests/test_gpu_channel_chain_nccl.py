"""The channel-partitioned chain (subbands.ChannelChain) on the GPU with the
NCCL backend.  Only one GPU is available per run, so the process group has
one rank: its all-to-all still goes through NCCL on device tensors (the
exchange the N > 1 bench line uses), and its result must equal the
single-process computation.  No two ranks share the GPU, so nothing waits on
another rank's kernels.  The multi-rank decomposition itself is tested on CPU
with gloo ranks (tests/test_multirank.py).  Runs in a child process so that
the process group never touches the other tests' CUDA state."""
import os
import socket
import subprocess
import sys

import pytest

from conftest import REPO

pytestmark = pytest.mark.gpu

CHILD = r"""
import datetime, os, sys
import numpy as np
import torch
import torch.distributed as dist
sys.path.insert(0, os.environ["SW_REPO"])
from skyweaver_b200 import stages, subbands, synthetic
torch.cuda.set_device(0)
dist.init_process_group("nccl", init_method="tcp://127.0.0.1:" + os.environ["SW_PORT"],
                        rank=0, world_size=1, timeout=datetime.timedelta(seconds=60),
                        device_id=torch.device("cuda", 0))
try:
    g = synthetic.rng(71)
    T, F, B = 3000, 32, 256
    tfb = torch.from_numpy(g.integers(-40, 40, size=(T, F, B), dtype=np.int8)).cuda()
    freqs = 1088e6 - 0.53125e6 * (F - np.arange(F) - 0.5)
    trials = np.linspace(0.0, 20.0, 12).astype(np.float32)
    k, tsamp = 4.148806423e15, 8 / 0.53125e6
    delays = np.array([[int(k * (1 / freqs[0] ** 2 - 1 / f ** 2) * d / tsamp + 0.5)
                        for f in freqs] for d in trials], np.int32)
    maxd = int(delays.max())
    d_delays = torch.from_numpy(delays).cuda()
    sf = float(np.float32(np.sqrt(F)))
    chain = subbands.ChannelChain(
        beamform=lambda x: x,
        dedisperse=lambda blk: stages.incoherent_dedisperse(blk, d_delays, maxd, 1, sf))
    got = chain(tfb)
    ref = stages.incoherent_dedisperse(tfb, d_delays, maxd, 1, sf)
    torch.cuda.synchronize()
    assert got.shape == ref.shape, (got.shape, ref.shape)
    assert torch.equal(got, ref)
    print("nccl chain ok", tuple(got.shape), "max delay", maxd)
finally:
    dist.destroy_process_group()
"""


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_channel_chain_nccl_one_rank(cuda):
    env = dict(os.environ, SW_REPO=REPO, SW_PORT=str(_free_port()), NCCL_NVLS_ENABLE="0",
               MASTER_ADDR="127.0.0.1")
    r = subprocess.run([sys.executable, "-c", CHILD], env=env, capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-4000:]
    assert "nccl chain ok" in r.stdout
