"""sw_statistics_noalloc: the statistics stage for callers that cannot
allocate device memory (for example a real-time ingest loop that must not
take the implicit device synchronisation of cudaMalloc, or a process whose
device memory belongs to another component).  It keeps its workspace in a
file-scope device array of the library instead of a caller buffer.

Checked through the C ABI against sw_statistics (the entry point with a
caller workspace) on the same inputs, twice in a row with different data, so
that the second call shows the shared array is cleared between calls.  This
file is collected last (name order) and also passes on its own in a fresh
process.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _stats_pair(torch, L, fp, F, P, A, T, stride, off):
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    ref = torch.empty((F, P, A, 4), dtype=torch.float32, device="cuda")
    got = torch.full((F, P, A, 4), float("nan"), dtype=torch.float32, device="cuda")
    scratch = torch.empty(L.sw_statistics_scratch_bytes(F, P, A), dtype=torch.uint8,
                          device="cuda")
    assert L.sw_statistics(ctypes.c_void_p(fp.data_ptr()), stride, off, F, P, A, T,
                           ctypes.c_void_p(scratch.data_ptr()),
                           ctypes.c_void_p(ref.data_ptr()), stream) == 0, L.sw_last_error()
    assert L.sw_statistics_noalloc(ctypes.c_void_p(fp.data_ptr()), stride, off, F, P, A, T,
                                   ctypes.c_void_p(got.data_ptr()), stream) == 0, \
        L.sw_last_error()
    torch.cuda.synchronize()
    return ref.cpu().numpy(), got.cpu().numpy()


def test_statistics_noalloc_matches_workspace_entry_point(cuda):
    torch = cuda
    from skyweaver_b200._lib import lib
    L = lib()
    F, P, A, T, off = 8, 2, 64, 4096, 32
    stride = off + T
    for seed, sigma in ((1, 8.0), (2, 30.0)):   # two calls in a row, different data
        g = torch.Generator(device="cuda").manual_seed(seed)
        fp = (torch.randn((F, P, A, 2, stride), generator=g, device="cuda") * sigma)
        fp = fp.round_().clamp_(-127, 127).to(torch.int8)
        ref, got = _stats_pair(torch, L, fp, F, P, A, T, stride, off)
        # same kernels and the same exact integer sums: bit-identical results
        assert np.isfinite(got).all()
        assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))


def test_statistics_noalloc_rejects_oversized_shapes(cuda):
    torch = cuda
    from skyweaver_b200._lib import lib
    L = lib()
    stats = torch.empty(4, dtype=torch.float32, device="cuda")
    fp = torch.zeros(16, dtype=torch.int8, device="cuda")
    # 256 channels x 2 pols x 64 antennas = 32768 series > the 16384 built in
    rc = L.sw_statistics_noalloc(ctypes.c_void_p(fp.data_ptr()), 16, 0, 256, 2, 64, 16,
                                 ctypes.c_void_p(stats.data_ptr()), None)
    assert rc == 1
    assert b"exceed" in L.sw_last_error()
