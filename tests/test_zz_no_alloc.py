"""shm_sketch_device_noalloc: the sketch entry point for callers that must not
allocate device memory (for example a program whose device memory is fully
reserved by its own pool allocator, or a latency-critical loop that cannot pay
for cudaMalloc/cudaFree, which may synchronize the device). The test gives it
device buffers it allocated itself, calls it twice in a row on different
sequences, and checks each result against the allocating entry point
shm_sketch (the k-mer streams are integers: they must be identical). This file
is collected last so that a run stopping at its first failure has run every
other test already; it also passes on its own in a fresh process."""
import ctypes

import numpy as np
import pytest

import shmap_b200 as sb
from helpers import lcg_dna, xorshift_dna

pytestmark = pytest.mark.gpu

MAX_WINDOWS = 4_194_304


def _noalloc(torch, seq: bytes, k: int, h_frac: float, offset: int = 0):
    n = len(seq)
    d_seq = torch.zeros(n + 32, dtype=torch.uint8, device="cuda")
    if n:
        d_seq[:n].copy_(torch.frombuffer(bytearray(seq), dtype=torch.uint8))
    cap = max(1, n - k + 1)
    d_h = torch.zeros(cap, dtype=torch.int64, device="cuda")
    d_rs = torch.zeros(cap, dtype=torch.int32, device="cuda")
    n_out = ctypes.c_int64()
    torch.cuda.synchronize()
    rc = sb.lib().shm_sketch_device_noalloc(d_seq.data_ptr(), n, k, h_frac, offset, d_h.data_ptr(),
                                            d_rs.data_ptr(), cap, ctypes.byref(n_out), None)
    assert rc == sb.SHM_OK, sb.lib().shm_last_error()
    m = n_out.value
    h = d_h[:m].cpu().numpy().view(np.uint64)
    rs = d_rs[:m].cpu().numpy().view(np.uint32)
    return (rs >> 1).astype(np.int32), h, (rs & 1).astype(np.uint8)


def test_noalloc_matches_the_allocating_entry_twice_in_a_row():
    import torch

    ctx = sb.Context(0)
    cases = [(lcg_dna(77, 300_000), 25, 0.01, 0), (xorshift_dna(91, 50_000) + b"NNNNNNNNNNacgt" * 40, 15, 0.5, 1234)]
    for seq, k, r, off in cases:  # two calls in a row: the shared scratch keeps the first call's contents
        got = _noalloc(torch, seq, k, r, off)
        want = ctx.sketch(seq, k, r, off)
        assert len(want[0]) > 0
        for a, b in zip(got, want):
            assert np.array_equal(a, b)
    ctx.close()


def test_noalloc_rejects_inputs_beyond_its_limit():
    import torch

    k = 25
    n = MAX_WINDOWS + k  # one window too many
    d_seq = torch.zeros(n + 32, dtype=torch.uint8, device="cuda")
    n_out = ctypes.c_int64()
    rc = sb.lib().shm_sketch_device_noalloc(d_seq.data_ptr(), n, k, 0.01, 0, 0, 0, 0, ctypes.byref(n_out), None)
    assert rc == -1
    assert "too long" in sb.lib().shm_last_error().decode()
