"""shm_sketch_device_noalloc: the sketch entry point for callers that must not
allocate device memory (for example a program whose device memory is fully
reserved by its own pool allocator, or a latency-critical loop that cannot pay
for cudaMalloc/cudaFree, which may synchronize the device). The test gives it
device buffers it allocated itself, calls it twice in a row on different
sequences, and checks each result against the allocating entry point
shm_sketch (the k-mer streams are integers: they must be identical). It also
checks that a warm call leaves the device's free memory unchanged, the
capacity answer, an input of exactly the window limit and k above 32. This file
is collected last so that a run stopping at its first failure has run every
other test already; it also passes on its own in a fresh process."""
import ctypes

import numpy as np
import pytest

import shmap_b200 as sb
from helpers import lcg_dna, xorshift_dna

pytestmark = pytest.mark.gpu

MAX_WINDOWS = 4_194_304


def _buffers(torch, seq: bytes, k: int):
    n = len(seq)
    d_seq = torch.zeros(n + 32, dtype=torch.uint8, device="cuda")
    if n:
        d_seq[:n].copy_(torch.frombuffer(bytearray(seq), dtype=torch.uint8))
    cap = max(1, n - k + 1)
    d_h = torch.zeros(cap, dtype=torch.int64, device="cuda")
    d_rs = torch.zeros(cap, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    return d_seq, d_h, d_rs, cap


def _call(d_seq, n, k, h_frac, offset, d_h, d_rs, cap):
    n_out = ctypes.c_int64()
    rc = sb.lib().shm_sketch_device_noalloc(d_seq.data_ptr(), n, k, h_frac, offset, d_h.data_ptr(),
                                            d_rs.data_ptr(), cap, ctypes.byref(n_out), None)
    return rc, n_out.value


def _noalloc(torch, seq: bytes, k: int, h_frac: float, offset: int = 0):
    d_seq, d_h, d_rs, cap = _buffers(torch, seq, k)
    rc, m = _call(d_seq, len(seq), k, h_frac, offset, d_h, d_rs, cap)
    assert rc == sb.SHM_OK, sb.lib().shm_last_error()
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


def test_noalloc_leaves_free_device_memory_unchanged():
    """The point of the entry point: once a device has run it (the first call
    looks up the scratch array's address, and the library's kernels load),
    a call takes no device memory: the free memory the driver reports is the
    same before and after it."""
    import torch

    seq = lcg_dna(5, 200_000)
    k = 21
    d_seq, d_h, d_rs, cap = _buffers(torch, seq, k)
    rc, _ = _call(d_seq, len(seq), k, 0.05, 0, d_h, d_rs, cap)  # warm: first call on this device
    assert rc == sb.SHM_OK
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    rc, m = _call(d_seq, len(seq), k, 0.05, 0, d_h, d_rs, cap)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert rc == sb.SHM_OK and m > 0
    assert free1 == free0


def test_noalloc_capacity_exact_limit_and_long_k():
    """A cap below the count answers SHM_ERR_CAPACITY with the true count in
    *n_out; an input of exactly the window limit is accepted; k above 32
    (two-word rotations) matches the allocating entry point."""
    import torch

    ctx = sb.Context(0)
    seq = xorshift_dna(17, 60_000)
    want = ctx.sketch(seq, 25, 0.1)
    d_seq, d_h, d_rs, cap = _buffers(torch, seq, 25)
    rc, m = _call(d_seq, len(seq), 25, 0.1, 0, d_h, d_rs, len(want[0]) - 1)
    assert rc == sb.SHM_ERR_CAPACITY and m == len(want[0])
    rc, m = _call(d_seq, len(seq), 25, 0.1, 0, d_h, d_rs, len(want[0]))
    assert rc == sb.SHM_OK and m == len(want[0])
    k = 25
    big = lcg_dna(3, MAX_WINDOWS + k - 1)  # exactly MAX_WINDOWS windows
    got = _noalloc(torch, big, k, 0.01)
    ref = ctx.sketch(big, k, 0.01)
    assert len(ref[0]) > 0 and all(np.array_equal(a, b) for a, b in zip(got, ref))
    for kk in (33, 63):
        s2 = lcg_dna(40 + kk, 30_000)
        got = _noalloc(torch, s2, kk, 0.25, 9)
        ref = ctx.sketch(s2, kk, 0.25, 9)
        assert len(ref[0]) > 0 and all(np.array_equal(a, b) for a, b in zip(got, ref))
    ctx.close()
