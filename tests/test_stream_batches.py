"""The device batches of a host call's packing stream (cut_stream_batches in
csrc/shm_map.cu): every read in exactly one batch, in order; no batch above
the read or base limits (a single read may exceed the base limit alone); the
first about first_bases, then sizes growing, then halving, the last taking
what is left."""
import ctypes

import numpy as np
import pytest

import shmap_b200 as sb


def _cut(lens, first, last, max_bases, max_reads):
    f = sb.lib().shm_internal_cut_stream
    f.argtypes = [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64, ctypes.c_int32,
                  ctypes.c_void_p, ctypes.c_int32]
    f.restype = ctypes.c_int
    offs = np.zeros(len(lens) + 1, np.int64)
    offs[1:] = np.cumsum(lens)
    out = np.zeros(2 * (len(lens) + 1), np.int32)
    nb = f(offs.ctypes.data, len(lens), first, last, max_bases, max_reads, out.ctypes.data, len(lens) + 1)
    assert nb >= 0
    return offs, [(int(out[2 * i]), int(out[2 * i + 1])) for i in range(nb)]


@pytest.mark.parametrize("seed", range(6))
def test_stream_batches_cover_every_read_within_the_limits(seed):
    rng = np.random.default_rng(seed)
    n = int(rng.integers(1, 20000))
    lens = rng.lognormal(np.log(20000), 0.4, n).astype(np.int64) + 1
    first, last = 1 << int(rng.integers(20, 25)), 1 << int(rng.integers(22, 27))
    max_bases, max_reads = 1 << int(rng.integers(26, 30)), int(rng.integers(100, 5000))
    offs, b = _cut(lens, first, last, max_bases, max_reads)
    assert b[0][0] == 0 and b[-1][1] == n
    assert all(b[i][1] == b[i + 1][0] and b[i][0] < b[i][1] for i in range(len(b) - 1))
    for i, j in b:
        assert j - i <= max_reads
        assert offs[j] - offs[i] <= max_bases or j - i == 1
    # the first batch is the first target's size (or one read), the last not below last_bases unless
    # the reads cap or the whole call makes it so
    i, j = b[0]
    assert offs[j] - offs[i] <= max(first, max(last, lens[0])) or j - i == 1



def test_stream_batches_grow_and_shrink():
    lens = np.full(100_000, 10_000, np.int64)  # 1 GB of 10 kb reads
    offs, b = _cut(lens, 1 << 24, 1 << 26, 1 << 30, 1 << 20)
    sizes = [int(offs[j] - offs[i]) for i, j in b]
    k = int(np.argmax(sizes))
    assert sizes[0] <= 1 << 24
    assert all(sizes[t + 1] >= sizes[t] for t in range(k))  # growing up to the largest
    assert all(sizes[t + 1] <= sizes[t] for t in range(k, len(sizes) - 2))  # then halving
    # the last takes what is left: about the one before, plus a rest below last_bases
    assert sizes[-1] <= sizes[-2] + (1 << 26) + 10_000
    assert sizes[-1] >= (1 << 26) // 2
    assert sum(sizes) == int(offs[-1])
