"""Host packing of reads (shmap-rs_b200/host/pack.cpp): 2-bit codes and the
non-ACGT mask the host-buffer path uploads, checked against a numpy model
of the definition on every byte value, both cases and ragged lengths; the
AVX-512 form (where the CPU has it), the AVX2 form (SHMAP_PACK_AVX2) and the
scalar form must agree bit for bit."""
import ctypes

import numpy as np
import pytest

import shmap_b200 as sb


def _lib():
    lib = sb.lib()
    f = lib.shm_internal_pack_reads
    f.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
    f.restype = ctypes.c_int
    return f


def _model(seq: np.ndarray):
    """codes[p >> 4] bits 2(p & 15) = (b >> 1) & 3; mask bit p set unless b is ACGT/acgt."""
    nb = len(seq)
    groups = nb // 32 + 3
    code = ((seq >> 1) & 3).astype(np.uint64)
    ok = np.isin(seq, np.frombuffer(b"ACGTacgt", np.uint8))
    codes = np.zeros(2 * groups, np.uint64)
    mask = np.zeros(groups, np.uint64)
    p = np.arange(nb, dtype=np.int64)
    np.bitwise_or.at(codes, p >> 4, code << (2 * (p & 15)).astype(np.uint64))
    np.bitwise_or.at(mask, p >> 5, (~ok).astype(np.uint64) << (p & 31).astype(np.uint64))
    # positions past the end are masked (codes 0)
    pos = np.arange(nb, 32 * groups, dtype=np.int64)
    np.bitwise_or.at(mask, pos >> 5, np.uint64(1) << (pos & 31).astype(np.uint64))
    return codes.astype(np.uint32), mask.astype(np.uint32)


def _pack(seq: np.ndarray, scalar: int):
    f = _lib()
    groups = len(seq) // 32 + 3
    codes = np.full(2 * groups, 0xDEADBEEF, np.uint32)
    mask = np.full(groups, 0xDEADBEEF, np.uint32)
    buf = np.ascontiguousarray(seq)
    assert f(buf.ctypes.data if len(buf) else None, len(buf), codes.ctypes.data, mask.ctypes.data, scalar) == 0
    return codes, mask


@pytest.mark.parametrize("avx2", [False, True])
@pytest.mark.parametrize("nb", [0, 1, 31, 32, 33, 64, 95, 1000, 1 << 16, (1 << 20) + 7, (1 << 21) + 40])
def test_pack_matches_model(nb, avx2, monkeypatch):
    if avx2:
        monkeypatch.setenv("SHMAP_PACK_AVX2", "1")
    rng = np.random.default_rng(nb + 1)
    # mostly bases of both cases, with every other byte value sprinkled in
    seq = rng.choice(np.frombuffer(b"ACGTacgt", np.uint8), nb)
    if nb:
        k = max(1, nb // 50)
        seq[rng.integers(0, nb, k)] = rng.integers(0, 256, k).astype(np.uint8)
    want_c, want_m = _model(seq)
    for scalar in (0, 1):
        c, m = _pack(seq, scalar)
        assert np.array_equal(m, want_m), scalar
        assert np.array_equal(c, want_c), scalar


@pytest.mark.parametrize("avx2", [False, True])
def test_pack_every_byte_value(avx2, monkeypatch):
    if avx2:
        monkeypatch.setenv("SHMAP_PACK_AVX2", "1")
    seq = np.tile(np.arange(256, dtype=np.uint8), 40)  # 10240 bytes, every value at every offset mod 32
    want_c, want_m = _model(seq)
    for scalar in (0, 1):
        c, m = _pack(seq, scalar)
        assert np.array_equal(m, want_m) and np.array_equal(c, want_c)
    ok = np.isin(np.arange(256), np.frombuffer(b"ACGTacgt", np.uint8))
    assert ok.sum() == 8


@pytest.mark.gpu
@pytest.mark.parametrize("nb", [0, 1, 31, 32, 33, 100, 4096, 100_003])
def test_device_packing_equals_the_model(nb):
    """Reads packed on the device (shm_pack.cu, used for reads that are in
    device memory) give the host packing's words: every byte value, both
    cases, ragged lengths, a start that is not 16-byte aligned."""
    f = sb.lib().shm_internal_pack_reads_device
    f.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p]
    f.restype = ctypes.c_int
    rng = np.random.default_rng(nb)
    seq = rng.choice(np.frombuffer(b"ACGTacgtACGTACGTN", np.uint8), nb)
    seq[: min(nb, 256)] = np.arange(min(nb, 256), dtype=np.uint8)  # every byte value
    groups = nb // 32 + 3
    codes = np.zeros(2 * groups, np.uint32)
    mask = np.zeros(groups, np.uint32)
    assert f(0, seq.ctypes.data, nb, codes.ctypes.data, mask.ctypes.data) == 0
    want_c, want_m = _model(seq)
    assert np.array_equal(codes, want_c) and np.array_equal(mask, want_m)


@pytest.mark.parametrize("nb", [0, 1, 31, 32, 33, 64, 95, 1000, 1 << 16, (1 << 20) + 7, (1 << 21) + 40])
@pytest.mark.parametrize("task_groups,chunk_tasks", [(2, 1), (2, 7), (64, 3), (8192, 128)])
def test_streamed_packing_equals_the_model(nb, task_groups, chunk_tasks):
    """The streamed packing of the host-buffer path: tasks packed in the
    background, chunks taken in order as their tasks finish, each chunk's
    nonzero mask words (the last chunk's with the tail groups) scattered into
    a zeroed mask: the same codes and mask as the definition."""
    f = sb.lib().shm_internal_pack_stream
    f.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int]
    f.restype = ctypes.c_int
    rng = np.random.default_rng(nb + 7 * task_groups + chunk_tasks)
    seq = rng.choice(np.frombuffer(b"ACGTACGTACGTacgtNnRY\x00\xff", np.uint8), nb).astype(np.uint8)
    groups = nb // 32 + 3
    codes = np.full(2 * groups, 0xDEADBEEF, np.uint32)
    mask = np.full(groups, 0xDEADBEEF, np.uint32)
    buf = np.ascontiguousarray(seq)
    chunks = f(buf.ctypes.data if nb else None, nb, codes.ctypes.data, mask.ctypes.data, task_groups, chunk_tasks)
    assert chunks >= 1
    wc, wm = _model(seq)
    assert np.array_equal(codes, wc)
    assert np.array_equal(mask, wm)
