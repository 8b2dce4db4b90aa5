"""Serving with continuous batching (shm_server_create / shm_submit / shm_poll).

CPU: the admission rule of a slot (requests taken in arrival order while the
batch stays within its read and base limits; a request too large for one
batch taken in parts) against a model. GPU: requests submitted from several
threads at once, mapped in mixed batches by two slots, get exactly the
records each gets mapped alone; some batches carry several requests; a
request larger than a batch is mapped in parts; empty requests, unknown
tickets and a destroy with requests still queued behave as documented."""
import ctypes
import threading

import numpy as np
import pytest

import shmap_b200 as sb
from helpers import pack, record_mismatches, xorshift_dna


def _admit(reads, bases, max_reads, max_bases, front_lens=()):
    f = sb.lib().shm_internal_serve_admit
    f.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64,
                  ctypes.c_void_p]
    f.restype = ctypes.c_int64
    r = np.ascontiguousarray(reads, np.int64)
    b = np.ascontiguousarray(bases, np.int64)
    fl = np.ascontiguousarray(list(front_lens) or [0], np.int64)
    part = ctypes.c_int64()
    k = f(r.ctypes.data, b.ctypes.data, len(r), fl.ctypes.data, max_reads, max_bases, ctypes.byref(part))
    return k, part.value


def _admit_model(reads, bases, max_reads, max_bases, front_lens):
    k = tr = tb = 0
    while k < len(reads) and tr + reads[k] <= max_reads and tb + bases[k] <= max_bases:
        tr += reads[k]
        tb += bases[k]
        k += 1
    part = 0
    if k == 0 and reads:
        c = cb = 0
        while c < reads[0] and c < max_reads and cb + front_lens[c] <= max_bases:
            cb += front_lens[c]
            c += 1
        part = max(c, 1)
    return k, part


def test_admission_rule():
    """Whole requests in arrival order while both totals fit; a front request
    that alone does not fit gives the longest run of its first reads that
    does (so no batch exceeds the slot's budget)."""
    rng = np.random.default_rng(3)
    for _ in range(2000):
        n = int(rng.integers(0, 12))
        reads = rng.integers(1, 5000, n)
        mr = int(rng.integers(1, 20000))
        mb = int(rng.integers(60_000, 1 << 28))
        lens = [rng.integers(100, 60_000, int(x)) for x in reads]
        bases = np.array([int(v.sum()) for v in lens], np.int64)
        front = lens[0][: min(int(reads[0]), mr)] if n else []
        got = _admit(reads, bases, mr, mb, front)
        assert got == _admit_model(list(reads), list(bases), mr, mb, list(front))
        if got[1]:
            assert got[1] <= mr and sum(front[: got[1]]) <= mb
    assert _admit([10**6], [10**9], 10, 10**9, [10**3] * 10) == (0, 10)
    assert _admit([], [], 10, 10) == (0, 0)


def _workload():
    ref = xorshift_dna(21, 3_000_000)
    rng = np.random.default_rng(4)
    comp = bytes.maketrans(b"ACGT", b"TGCA")
    reads = []
    for i in range(6000):
        L = int(rng.integers(800, 6000))
        a = int(rng.integers(0, len(ref) - L))
        r = bytearray(ref[a:a + L])
        for j in rng.integers(0, L, L // 100):
            r[j] = b"ACGT"[int(rng.integers(0, 4))]
        r = bytes(r)
        reads.append(r.translate(comp)[::-1] if i % 2 else r)
    return [("chrS", ref)], reads


@pytest.mark.gpu
def test_requests_alone_and_in_the_mix(gpu_ctx):
    refs, reads = _workload()
    g = sb.SketchIndex.from_records(gpu_ctx, refs, 15, 0.1)
    p = sb.Params(k=15, h_frac=0.1, theta=0.4)
    rng = np.random.default_rng(5)
    cuts = np.unique(np.concatenate([[0, len(reads)], rng.integers(1, len(reads), 60)]))
    requests = [pack(reads[a:b]) for a, b in zip(cuts[:-1], cuts[1:])]
    alone = [g.map_reads(p, seq, offs) for seq, offs in requests]
    assert np.mean([(r["status"] == 0).mean() for r in alone]) > 0.9
    with sb.Server(gpu_ctx, g, p, slots=2, max_batch_reads=1500) as srv:
        tickets = [None] * len(requests)

        def submit(part):
            for i in part:
                tickets[i] = srv.submit(*requests[i])

        ths = [threading.Thread(target=submit, args=(range(t, len(requests), 4),)) for t in range(4)]
        for t in ths:
            t.start()
        for t in ths:
            t.join()
        empty = srv.submit(np.zeros(0, np.uint8), np.zeros(1, np.int64))
        mixed = 0
        for i, t in enumerate(tickets):
            got = srv.poll(t, 120_000)
            assert got is not None, i
            rec, st = got
            assert st["status"] == 0 and st["reads"] == len(requests[i][1]) - 1
            assert st["total_ms"] >= st["queued_ms"] >= 0 and st["batch_reads"] >= st["reads"]
            assert st["batch_reads"] <= 1500 or st["batch_requests"] == 1
            mixed += st["batch_requests"] > 1
            assert not record_mismatches(rec, alone[i]), i
        assert mixed > 0
        rec, st = srv.poll(empty, 0)
        assert len(rec) == 0 and st["reads"] == 0
        with pytest.raises(sb.ShmError) as e:
            srv.poll(12345678, 0)
        assert e.value.code == sb.SHM_ERR_INVALID


@pytest.mark.gpu
def test_destroy_maps_what_is_queued(gpu_ctx):
    refs, reads = _workload()
    g = sb.SketchIndex.from_records(gpu_ctx, refs, 15, 0.1)
    p = sb.Params(k=15, h_frac=0.1, theta=0.4)
    seq, offs = pack(reads[:3000])
    want = g.map_reads(p, seq, offs)
    srv = sb.Server(gpu_ctx, g, p, slots=1, max_batch_reads=500)
    outs = []
    for a in range(0, 3000, 300):
        s2, o2 = pack(reads[a:a + 300])
        out = np.zeros(300, sb.RECORD_DTYPE)
        srv.submit(s2, o2, out)
        outs.append(out)
    live = dict(srv._live)  # the arrays stay alive until the slots are done
    srv.close()
    assert not record_mismatches(np.concatenate(outs), want)
    del live


@pytest.mark.gpu
def test_request_larger_than_a_batch_goes_in_parts(gpu_ctx):
    """A request with more reads and bases than one batch may hold is mapped
    in parts (each within the slot's limits) and gets the records it gets
    alone; a single read longer than a batch holds is refused at submit."""
    refs, reads = _workload()
    g = sb.SketchIndex.from_records(gpu_ctx, refs, 15, 0.1)
    p = sb.Params(k=15, h_frac=0.1, theta=0.4)
    seq, offs = pack(reads[:2500])
    want = g.map_reads(p, seq, offs)
    small = pack(reads[2500:2520])
    want_small = g.map_reads(p, *small)
    with sb.Server(gpu_ctx, g, p, slots=2, max_batch_reads=400, max_batch_bases=1_000_000) as srv:
        big = srv.submit(seq, offs)
        t2 = srv.submit(*small)
        rec, st = srv.poll(big, 120_000)
        assert not record_mismatches(rec, want)
        assert st["batch_reads"] <= 400 and st["reads"] == 2500
        rec2, _ = srv.poll(t2, 120_000)
        assert not record_mismatches(rec2, want_small)
        long_read = pack([xorshift_dna(8, 1_000_001)])
        with pytest.raises(sb.ShmError) as e:
            srv.submit(*long_read)
        assert e.value.code == sb.SHM_ERR_INVALID
