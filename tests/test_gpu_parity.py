"""Parity of the device path with the CPU oracle (bit-exact: integers, hashes,
indices and the f64 scores alike), through the C ABI. Run on a B200 with
`pytest -m gpu`."""
import os

import numpy as np
import pytest

import oracle as O
import shmap_b200 as sb
from helpers import (floor_reads, floor_reference, lcg_dna, pack, record_mismatches, strip_t, thread_parity_workload,
                     xorshift_dna)
from shmap_b200 import fasta, synth

pytestmark = pytest.mark.gpu


def _both_indexes(ctx, records, k, r, max_matches=None):
    g = sb.SketchIndex.from_records(ctx, records, k, r, max_matches)
    o = O.Index.from_records(records, k, r, max_matches, threads=4)
    return g, o


def _compare_mapping(g, o, reads, **pkw):
    names = [n for n, _ in reads]
    seq, offs = pack([s for _, s in reads])
    gp = sb.Params(**pkw)
    op = O.params(**pkw)
    grec = g.map_reads(gp, seq, offs)
    orec = o.map_reads(op, seq, offs, threads=8)
    mm = record_mismatches(grec, orec)
    assert not mm, f"record mismatches (read, field, gpu, oracle): {mm}"
    gpaf = strip_t(g.format_paf(gp, grec, names))
    opaf = strip_t(o.paf(op, seq, offs, names, threads=8))
    assert gpaf == opaf
    return grec, gpaf


# ---------------------------------------------------------------- sketch
@pytest.mark.parametrize("k", [1, 5, 8, 15, 25, 31, 32, 33, 64, 65, 100])
@pytest.mark.parametrize("r", [1.0, 0.5, 0.01])
def test_sketch_parity(gpu_ctx, k, r):
    seq = bytearray(lcg_dna(1000 + k, 5000))
    for i in range(0, len(seq), 331):
        seq[i] = ord("n")
    for i in range(100, 160):
        seq[i] = ord("N")
    for i in range(2000, 2400):
        seq[i] = seq[i] | 0x20  # lower case
    seq[3000:3004] = b"RYK-"
    seq = bytes(seq)
    for off in (0, 7, 123456):
        a = gpu_ctx.sketch(seq, k, r, off)
        b = O.sketch(seq, k, r, off)
        for x, y in zip(a, b):
            assert np.array_equal(x, y), (k, r, off)


def test_sketch_edge_lengths(gpu_ctx):
    for n in (0, 1, 7, 8, 9, 63, 64, 65, 127, 128, 129, 1000):
        s = xorshift_dna(n + 3, n)
        a = gpu_ctx.sketch(s, 8, 1.0)
        b = O.sketch(s, 8, 1.0)
        assert all(np.array_equal(x, y) for x, y in zip(a, b)), n


# ---------------------------------------------------------------- index
def test_index_known_answers(gpu_ctx):
    """src/index.rs:715-769."""
    for fa, counts, hits, kmers in ((">ref\nACCAGTACCA\n", [2, 1, 1, 1, 1, 1, 2], 7, 6),
                                    (">segm1\nACCAGTACCA\n>segm2\nGGACCA\n", [3, 1, 1, 1, 1, 1, 3], 10, 8)):
        recs = [(b.split("\n", 1)[0], b.split("\n", 1)[1].replace("\n", "").encode()) for b in fa.strip().split(">")[1:]]
        g = sb.SketchIndex.from_records(gpu_ctx, recs, 4, 1.0)
        _, h, _ = gpu_ctx.sketch(b"ACCAGTACCA", 4, 1.0)
        assert list(g.count(h)) == counts
        st = g.stats()
        assert st["indexed_hits"] == hits and st["indexed_kmers"] == kmers


@pytest.mark.parametrize("mm", [None, 1, 3])
def test_index_parity_with_max_matches(gpu_ctx, mm):
    """src/index.rs:264-376 incl. the -M cap, the erase and the statistics."""
    rep = b"ACGTACGTACGTACGTACGT"
    recs = [(f"segm{i}", rep + b"TTTTGGGGCCCCAAAA" + str(i).encode()) for i in range(10)]
    recs += [("rand", xorshift_dna(5, 3000)), ("empty", b""), ("short", b"ACG"), ("rand2", xorshift_dna(6, 2000))]
    for k, r in ((6, 1.0), (4, 1.0), (11, 0.5)):
        g, o = _both_indexes(gpu_ctx, recs, k, r, mm)
        assert g.stats() == o.stats()
        for i in range(len(recs)):
            gr, gh, gs, nm, ln = g.segment(i)
            orr, oh, os_ = o.segment(i)
            assert np.array_equal(gr, orr) and np.array_equal(gh, oh) and np.array_equal(gs, os_)
            assert nm == recs[i][0] and ln == len(recs[i][1])
        hs = np.unique(np.concatenate([o.segment(i)[1] for i in range(len(recs))] + [np.arange(50, dtype=np.uint64)]))
        assert np.array_equal(g.count(hs), o.count(hs))
        for h in hs[:: max(1, len(hs) // 200)]:
            for x, y in zip(g.hits(int(h)), o.hits(int(h))):
                assert np.array_equal(x, y)


def test_index_parity_synthetic_genome(gpu_ctx):
    gen = synth.Genome(synth.scaled(synth.REFS["human31"], 0.004))
    recs = gen.records()
    g, o = _both_indexes(gpu_ctx, recs, 25, 0.01)
    assert g.stats() == o.stats()
    allh = np.concatenate([o.segment(i)[1] for i in range(len(recs))])
    assert np.array_equal(g.count(allh), o.count(allh))
    rng = np.random.default_rng(0)
    for h in rng.choice(allh, 300, replace=False):
        for x, y in zip(g.hits(int(h)), o.hits(int(h))):
            assert np.array_equal(x, y)


# ---------------------------------------------------------------- mapping
def test_golden_paf(gpu_ctx, golden_dir):
    """tests/golden_paf.rs:25-53 on the device path."""
    refs = fasta.read_fastx(os.path.join(golden_dir, "tiny_ref.fa"))
    reads = fasta.read_fastx(os.path.join(golden_dir, "tiny_reads.fa"))
    g = sb.SketchIndex.from_records(gpu_ctx, refs, 8, 1.0)
    p = sb.Params(k=8, h_frac=1.0, theta=0.1)
    seq, offs = pack([s for _, s in reads])
    rec = g.map_reads(p, seq, offs)
    paf = g.format_paf(p, rec, [n for n, _ in reads])
    want = open(os.path.join(golden_dir, "tiny.golden.paf")).read().rstrip("\n")
    assert strip_t(paf) == strip_t(want)


@pytest.mark.parametrize("metric", ["bucket_LCS", "bucket_SH"])
def test_golden_inputs_bucket_metrics(gpu_ctx, golden_dir, metric):
    """The golden fixture's inputs under the bucket metrics (scoring.rs:311-344):
    records and PAF as the oracle's."""
    refs = fasta.read_fastx(os.path.join(golden_dir, "tiny_ref.fa"))
    reads = fasta.read_fastx(os.path.join(golden_dir, "tiny_reads.fa"))
    g, o = _both_indexes(gpu_ctx, refs, 8, 1.0)
    rec, paf = _compare_mapping(g, o, reads, k=8, h_frac=1.0, theta=0.1, metric=metric)
    assert len(paf.splitlines()) == 2


def test_lcs_repeats(gpu_ctx):
    """bucket_LCS where seeds repeat: tandem copies of a 60-mer in read and
    reference give hashes with many read positions each (long pmatches),
    reads of both strands, sketches below and above 512 k-mers."""
    unit = xorshift_dna(11, 60)
    rng = np.random.default_rng(5)
    ref = xorshift_dna(12, 30000) + unit * 150 + xorshift_dna(13, 30000)
    comp = bytes.maketrans(b"ACGT", b"TGCA")
    reads = []
    for i, (a, L) in enumerate([(29000, 4000), (30500, 6000), (25000, 14000), (100, 1500), (36000, 30000)]):
        s = ref[a:a + L]
        reads.append((f"r{i}", s if i % 2 == 0 else s.translate(comp)[::-1]))
    reads.append(("tandem", unit * 40))
    reads.append(("swapped", ref[14000:17000] + ref[9000:12000]))  # collinear halves in the wrong order
    for i in range(len(reads)):  # 3% substitutions
        r = bytearray(reads[i][1])
        for j in rng.integers(0, len(r), len(r) * 3 // 100):
            r[j] = b"ACGT"[int(rng.integers(0, 4))]
        reads[i] = (reads[i][0], bytes(r))
    g, o = _both_indexes(gpu_ctx, [("chrA", ref)], 12, 0.25)
    for theta in (0.2, 0.5):
        rec, _ = _compare_mapping(g, o, reads, k=12, h_frac=0.25, theta=theta, metric="bucket_LCS")
    ok = rec["status"] == 0
    assert ok.sum() >= 4 and (rec["score"][ok] < 1.0).all()
    assert rec["sketch_size"].max() > 512 and rec["sketch_size"].min() < 512


def test_thread_parity_workload(gpu_ctx):
    refs, reads = thread_parity_workload()
    g, o = _both_indexes(gpu_ctx, refs, 12, 0.5)
    rec, paf = _compare_mapping(g, o, reads, k=12, h_frac=0.5, theta=0.2)
    assert len(paf.splitlines()) >= 50


def test_sketch_floor(gpu_ctx):
    """tests/short_read_sketch_floor.rs: K..K+3 unmapped, K+4.. mapped."""
    ref = floor_reference()
    g, o = _both_indexes(gpu_ctx, [("ref", ref)], 8, 1.0)
    rec, _ = _compare_mapping(g, o, floor_reads(ref, [8, 9, 10, 11]), k=8, h_frac=1.0, theta=0.4)
    assert (rec["status"] == 2).all()
    rec, paf = _compare_mapping(g, o, floor_reads(ref, [12, 20, 48]), k=8, h_frac=1.0, theta=0.4)
    assert (rec["status"] == 0).all() and len(paf.splitlines()) == 3
    rec, paf = _compare_mapping(g, o, floor_reads(ref, [28, 8, 28, 9, 28]), k=8, h_frac=1.0, theta=0.4)
    assert len(paf.splitlines()) == 3


@pytest.fixture(scope="module")
def uniform(gpu_ctx):
    gen = synth.Genome(synth.REFS["uniform5m"])
    reads = gen.reads(synth.READS["fixed10k"])
    g, o = _both_indexes(gpu_ctx, gen.records(), 25, 0.01)
    return gen, reads, g, o


@pytest.mark.parametrize("pkw", [
    dict(theta=0.4),
    dict(theta=0.4, min_diff=0.075, max_overlap=0.3),
    dict(theta=0.4, metric="Jaccard"),
    dict(theta=0.4, metric="bucket_SH"),
    dict(theta=0.4, metric="bucket_LCS"),
    dict(theta=0.9),
    dict(theta=0.0),
    dict(theta=0.4, min_diff=1.5),
])
def test_uniform_workload(uniform, pkw):
    """The 5 Mbp / 2,000 x 10 kb workload at k=25, r=0.01."""
    gen, (names, seq, offs), g, o = uniform
    reads = [(names[i], seq[offs[i]:offs[i + 1]].tobytes()) for i in range(len(names))]
    rec, paf = _compare_mapping(g, o, reads, k=25, h_frac=0.01, **pkw)
    if pkw.get("theta") == 0.4 and "metric" not in pkw:
        assert (rec["status"] == 0).mean() > 0.95


@pytest.mark.parametrize("flags", [dict(no_bucket_pruning=True), dict(one_sweep=True), dict(abs_pos=True),
                                   dict(no_bucket_pruning=True, one_sweep=True, abs_pos=True)])
def test_const_generic_variants(gpu_ctx, uniform, flags):
    """The (NBP, OS, AP) variants of src/mapper.rs:25-40."""
    gen, (names, seq, offs), g, o = uniform
    reads = [(names[i], seq[offs[i]:offs[i + 1]].tobytes()) for i in range(0, 300)]
    _compare_mapping(g, o, reads, k=25, h_frac=0.01, theta=0.4, **flags)
    refs, tr = thread_parity_workload()
    g2, o2 = _both_indexes(gpu_ctx, refs, 12, 0.5)
    _compare_mapping(g2, o2, tr, k=12, h_frac=0.5, theta=0.2, **flags)
    _compare_mapping(g2, o2, tr, k=12, h_frac=0.5, theta=0.2, metric="bucket_SH", **flags)
    _compare_mapping(g2, o2, tr, k=12, h_frac=0.5, theta=0.2, metric="bucket_LCS", **flags)


@pytest.fixture(scope="module")
def human_small(gpu_ctx):
    gen = synth.Genome(synth.scaled(synth.REFS["human31"], 0.01))
    return gen


@pytest.mark.parametrize("preset,r,metric,theta", [("hifi", 0.01, "Containment", 0.4),
                                                   ("ont", 0.01, "Containment", 0.4),
                                                   ("ont", 0.01, "Containment", 0.05),
                                                   ("ont", 0.01, "Jaccard", 0.05),
                                                   ("dense", 0.10, "bucket_SH", 0.4),
                                                   ("dense", 0.10, "bucket_LCS", 0.4),
                                                   ("ont", 0.01, "bucket_LCS", 0.05),
                                                   ("dense", 0.10, "Containment", 0.4)])
def test_human_like_workloads(gpu_ctx, human_small, preset, r, metric, theta):
    """Satellite arrays, interspersed repeats, HiFi/ONT/dense read shapes at 1% scale.
    (At 7% errors only ~0.93^25 = 16% of 25-mers survive, so ONT reads clear
    -t 0.4 nowhere, in the oracle as on the device; a low -t maps them.)"""
    gen = human_small
    names, seq, offs = gen.reads(synth.scaled(synth.READS[preset], 300 / synth.READS[preset].n_reads))
    reads = [(names[i], seq[offs[i]:offs[i + 1]].tobytes()) for i in range(len(names))]
    g, o = _both_indexes(gpu_ctx, gen.records(), 25, r)
    rec, paf = _compare_mapping(g, o, reads, k=25, h_frac=r, theta=theta, metric=metric)
    if preset != "ont" or theta < 0.1:
        assert (rec["status"] == 0).mean() > 0.5


def test_max_matches_mapping(gpu_ctx, human_small):
    gen = human_small
    names, seq, offs = gen.reads(synth.scaled(synth.READS["dense"], 0.001))
    reads = [(names[i], seq[offs[i]:offs[i + 1]].tobytes()) for i in range(len(names))]
    g, o = _both_indexes(gpu_ctx, gen.records(), 25, 0.01, max_matches=5)
    _compare_mapping(g, o, reads, k=25, h_frac=0.01, theta=0.4, max_matches=5)


def test_edge_reads(gpu_ctx, uniform):
    """Empty, shorter than k, all-N (every window hashes to 0 and is kept: the
    capacity-overflow retry), lower case, IUPAC bytes."""
    gen, (names, seq, offs), g, o = uniform
    r0 = seq[offs[0]:offs[1]].tobytes()
    r1 = seq[offs[1]:offs[2]].tobytes()
    reads = [("empty", b""), ("short", b"ACGTACGT"), ("allN", b"N" * 5000), ("lower", r0.lower()),
             ("withN", r1[:3000] + b"N" * 500 + r1[3500:]), ("iupac", r0.replace(b"A", b"R", 50)),
             ("ok", r1), ("mixedN", (b"N" * 30 + r0[:200]) * 20)]
    _compare_mapping(g, o, reads, k=25, h_frac=0.01, theta=0.4)


def test_plain_equals_batched(gpu_ctx, uniform):
    """One-read-per-launch and batched forms give identical records (the
    device analogue of the reference's thread-count invariance)."""
    gen, (names, seq, offs), g, o = uniform
    p = sb.Params(k=25, h_frac=0.01, theta=0.4)
    sub = offs[:101]
    a = g.map_reads(p, seq[: sub[-1]], sub)
    b = g.map_reads(p, seq[: sub[-1]], sub, plain=True)
    assert not record_mismatches(a, b)


def test_device_resident_entry(gpu_ctx, uniform):
    import torch

    gen, (names, seq, offs), g, o = uniform
    p = sb.Params(k=25, h_frac=0.01, theta=0.4)
    d_seq = torch.empty(len(seq) + 32, dtype=torch.uint8, device="cuda")
    d_seq[: len(seq)].copy_(torch.from_numpy(np.ascontiguousarray(seq)))
    d_out = torch.empty(len(names) * sb.RECORD_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
    g.map_reads_device(p, d_seq.data_ptr(), offs, d_out.data_ptr())
    torch.cuda.synchronize()
    rec = d_out.cpu().numpy().view(sb.RECORD_DTYPE)
    want = o.map_reads(O.params(k=25, h_frac=0.01, theta=0.4), seq, offs, threads=8)
    assert not record_mismatches(rec, want)


@pytest.mark.parametrize("env", [{"SHMAP_BT_FAST_SLOTS": "16", "SHMAP_BT_SPARE_SLOTS": "0"},
                                 {"SHMAP_BT_FAST_SLOTS": "16"},
                                 {"SHMAP_BT_FAST_SLOTS": "16", "SHMAP_BT_SPARE_SLOTS": "4096"},
                                 {"SHMAP_FAST_JOB_CAP": "7"},
                                 {"SHMAP_BT_FAST_SLOTS": "32", "SHMAP_FAST_JOB_CAP": "40"},
                                 {"SHMAP_BT_FAST_SLOTS": "16", "SHMAP_BT_FAST_READ": "4096",
                                  "SHMAP_BT_SPARE_SLOTS": "0"},
                                 {"SHMAP_BT_FAST_SLOTS": "16", "SHMAP_BT_FAST_READ": "4096"}])
def test_capacity_fallbacks(gpu_ctx, human_small, env, monkeypatch):
    """Batches are queued without waiting for their sizes: bucket tables are
    capped per read and share a pool; a read whose table fills up (or would
    end past the pool) gets a second table from spare slots and contributes
    again, and is mapped again by the host with the full bound when that
    fills up or there is no room; bucket jobs per batch are capped (a batch
    with more is mapped again with exact sizes). Tiny caps, pools and spares
    force every path; the records must not change."""
    for key, val in env.items():
        monkeypatch.setenv(key, val)
    gen = human_small
    names, seq, offs = gen.reads(synth.scaled(synth.READS["hifi"], 200 / synth.READS["hifi"].n_reads))
    reads = [(names[i], seq[offs[i]:offs[i + 1]].tobytes()) for i in range(len(names))]
    g, o = _both_indexes(gpu_ctx, gen.records(), 25, 0.01)
    rec, paf = _compare_mapping(g, o, reads, k=25, h_frac=0.01, theta=0.4)
    assert (rec["status"] == 0).mean() > 0.5
    import torch

    p = sb.Params(k=25, h_frac=0.01, theta=0.4)
    pseq, poffs = pack([s for _, s in reads])
    d_seq = torch.empty(len(pseq) + 32, dtype=torch.uint8, device="cuda")
    d_seq[: len(pseq)].copy_(torch.from_numpy(np.ascontiguousarray(pseq)))
    d_out = torch.empty(len(reads) * sb.RECORD_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
    g.map_reads_device(p, d_seq.data_ptr(), poffs, d_out.data_ptr())
    torch.cuda.synchronize()
    assert not record_mismatches(d_out.cpu().numpy().view(sb.RECORD_DTYPE), rec)


def test_pinned_host_batches(gpu_ctx):
    """Reads in pinned host memory, over five host-buffer batches: the records
    equal those of the same reads in pageable memory and of the
    device-resident call."""
    import torch

    ref = bytearray(xorshift_dna(77, 2_000_000))
    for a in range(1000, len(ref), 50_000):
        ref[a:a + 40] = b"N" * 40
    ref = bytes(ref)
    g = sb.SketchIndex.from_records(gpu_ctx, [("chrU", ref)], 15, 0.1)
    rng = np.random.default_rng(8)
    comp = bytes.maketrans(b"ACGTN", b"TGCAN")
    reads = []
    for i in range(100_000):
        a = int(rng.integers(0, len(ref) - 400))
        r = bytearray(ref[a:a + int(rng.integers(250, 400))])
        if i % 7 == 0:
            r[5:9] = b"acgt"
        r = bytes(r)
        reads.append(r.translate(comp)[::-1] if i % 2 else r)
    seq, offs = pack(reads)
    p = sb.Params(k=15, h_frac=0.1, theta=0.4)
    want = g.map_reads(p, seq, offs)
    assert (want["status"] == 0).mean() > 0.9
    pinned = torch.empty(len(seq) + 32, dtype=torch.uint8).pin_memory()
    pinned[: len(seq)].copy_(torch.from_numpy(np.ascontiguousarray(seq)))
    got = g.map_reads(p, pinned.numpy()[: len(seq)], offs)
    assert not record_mismatches(got, want)
    d_seq = torch.zeros(len(seq) + 32, dtype=torch.uint8, device="cuda:0")
    d_seq[: len(seq)].copy_(pinned[: len(seq)])
    d_out = torch.empty(len(reads) * sb.RECORD_DTYPE.itemsize, dtype=torch.uint8, device="cuda:0")
    g.map_reads_device(p, d_seq.data_ptr(), offs, d_out.data_ptr())
    torch.cuda.synchronize()
    dev = d_out.cpu().numpy().view(sb.RECORD_DTYPE)
    assert not record_mismatches(dev, want)


def test_hifi_five_percent_scale(gpu_ctx):
    """The hifi configuration at 5% scale: a 155 Mbp reference with its
    satellite arrays and interspersed repeats, 7,500 HiFi-like reads (lists of
    hundreds of hits per k-mer, reads up to 60 kb). Every record equals the
    oracle's bit for bit, and the PAF text of shm_map_paf (reads in, text out)
    equals the oracle's byte for byte, t:f: aside (tests/golden_paf.rs:13-53)."""
    gen = synth.Genome(synth.scaled(synth.REFS["human31"], 0.05))
    names, seq, offs = gen.reads(synth.scaled(synth.READS["hifi"], 0.05))
    assert len(names) == 7500
    g = sb.SketchIndex(gpu_ctx, gen.names, gen.seq, gen.seg_off, 25, 0.01)
    o = O.Index(gen.names, gen.seq, gen.seg_off, 25, 0.01, threads=os.cpu_count() or 4)
    assert g.stats() == o.stats()
    text, rec = g.map_paf(sb.Params(k=25, h_frac=0.01, theta=0.4), seq, offs, names)
    orec, otext, _ = o.map_paf(O.params(k=25, h_frac=0.01, theta=0.4), seq, offs, names, os.cpu_count() or 4)
    mm = record_mismatches(rec, orec)
    assert not mm, f"record mismatches (read, field, gpu, oracle): {mm}"
    assert strip_t(text) == strip_t(otext.decode())
    assert (rec["status"] == 0).mean() > 0.9
    g.close()


def _read_sketches(reads, k, r, packed):
    """The mapping path's read sketch (SK_APPEND) through the library's test
    hook: per read, its k-mers sorted by position."""
    import ctypes

    L = sb.lib()
    f = L.shm_internal_sketch_reads
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_double,
                  ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    seq, offs = pack(reads)
    caps = np.array([max(0, len(x) - k + 1) for x in reads], np.uint64)
    cap_off = np.concatenate([[0], np.cumsum(caps)]).astype(np.uint64)
    tot = max(1, int(cap_off[-1]))
    h = np.zeros(tot, np.uint64)
    rs = np.zeros(tot, np.uint32)
    cnt = np.zeros(max(1, len(reads)), np.uint32)
    assert f(0, seq.ctypes.data, offs.ctypes.data, len(reads), k, r, int(packed), cap_off.ctypes.data,
             h.ctypes.data, rs.ctypes.data, cnt.ctypes.data) == 0
    out = []
    for i in range(len(reads)):
        a = int(cap_off[i])
        m = int(cnt[i])
        assert m <= caps[i]
        hh, rr = h[a:a + m], rs[a:a + m]
        o = np.argsort(rr >> 1, kind="stable")
        out.append(((rr[o] >> 1).astype(np.int32), hh[o], (rr[o] & 1).astype(np.uint8)))
    return out


@pytest.mark.parametrize("k", [1, 5, 15, 25, 31, 32, 33, 64, 65, 100])
@pytest.mark.parametrize("r", [1.0, 0.5, 0.1, 0.01])
def test_read_sketch_packed_and_ascii(gpu_ctx, k, r):
    """The read sketch from 2-bit packed reads (rotated-frame rolling) and
    from the reads' bytes equals the oracle's sketch, per read: lengths around
    the 128-window runs, reads shorter than k, N runs, lower case and IUPAC
    bytes (which the packed form marks and rolls through the letter tables)."""
    rng = np.random.default_rng(k * 10 + int(r * 100))
    reads = []
    for L in [0, 1, k - 1, k, k + 1, 127 + k, 128 + k, 129 + k, 255 + k, 256 + k, 1000, 5003, 20000]:
        reads.append(lcg_dna(int(rng.integers(1, 1 << 30)), max(0, L)))
    s = bytearray(lcg_dna(77, 9000))
    s[3000:3040] = b"N" * 40
    s[5000:5400] = bytes(s[5000:5400]).lower()
    s[7000:7004] = b"RYK-"
    reads.append(bytes(s))
    reads.append(b"N" * 300)
    reads.append(xorshift_dna(5, 4000).lower())
    for packed in (1, 0):
        got = _read_sketches(reads, k, r, packed)
        for i, x in enumerate(reads):
            want = O.sketch(x, k, r)
            assert all(np.array_equal(a, b) for a, b in zip(got[i], want)), (packed, i, len(x))
