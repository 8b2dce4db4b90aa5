"""PAF text rendered on the device (shm_format_paf_device) against the host
formatter (shm_format_paf, itself pinned to the reference's golden PAF): the
same bytes for the mapped reads of all four metrics, for the golden fixture,
and for records whose f64 fields are ties at the printed precision (1/64 at
five places, 1/16 at three), NaN, infinities, negative zero, subnormals,
huge values and random doubles; a short buffer gives SHM_ERR_CAPACITY."""
import ctypes
import os

import numpy as np
import pytest

import shmap_b200 as sb
from helpers import pack
from shmap_b200 import fasta, synth

pytestmark = pytest.mark.gpu


def _same(g, p, rec, names, mt=None):
    host = g.format_paf(p, rec, names, mt)
    dev = sb.format_paf_device(g, p, rec, names, mt)
    assert dev == host
    return host


def test_golden_fixture(gpu_ctx, golden_dir):
    refs = fasta.read_fastx(os.path.join(golden_dir, "tiny_ref.fa"))
    reads = fasta.read_fastx(os.path.join(golden_dir, "tiny_reads.fa"))
    g = sb.SketchIndex.from_records(gpu_ctx, refs, 8, 1.0)
    p = sb.Params(k=8, h_frac=1.0, theta=0.1)
    seq, offs = pack([s for _, s in reads])
    rec = g.map_reads(p, seq, offs)
    assert len(_same(g, p, rec, [n for n, _ in reads]).splitlines()) == 2


@pytest.mark.parametrize("metric", ["Containment", "Jaccard", "bucket_SH", "bucket_LCS"])
def test_mapped_reads(gpu_ctx, metric):
    gen = synth.Genome(synth.REFS["uniform5m"])
    names, seq, offs = gen.reads(synth.READS["fixed10k"])
    g = sb.SketchIndex.from_records(gpu_ctx, gen.records(), 25, 0.01)
    p = sb.Params(k=25, h_frac=0.01, theta=0.4, metric=metric)
    rec = g.map_reads(p, seq, offs)
    mt = np.random.default_rng(1).random(len(rec)) * 1e-3
    text = _same(g, p, rec, list(names), mt)
    assert len(text.splitlines()) == int((rec["status"] == 0).sum()) > 0


def test_adversarial_doubles(gpu_ctx):
    gen = synth.Genome(synth.REFS["uniform5m"])
    names, seq, offs = gen.reads(synth.scaled(synth.READS["fixed10k"], 0.1))
    g = sb.SketchIndex.from_records(gpu_ctx, gen.records(), 25, 0.01)
    p = sb.Params(k=25, h_frac=0.01, theta=0.4)
    rec = g.map_reads(p, seq, offs)
    ok = np.nonzero(rec["status"] == 0)[0]
    rec = rec[np.resize(ok, 400)].copy()
    rng = np.random.default_rng(2)
    special = np.array([1 / 64, -1 / 64, 3 / 64, 0.5, 0.0, -0.0, np.nan, np.inf, -np.inf, 5e-324, 2.2250738585072014e-308,
                        1e300, -1e300, 1.7976931348623157e308, 2.0 ** 109, 2.0 ** 110 + 2.0 ** 58, 2.0 ** 56 * 3,
                        123456789.123456789, 0.999995, 0.000005, 1e-5, 0.3, 0.1 + 0.2, 2.5e-6, 7.5e-6])
    n = len(rec)
    for f in ("score", "sh", "score2"):
        v = rng.random(n)
        v[: len(special)] = special
        rng.shuffle(v)
        rec[f] = v
    rec["has_second"] = rng.integers(0, 2, n)
    rec["intersection2"] = rng.choice([-1, 0, 3, 1000], n)
    rec["intersection"] = rng.choice([0, 1, 16, 200, 7], n)
    rec["total_matches"] = rng.choice([0, 1, 3, 100000], n)  # 1/16 = 0.0625 is a tie at three places
    rec["same_strand"] = rng.integers(-300, 300, n)
    mt = np.concatenate([special, rng.random(n - len(special)) * 10.0 ** rng.integers(-8, 8, n - len(special))])
    names = [f"q{i}" for i in range(n)]
    text = _same(g, p, rec, names, mt)
    assert "NaN" in text and "inf" in text and "-0.00000" in text
    assert "J:f:0.01562" in text  # 1562.5 rounds to even


def test_capacity(gpu_ctx, golden_dir):
    import ctypes

    refs = fasta.read_fastx(os.path.join(golden_dir, "tiny_ref.fa"))
    reads = fasta.read_fastx(os.path.join(golden_dir, "tiny_reads.fa"))
    g = sb.SketchIndex.from_records(gpu_ctx, refs, 8, 1.0)
    p = sb.Params(k=8, h_frac=1.0, theta=0.1)
    seq, offs = pack([s for _, s in reads])
    rec = g.map_reads(p, seq, offs)
    names = [n for n, _ in reads]
    full = g.format_paf(p, rec, names).encode()
    buf = ctypes.create_string_buffer(50)
    need = ctypes.c_int64()
    cp = p.c()
    rc = sb.lib().shm_format_paf_device(gpu_ctx.h, g.h, ctypes.byref(cp), rec.ctypes.data, len(rec),
                                        "\n".join(names).encode(), None, buf, 50, ctypes.byref(need))
    assert rc == sb.SHM_ERR_CAPACITY and need.value == len(full)
    assert buf.raw[:50] == full[:50]


@pytest.mark.parametrize("env", [{}, {"SHMAP_FAST_JOB_CAP": "7"}])
@pytest.mark.parametrize("metric", ["Containment", "bucket_SH"])
def test_map_paf(gpu_ctx, monkeypatch, metric, env):
    """shm_map_paf (reads in, PAF text out, each batch rendered on the device
    as soon as it is mapped) gives the host formatter's bytes over the same
    records, and the oracle's PAF (t:f: aside). More reads than one host batch
    holds, so several batches write into the one text; with a tiny bucket-job
    capacity batches are mapped again and the call renders from the final
    records instead."""
    import oracle as O

    for k, v in env.items():
        monkeypatch.setenv(k, v)
    gen = synth.Genome(synth.REFS["uniform5m"])
    names, seq, offs = gen.reads(synth.scaled(synth.READS["fixed10k"], 2.5))  # 5,000 reads, 50 Mbp
    names = [f"{n} extra-{i}" if i % 7 == 0 else n for i, n in enumerate(names)]
    g = sb.SketchIndex.from_records(gpu_ctx, gen.records(), 25, 0.01)
    p = sb.Params(k=25, h_frac=0.01, theta=0.4, metric=metric)
    text, rec = g.map_paf(p, seq, offs, names)
    assert not np.any(rec["status"] == 3)
    assert text == g.format_paf(p, rec, names)
    o = O.Index.from_records(gen.records(), 25, 0.01, threads=8)
    orec, otext, _ = o.map_paf(O.params(k=25, h_frac=0.01, theta=0.4, metric=metric), seq, offs, names, 8)
    assert rec.tobytes() == orec.tobytes()
    assert sb.strip_timing(text) == sb.strip_timing(otext.decode())
    assert len(text.splitlines()) == int((rec["status"] == 0).sum()) > 4000
    t2, r2 = g.map_paf(p, seq[: offs[3]], offs[:4], names[:3], with_records=False)
    assert r2 is None and t2 == g.format_paf(p, rec[:3], names[:3])
    t0, _ = g.map_paf(p, seq[:0], offs[:1], [])
    assert t0 == ""


@pytest.mark.gpu
@pytest.mark.parametrize("env", [{}, {"SHMAP_FAST_JOB_CAP": "7"}])
def test_map_paf_pinned_buffer(gpu_ctx, monkeypatch, env):
    """Into a pinned, aligned caller buffer shm_map_paf writes each batch's
    text through the buffer's device mapping while later batches map; the
    bytes equal those written into pageable memory, also at an offset of one
    byte (no mapping used), with a capacity short of the text (its first cap
    bytes), and when batches are mapped again (the call renders from the
    final records)."""
    import torch

    for k, v in env.items():
        monkeypatch.setenv(k, v)
    gen = synth.Genome(synth.REFS["uniform5m"])
    names, seq, offs = gen.reads(synth.scaled(synth.READS["fixed10k"], 2.5))  # 5,000 reads
    g = sb.SketchIndex.from_records(gpu_ctx, gen.records(), 25, 0.01)
    p = sb.Params(k=25, h_frac=0.01, theta=0.4)
    want, _ = g.map_paf(p, seq, offs, names)
    want_b = want.encode()
    seq = np.ascontiguousarray(seq, dtype=np.uint8)
    offs = np.ascontiguousarray(offs, dtype=np.int64)
    joined = "\n".join(names).encode()
    cp = p.c()
    pin = torch.zeros(len(want_b) + 64, dtype=torch.uint8).pin_memory()
    base = pin.data_ptr()
    for shift, cap in ((0, len(want_b) + 32), (1, len(want_b) + 32), (0, len(want_b) // 3)):
        pin.fill_(0)
        need = ctypes.c_int64()
        rc = sb.lib().shm_map_paf(gpu_ctx.h, g.h, ctypes.byref(cp), seq.ctypes.data, offs.ctypes.data, len(names),
                                  joined, None, base + shift, cap, ctypes.byref(need))
        assert need.value == len(want_b)
        got = bytes(pin.numpy()[shift:shift + min(cap, need.value)])
        assert got == want_b[:min(cap, need.value)], (shift, cap)
        assert rc == (0 if cap >= need.value else sb.SHM_ERR_CAPACITY)
