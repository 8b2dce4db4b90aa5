"""FASTA parsed on the device (shm_fasta_parse_device) against the host reader
(shmap_b200.fasta.read_fastx, the reference's record rules, src/io/mod.rs:383-427):
the same names, offsets and bases for files of random records, line breaks
('\\n', '\\r\\n', none at the end), blank lines, long lines across the parser's
chunk boundaries and headers with spaces and tabs. FASTQ (a first byte '@')
is parsed as four-line records by line index: quality lines starting with
'@', CRLF, long reads across chunks, trailing blank lines. A FASTA file with
'@' lines or text before the first header, and FASTQ that is not four-line
records, are refused (the host reader takes those). An index built from
the device copy equals the one built from host records, reads mapped from it
get the same records, and the command line prints the same PAF either way."""
import os
import subprocess

import numpy as np
import pytest

import shmap_b200 as sb
from helpers import pack, record_mismatches, strip_t, xorshift_dna
from shmap_b200 import fasta

pytestmark = pytest.mark.gpu


def _random_fasta(seed, n_rec, max_len, width_choices=(0, 60, 61, 16384, 40000)):
    rng = np.random.default_rng(seed)
    out = bytearray()
    for i in range(n_rec):
        eol = b"\r\n" if rng.integers(0, 3) == 0 else b"\n"
        name = f"rec{i}" + ["", " desc x", "\tt", " "][int(rng.integers(0, 4))]
        out += b">" + name.encode() + eol
        L = int(rng.integers(0, max_len))
        s = xorshift_dna(seed * 1000 + i, L)
        w = int(width_choices[int(rng.integers(0, len(width_choices)))]) or max(L, 1)
        for j in range(0, L, w):
            out += s[j:j + w] + eol
            if rng.integers(0, 20) == 0:
                out += eol  # a blank line inside the record
    if len(out) and rng.integers(0, 2):
        out = out.rstrip(b"\r\n")  # no line end after the last line
    return bytes(out)


def _host(tmp_path, data):
    p = tmp_path / "x.fa"
    p.write_bytes(data)
    return fasta.read_fastx(str(p))


@pytest.mark.parametrize("seed,n_rec,max_len", [(1, 1, 10), (2, 50, 3000), (3, 400, 70000), (4, 5, 300000),
                                                (5, 3000, 200)])
def test_records_as_the_host_reads_them(gpu_ctx, tmp_path, seed, n_rec, max_len):
    data = _random_fasta(seed, n_rec, max_len)
    want = _host(tmp_path, data)
    fa = sb.DeviceFasta(gpu_ctx, data)
    assert fa.n == len(want)
    assert fa.names == [n for n, _ in want]
    seq = fa.seq().tobytes()
    got = [seq[fa.offs[i]:fa.offs[i + 1]] for i in range(fa.n)]
    assert got == [s for _, s in want]
    fa.close()


@pytest.mark.parametrize("data", [b"", b"\n\n", b">only\n", b">a\r\n\r\nAC\r\nGT\r\n>b\n>c\nTT", b">x y\tz\n" + b"A" * 20000,
                                  b"\r\n>r\nACGT\r", b">caf\xe9 x\nACGT\n>\xf0\x90\x80\nGG\n>ok\xe2\x82\xac\xff\nT\n"])
def test_edge_files(gpu_ctx, tmp_path, data):
    want = _host(tmp_path, data)
    fa = sb.DeviceFasta(gpu_ctx, data)
    seq = fa.seq().tobytes()
    assert fa.names == [n for n, _ in want]
    assert [seq[fa.offs[i]:fa.offs[i + 1]] for i in range(fa.n)] == [s for _, s in want]


@pytest.mark.parametrize("data", [b">a\nAC\n@b\nGG\n", b"ACGT\n>a\nAC\n", b" \n>a\nA\n",
                                  b"@q\nACGT\nIIII\nIIII\n", b"@q\nAC\n+\nII\n\n@r\nGG\n+\nII\n",
                                  b"@q\nAC\n+\nII\nr\nGG\n+\nII\n"])
def test_refused_files(gpu_ctx, data):
    with pytest.raises(sb.ShmError) as e:
        sb.DeviceFasta(gpu_ctx, data)
    assert e.value.code == sb.SHM_ERR_INVALID


def test_index_and_mapping_from_the_device_copy(gpu_ctx, tmp_path):
    ref_recs = [(f"chr{i}", xorshift_dna(40 + i, 200_000 + 7919 * i)) for i in range(4)]
    ref = b"".join(b">" + n.encode() + b" sample\n" + b"\n".join(s[j:j + 80] for j in range(0, len(s), 80)) + b"\n"
                   for n, s in ref_recs)
    rng = np.random.default_rng(9)
    reads = []
    for i in range(500):
        name, s = ref_recs[int(rng.integers(0, 4))]
        L = int(rng.integers(1000, 8000))
        a = int(rng.integers(0, len(s) - L))
        reads.append((f"read{i}", s[a:a + L]))
    rd = b"".join(b">" + n.encode() + b"\n" + s + b"\n" for n, s in reads)
    tfa = sb.DeviceFasta(gpu_ctx, ref)
    g_dev = sb.SketchIndex.from_device_fasta(gpu_ctx, tfa, 15, 0.1)
    g_host = sb.SketchIndex.from_records(gpu_ctx, ref_recs, 15, 0.1)
    assert g_dev.stats() == g_host.stats()
    for i in range(4):
        a, b = g_dev.segment(i), g_host.segment(i)
        assert all(np.array_equal(x, y) for x, y in zip(a[:3], b[:3]))
    pfa = sb.DeviceFasta(gpu_ctx, rd)
    p = sb.Params(k=15, h_frac=0.1, theta=0.4)
    got = g_dev.map_device_fasta(p, pfa)
    seq, offs = pack([s for _, s in reads])
    want = g_host.map_reads(p, seq, offs)
    assert (want["status"] == 0).mean() > 0.9
    assert not record_mismatches(got, want)
    part = g_dev.map_device_fasta(p, pfa, 100, 50)
    assert not record_mismatches(part, want[100:150])

    (tmp_path / "ref.fa").write_bytes(ref)
    (tmp_path / "reads.fa").write_bytes(rd)
    args = [sb.CLI_PATH, "-s", str(tmp_path / "ref.fa"), "-p", str(tmp_path / "reads.fa"), "-k", "15", "-r", "0.1",
            "-t", "0.4"]
    dev = subprocess.run(args, capture_output=True, text=True, timeout=300)
    host = subprocess.run(args + ["--host-fasta"], capture_output=True, text=True, timeout=300)
    assert dev.returncode == 0 and host.returncode == 0, dev.stderr + host.stderr
    assert strip_t(dev.stdout) == strip_t(host.stdout) and len(dev.stdout.splitlines()) > 400


def _random_fastq(seed, n_rec, max_len, crlf=False):
    rng = np.random.default_rng(seed)
    nl = b"\r\n" if crlf else b"\n"
    parts = []
    for i in range(n_rec):
        L = int(rng.integers(0, max_len + 1))
        sq = bytes(rng.choice(np.frombuffer(b"ACGTNacgt", np.uint8), L))
        qual = bytes(rng.choice(np.frombuffer(b"@!#IJ+>", np.uint8), L))  # quality lines may start with '@'
        hdr = b"@r%d" % i + (b" extra\tx" if i % 3 == 0 else b"")
        parts.append(hdr + nl + sq + nl + (b"+" if i % 2 else b"+" + hdr[1:]) + nl + qual)
        if i + 1 < n_rec or i % 2:
            parts.append(nl)
    return b"".join(parts) + (b"\n\n" if seed % 2 else b"")


@pytest.mark.parametrize("seed,n_rec,max_len,crlf", [(1, 1, 10, False), (2, 300, 3000, True), (3, 40, 60000, False),
                                                     (4, 2000, 200, True), (5, 3, 0, False)])
def test_fastq_records_as_the_host_reads_them(gpu_ctx, tmp_path, seed, n_rec, max_len, crlf):
    data = _random_fastq(seed, n_rec, max_len, crlf)
    want = _host(tmp_path, data)
    assert len(want) == n_rec
    fa = sb.DeviceFasta(gpu_ctx, data)
    assert fa.n == n_rec and fa.names == [n for n, _ in want]
    seq = fa.seq().tobytes()
    assert [seq[fa.offs[i]:fa.offs[i + 1]] for i in range(fa.n)] == [s for _, s in want]
    fa.close()


@pytest.mark.parametrize("data", [b"@q\nACGT\n+\n", b"@q\nACGT\n+\n\n\n", b"@q x\nAC\r\n+\r\n\r\n@r\nGG", b"@q\n"])
def test_fastq_short_last_records(gpu_ctx, tmp_path, data):
    """A last record without its (empty) quality line, or with only its
    header, reads as the host reader reads it."""
    want = _host(tmp_path, data)
    fa = sb.DeviceFasta(gpu_ctx, data)
    seq = fa.seq().tobytes()
    assert fa.names == [n for n, _ in want]
    assert [seq[fa.offs[i]:fa.offs[i + 1]] for i in range(fa.n)] == [s2 for _, s2 in want]
    fa.close()
