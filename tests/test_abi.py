"""The C ABI library loads and exports every entry point include/shmap_gpu.h
declares; the host-side logic that needs no GPU behaves like the reference's
(CPU only: nothing here launches a kernel)."""
import ctypes
import os
import re

import numpy as np
import pytest

import oracle as O
import shmap_b200 as sb
from shmap_b200 import fasta, synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    hdr = open(os.path.join(ROOT, "include", "shmap_gpu.h")).read()
    return sorted(set(re.findall(r"\b(shm_[a-z_0-9]+)\s*\(", hdr)))


def test_library_exports_every_declared_symbol():
    L = ctypes.CDLL(sb.LIB_PATH)
    names = declared_symbols()
    assert len(names) >= 18
    for n in names:
        assert hasattr(L, n), n


def test_python_binding_covers_every_symbol():
    L = sb.lib()
    for n in declared_symbols():
        assert getattr(L, n).argtypes is not None, n


@pytest.mark.parametrize("kw,msg", [
    (dict(k=0), "K-mer length (-k) should be positive. You provided 0."),
    (dict(h_frac=0.0), "Given hash ratio (-r) should be between 0 and 1. You provided 0."),
    (dict(h_frac=1.5), "Given hash ratio (-r) should be between 0 and 1. You provided 1.5."),
    (dict(max_matches=0), "The number of seed matches (-M) should be positive. You provided 0."),
    (dict(theta=1.2), "The threshold (-t) should be between 0 and 1. You provided 1.2."),
    (dict(min_diff=-0.1), "The minimum difference (-d) should be >= 0. You provided -0.1."),
    (dict(max_overlap=2.0), "The maximum overlap (-o) should be between 0 and 1. You provided 2."),
])
def test_params_validation_messages(kw, msg):
    """src/params.rs:191-263: same checks, same messages."""
    with pytest.raises(sb.ShmError) as e:
        sb.Params(**kw).validate()
    assert msg in str(e.value)


def test_params_defaults():
    """src/params.rs:29-116."""
    p = sb.CParams()
    sb.lib().shm_params_default(ctypes.byref(p))
    assert (p.k, p.h_frac, p.max_matches, p.theta, p.min_diff, p.max_overlap, p.metric) == (
        15, 0.05, -1, 0.9, 0.02, 0.5, sb.CONTAINMENT)
    sb.Params().validate()


@pytest.mark.parametrize("r", [0.01, 0.05, 0.1, 0.25, 0.5, 1.0])
def test_h_thres_matches_oracle(r):
    assert sb.h_thres(r) == O.h_thres(r)


def test_synthetic_generator_is_deterministic():
    spec = synth.scaled(synth.REFS["human31"], 0.002)
    a = synth.Genome(spec, threads=1)
    b = synth.Genome(spec, threads=7)
    assert np.array_equal(a.seq, b.seq) and a.names == b.names
    assert a.spec.total_bases == len(a.seq)
    ra = a.reads(synth.scaled(synth.READS["hifi"], 0.001), threads=1)
    rb = b.reads(synth.scaled(synth.READS["hifi"], 0.001), threads=5)
    assert ra[0] == rb[0] and np.array_equal(ra[1], rb[1]) and np.array_equal(ra[2], rb[2])
    assert set(np.unique(a.seq).tobytes()) <= set(b"ACGT")


def test_read_headers_follow_simulator_convention():
    g = synth.Genome(synth.REFS["uniform5m"])
    names, seq, offs = g.reads(synth.scaled(synth.READS["fixed10k"], 0.01))
    for nm in names:
        f = nm.split("!")
        assert len(f) == 5 and f[0].startswith("S") and f[0].endswith("_1") and f[4] in "+-"
        assert int(f[3]) - int(f[2]) == 10_000


def test_fasta_reader_semantics(tmp_path):
    """src/io/mod.rs:434-452 and 521-549: id cut at whitespace, CRLF, no final newline."""
    p = tmp_path / "x.fa"
    p.write_bytes(b">a desc\r\nACGT\r\nGGTT\r\n>b\tmore\r\nTTTT")
    assert fasta.read_fastx(str(p)) == [("a", b"ACGTGGTT"), ("b", b"TTTT")]


def test_no_gpu_is_an_error_not_a_fallback():
    """Without a usable device the context call fails loudly."""
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if has_gpu:
        pytest.skip("a GPU is present")
    with pytest.raises(sb.ShmError):
        sb.Context(0)
