"""Index files (shm_index_save / shm_index_load): an index written to a file
and read back answers exactly as the index that was built — statistics,
segments, count() probes, hit lists and the mapping records and PAF of a read
set — at r < 1 (bucket table) and r = 1 (directory only), with and without
-M. Files that are missing, of another kind or truncated are refused with
SHM_ERR_INVALID. Run on a B200 with `pytest -m gpu`."""
import os

import numpy as np
import pytest

import shmap_b200 as sb
from helpers import pack, record_mismatches, xorshift_dna

pytestmark = pytest.mark.gpu


def _records():
    rep = b"ACGTACGTACGTACGTACGT"
    recs = [(f"chr{i}", xorshift_dna(100 + i, 40000 + 977 * i)) for i in range(6)]
    recs += [("repeats", (rep + b"TTGGCCAA") * 200), ("empty", b""), ("short", b"ACG")]
    return recs


def _reads(recs, n=300, seed=7):
    rng = np.random.default_rng(seed)
    comp = bytes.maketrans(b"ACGTacgt", b"TGCAtgca")
    out = []
    for i in range(n):
        name, s = recs[int(rng.integers(0, 6))]
        L = int(rng.integers(500, 6000))
        a = int(rng.integers(0, len(s) - L))
        r = bytearray(s[a:a + L])
        for j in rng.integers(0, L, L // 100):
            r[j] = b"ACGT"[int(rng.integers(0, 4))]
        r = bytes(r)
        if rng.integers(0, 2):
            r = r.translate(comp)[::-1]
        out.append((f"read{i}", r))
    return out


@pytest.mark.parametrize("k,r,mm", [(15, 0.05, None), (12, 0.2, 3), (8, 1.0, None)])
def test_saved_index_answers_as_built(gpu_ctx, tmp_path, k, r, mm):
    recs = _records()
    g = sb.SketchIndex.from_records(gpu_ctx, recs, k, r, mm)
    path = str(tmp_path / "ref.shmapidx")
    g.save(path)
    h = sb.SketchIndex.load(gpu_ctx, path)
    assert (h.k, h.h_frac) == (k, r) and h.names == [n for n, _ in recs]
    assert h.stats() == g.stats()
    for i in range(len(recs)):
        a, b = g.segment(i), h.segment(i)
        assert all(np.array_equal(x, y) for x, y in zip(a[:3], b[:3])) and a[3:] == b[3:]
    hs = np.unique(np.concatenate([g.segment(i)[1] for i in range(len(recs))] + [np.arange(64, dtype=np.uint64)]))
    assert np.array_equal(g.count(hs), h.count(hs))
    for x in hs[:: max(1, len(hs) // 50)]:
        assert all(np.array_equal(p, q) for p, q in zip(g.hits(int(x)), h.hits(int(x))))
    reads = _reads(recs)
    seq, offs = pack([s for _, s in reads])
    p = sb.Params(k=k, h_frac=r, theta=0.4)
    ra, rb = g.map_reads(p, seq, offs), h.map_reads(p, seq, offs)
    assert (ra["status"] == 0).sum() > 0
    assert not record_mismatches(ra, rb)
    names = [n for n, _ in reads]
    assert g.format_paf(p, ra, names) == h.format_paf(p, rb, names)
    h.close()
    g.close()


def test_bad_index_files_are_refused(gpu_ctx, tmp_path):
    g = sb.SketchIndex.from_records(gpu_ctx, _records(), 15, 0.05)
    good = str(tmp_path / "good.shmapidx")
    g.save(good)
    blob = open(good, "rb").read()
    cases = {"missing": None, "foreign": b"not an index at all" * 10, "truncated": blob[: len(blob) // 2],
             "short_tail": blob[:-3]}
    for name, data in cases.items():
        path = str(tmp_path / f"{name}.shmapidx")
        if data is not None:
            open(path, "wb").write(data)
        with pytest.raises(sb.ShmError) as e:
            sb.SketchIndex.load(gpu_ctx, path)
        assert e.value.code == -1, name  # SHM_ERR_INVALID
    g.close()


def test_file_written_from_the_oracle_loads_as_the_built_index(gpu_ctx, tmp_path):
    """A file written in the library's format from the CPU oracle's index
    (tests/test_index_file_check.py's writer) loads and answers as the index
    built on the device: the file format is the oracle's index, section for
    section."""
    from test_index_file_check import index_sections, write_index

    recs = _records()
    path = str(tmp_path / "oracle.shmapidx")
    write_index(path, index_sections(recs, 12, 0.2))
    g = sb.SketchIndex.from_records(gpu_ctx, recs, 12, 0.2)
    h = sb.SketchIndex.load(gpu_ctx, path)
    assert h.stats() == g.stats()
    hs = np.unique(np.concatenate([g.segment(i)[1] for i in range(len(recs))]))
    assert np.array_equal(g.count(hs), h.count(hs))
    reads = _reads(recs, 100)
    seq, offs = pack([s for _, s in reads])
    p = sb.Params(k=12, h_frac=0.2, theta=0.4)
    assert not record_mismatches(g.map_reads(p, seq, offs), h.map_reads(p, seq, offs))
    h.close()
    g.close()
