"""Pins the CPU oracle to the reference's own golden PAF and known-answer
tests (CPU only). The oracle is the checker of the GPU parity tests, so it is
checked first, against every fixture and constant the reference's tests hold
for this path."""
import json
import os
import tempfile

import numpy as np
import pytest

import oracle as O
from helpers import (floor_reads, floor_reference, lcg_dna, nthash_direct, pack, strip_t, thread_parity_workload,
                     xorshift_dna)


@pytest.fixture(scope="module")
def known(golden_dir):
    with open(os.path.join(golden_dir, "known_answers.json")) as f:
        return json.load(f)


def _fa(tmp, name, records):
    p = os.path.join(tmp, name)
    with open(p, "w") as f:
        for n, s in records:
            f.write(f">{n}\n{s.decode() if isinstance(s, bytes) else s}\n")
    return p


def test_golden_paf_matches(golden_dir):
    """tests/golden_paf.rs:25-53: every field except the wall-clock t:f:."""
    r = O.run_cli(["-s", os.path.join(golden_dir, "tiny_ref.fa"), "-p", os.path.join(golden_dir, "tiny_reads.fa"),
                   "-k", "8", "-r", "1.0", "-t", "0.1"])
    assert r.returncode == 0, r.stderr
    want = strip_t(open(os.path.join(golden_dir, "tiny.golden.paf")).read().rstrip("\n"))
    assert strip_t(r.stdout) == want


def test_integration_lines(golden_dir):
    """tests/integration_paf.rs:8-43."""
    r = O.run_cli(["-s", os.path.join(golden_dir, "tiny_ref.fa"), "-p", os.path.join(golden_dir, "tiny_reads.fa"),
                   "-k", "8", "-r", "1.0", "-t", "0.1"])
    lines = r.stdout.splitlines()
    assert len(lines) == 2
    for ln in lines:
        f = ln.split("\t")
        assert len(f) >= 12 and f[5] == "ref" and f[4] == "+"
    assert lines[0].startswith("read1\t") and lines[1].startswith("read2\t")


def test_invalid_k_rejected(golden_dir):
    """tests/integration_paf.rs:45-57."""
    r = O.run_cli(["-s", os.path.join(golden_dir, "tiny_ref.fa"), "-p", os.path.join(golden_dir, "tiny_reads.fa"),
                   "-k", "0"])
    assert r.returncode != 0 and "K-mer length" in r.stderr


@pytest.mark.parametrize("r", [0.01, 0.05, 0.1, 0.5, 0.999, 1.0])
def test_h_thres(r):
    """src/sketch.rs:126-132: (h_frac * u64::MAX as f64) as u64, u64::MAX at 1.0."""
    want = (1 << 64) - 1 if r >= 1.0 else int(r * float((1 << 64) - 1))
    assert O.h_thres(r) == want
    if r == 0.01:
        assert want == 0x028F5C28F5C28F60
    if r == 0.1:
        assert want == 0x1999999999999A00


@pytest.mark.parametrize("k", [15, 21, 25, 31])
def test_rolling_hash_is_the_direct_definition(k):
    """tests/nthash_equivalence.rs:65-112: rolling == definition; canonical is xor; strand = fw > rc."""
    seq = xorshift_dna(12 + k, 600)
    r, h, st = O.sketch(seq, k, 1.0)
    d = nthash_direct(seq, k)
    assert len(h) == len(d)
    assert [int(x) for x in h] == [f ^ c for f, c in d]
    assert [bool(x) for x in st] == [f > c for f, c in d]
    assert list(r) == list(range(k - 1, len(seq)))


def test_non_acgt_and_lowercase():
    """src/sketch.rs:65-88: lower/upper case alike; every other byte hashes to 0."""
    seq = b"ACGTNNNNNNNacgtRYKMacgtACGTnnnnACGT" * 4
    r, h, st = O.sketch(seq, 5, 1.0)
    d = nthash_direct(seq, 5)
    assert [int(x) for x in h] == [f ^ c for f, c in d]
    assert 0 in set(int(x) for x in h)  # an all-N window hashes to 0 and is always kept
    lower = O.sketch(seq.lower(), 5, 1.0)[1]
    assert np.array_equal(lower, h)


def test_chunked_sketch_concatenates():
    """src/sketch.rs:235-270."""
    k = 7
    seq = lcg_dna(0x123456789ABCDEF0, 5000)
    whole = O.sketch(seq, k, 0.5)
    nw = len(seq) - k + 1
    for chunk in (1, 2, 13, 500, nw - 1, nw):
        parts = []
        w0 = 0
        while w0 < nw:
            w1 = min(w0 + chunk, nw)
            parts.append(O.sketch(seq[w0:w1 + k - 1], k, 0.5, offset=w0))
            w0 = w1
        for a, b in zip(whole, (np.concatenate([p[i] for p in parts]) for i in range(3))):
            assert np.array_equal(a, b), chunk


def test_rc_symmetry(known):
    """src/sketch.rs:272-296."""
    c = known["rc_symmetry"]
    k = c["k"]
    a = O.sketch(c["s"].encode(), k, 1.0)
    b = O.sketch(c["s_rc"].encode(), k, 1.0)
    assert len(a[0]) == len(b[0])
    br = (b[0][::-1], b[1][::-1])
    for i in range(len(a[0])):
        assert a[0][i] == i + k - 1
        assert a[0][i] == len(a[0]) - br[0][i] + k + 1
        assert a[1][i] == br[1][i]


def test_shorter_than_k(known):
    c = known["shorter_than_k"]
    assert len(O.sketch(c["s"].encode(), c["k"], 1.0)[0]) == 0


@pytest.mark.parametrize("case", ["single_segment", "two_segments"])
def test_index_counts(known, case):
    """src/index.rs:715-769."""
    c = known[case]
    recs = []
    for blk in c["fasta"].strip().split(">")[1:]:
        name, s = blk.split("\n", 1)
        recs.append((name, s.replace("\n", "").encode()))
    idx = O.Index.from_records(recs, c["k"], c["r"])
    _, h, _ = O.sketch(b"ACCAGTACCA", c["k"], c["r"])
    assert list(idx.count(h)) == c["counts"]
    st = idx.stats()
    assert st["indexed_hits"] == c["indexed_hits"] and st["indexed_kmers"] == c["indexed_kmers"]


def _max_matches_records(c):
    return [(f"segm{i}", (c["repeated"] + c["suffix"] + str(i)).encode()) for i in range(10)]


def test_max_matches_thread_invariance(known):
    """src/index.rs:783-855: -M 3, -@1 vs -@8 give the same index."""
    c = known["max_matches_case"]
    recs = _max_matches_records(c)
    a = O.Index.from_records(recs, c["k"], c["r"], c["max_matches"], threads=1)
    b = O.Index.from_records(recs, c["k"], c["r"], c["max_matches"], threads=8)
    assert a.stats()["blacklisted_kmers"] > 0
    assert a.stats() == b.stats()
    hs = np.unique(np.concatenate([O.sketch(s, c["k"], 1.0)[1] for _, s in recs]))
    assert np.array_equal(a.count(hs), b.count(hs))
    for h in hs[:50]:
        for x, y in zip(a.hits(int(h)), b.hits(int(h))):
            assert np.array_equal(x, y)


def _cli_map(tmp, ref_recs, read_recs, args):
    rp = _fa(tmp, "ref.fa", ref_recs)
    qp = _fa(tmp, "reads.fa", read_recs)
    r = O.run_cli(["-s", rp, "-p", qp, *args])
    assert r.returncode == 0, r.stderr
    return r.stdout


def test_sketch_floor(known):
    """tests/short_read_sketch_floor.rs:275-310."""
    c = known["sketch_floor"]
    ref = floor_reference()
    with tempfile.TemporaryDirectory() as tmp:
        out = _cli_map(tmp, [("ref", ref)], floor_reads(ref, c["below"]), c["params"])
        assert out.strip() == ""
        out = _cli_map(tmp, [("ref", ref)], floor_reads(ref, c["above"]), c["params"])
        lines = [ln for ln in out.splitlines() if ln.strip()]
        assert len(lines) == len(c["above"])
        for ln in lines:
            f = ln.split("\t")
            assert 0 <= int(f[2]) < int(f[3]) <= int(f[1])
        out = _cli_map(tmp, [("ref", ref)], floor_reads(ref, c["mixed"]), c["params"])
        assert len([ln for ln in out.splitlines() if ln.strip()]) == c["mixed_mapped"]


def test_thread_parity():
    """tests/multithreaded_parity.rs:60-101: -@1/3/8 give byte-identical PAF."""
    refs, reads = thread_parity_workload()
    with tempfile.TemporaryDirectory() as tmp:
        outs = [strip_t(_cli_map(tmp, refs, reads, ["-k", "12", "-r", "0.5", "-t", "0.2", "-@", t]))
                for t in ("1", "3", "8")]
    assert outs[0] and outs[0] == outs[1] == outs[2]


def test_records_and_paf_agree():
    """The ctypes record path and the CLI path of the oracle render the same PAF."""
    refs, reads = thread_parity_workload()
    seq, off = pack([s for _, s in refs])
    idx = O.Index([n for n, _ in refs], seq, off, 12, 0.5)
    p = O.params(k=12, h_frac=0.5, theta=0.2)
    rs, ro = pack([s for _, s in reads])
    paf = idx.paf(p, rs, ro, [n for n, _ in reads])
    with tempfile.TemporaryDirectory() as tmp:
        cli = _cli_map(tmp, refs, reads, ["-k", "12", "-r", "0.5", "-t", "0.2"])
    assert strip_t(paf) == strip_t(cli)
    rec = idx.map_reads(p, rs, ro)
    assert (rec["status"] == 0).sum() == len(paf.splitlines())


def test_lcs_known_answer():
    """src/shmap/scoring.rs:498-535: bucket 1 at half-length 2 over seven
    reference k-mers, three seeds with pmatches [5, 1], [4, 2], [3] -> 3."""
    t = [(10, 0x111111), (20, 0x222222), (30, 0x111111), (40, 0x444444), (50, 0x555555), (60, 0x111111),
         (70, 0x222222)]
    assert O.lcs(t, 2, 6, {0x111111: [5, 1], 0x222222: [4, 2], 0x444444: [3]}) == 3


def _lis_brute(xs):
    """Longest strictly increasing subsequence by the quadratic recurrence."""
    best = [1] * len(xs)
    for i in range(len(xs)):
        for j in range(i):
            if xs[j] < xs[i]:
                best[i] = max(best[i], best[j] + 1)
    return max(best, default=0)


@pytest.mark.parametrize("seed", range(6))
def test_lcs_matches_the_definition(seed):
    """scoring.rs:114-170 restated: positions of every window k-mer's seed,
    then the longer of the increasing runs forward and backward."""
    rng = np.random.default_rng(seed)
    hashes = [int(x) for x in rng.integers(1, 1 << 40, 12)]
    t = [(10 * i, hashes[int(rng.integers(0, 12))]) for i in range(60)]
    seeds = {h: sorted(rng.choice(200, int(rng.integers(1, 4)), replace=False).tolist(), reverse=True)
             for h in hashes[:8]}
    for bgn, end in [(0, 60), (7, 31), (40, 80), (59, 60), (5, 5)]:
        pp = [x for _, h in t[bgn:min(end, len(t))] if h in seeds for x in seeds[h]]
        assert O.lcs(t, bgn, end, seeds) == max(_lis_brute(pp), _lis_brute(pp[::-1]))


def _rarity_workload(seed=31, n=150):
    ref = lcg_dna(seed, 400_000)
    rep = lcg_dna(seed + 1, 3000)
    ref_rep = ref[:100_000] + rep * 6 + ref[100_000:200_000] + rep * 4 + ref[200_000:]  # copies of one repeat
    rng = np.random.default_rng(seed)
    comp = bytes.maketrans(b"ACGT", b"TGCA")
    reads = []
    for i in range(n):
        L = int(rng.integers(2000, 6000))
        a = int(rng.integers(0, len(ref_rep) - L))
        r = bytearray(ref_rep[a:a + L])
        for j in rng.integers(0, L, L // 50):
            r[j] = b"ACGT"[int(rng.integers(0, 4))]
        r = bytes(r)
        reads.append(r.translate(comp)[::-1] if i % 2 else r)
    return ref, ref_rep, reads


def test_rarity_weight_is_containment_when_every_kmer_is_unique():
    """src/shmap/mod.rs:694-723, scoring.rs:214-281: with hits_in_t = 1 for
    every seed all weights are 1, the weighted support is the count and the
    weighted score is Containment's, record for record."""
    ref, _, reads = _rarity_workload()
    idx = O.Index.from_records([("u", ref)], 21, 0.1)
    # the reads none of whose sketched k-mers occurs twice in the reference
    unique = [r for r in reads if (idx.count(O.sketch(r, 21, 0.1)[1]) <= 1).all()]
    assert len(unique) >= 40
    seq, offs = pack(unique)
    base = idx.map_reads(O.params(k=21, h_frac=0.1, theta=0.3), seq, offs, threads=4)
    assert (base["status"] == 0).mean() > 0.9
    for alpha in (0.5, 1.0, 2.0):
        w = idx.map_reads(O.params(k=21, h_frac=0.1, theta=0.3, rarity_weight=alpha), seq, offs, threads=4)
        assert np.array_equal(w.view(np.uint8), base.view(np.uint8)), alpha


def test_rarity_tiebreak_only_admits_more():
    """scoring.rs:409-481: the band lowers the admission bar and decides near
    ties by rarity support; a read mapped without it stays mapped."""
    _, ref_rep, reads = _rarity_workload()
    idx = O.Index.from_records([("r", ref_rep)], 15, 0.2)
    seq, offs = pack(reads)
    base = idx.map_reads(O.params(k=15, h_frac=0.2, theta=0.3), seq, offs, threads=4)
    for band, alpha in ((0.01, 0.0), (0.05, 1.0), (0.2, 2.0)):
        tb = idx.map_reads(O.params(k=15, h_frac=0.2, theta=0.3, rarity_tiebreak=band, rarity_alpha=alpha), seq,
                           offs, threads=4)
        mapped_base = base["status"] == 0
        assert (tb["status"][mapped_base] == 0).all(), band
    wt = idx.map_reads(O.params(k=15, h_frac=0.2, theta=0.3, rarity_weight=1.0), seq, offs, threads=4)
    ok = wt["status"] == 0
    assert ok.any() and ((wt["score"][ok] >= 0.0) & (wt["score"][ok] <= 1.0)).all()
    assert not np.array_equal(wt["score"][ok], base["score"][ok])  # repeats are down-weighted


def test_rarity_flag_validation(golden_dir):
    """src/params.rs:223-242."""
    args = ["-s", os.path.join(golden_dir, "tiny_ref.fa"), "-p", os.path.join(golden_dir, "tiny_reads.fa"), "-k", "8"]
    r = O.run_cli(args + ["--rarity-weight", "5"])
    assert r.returncode != 0 and "rarity weight" in r.stderr
    r = O.run_cli(args + ["--rarity-weight", "1", "-m", "Jaccard"])
    assert r.returncode != 0 and "only defined for -m Containment" in r.stderr
    r = O.run_cli(args + ["-r", "1.0", "-t", "0.1", "--rarity-tiebreak", "0.01"])
    assert r.returncode == 0 and len(r.stdout.splitlines()) == 2
