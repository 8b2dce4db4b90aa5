"""The reference's own unit tests of the bucket accumulator, bucket content,
Mapping, the seed grouping and the FASTA reader, restated on the oracle
through its test hooks (and, for the reader, on the package's reader that the
device parser is compared with): the known answers of src/buckets.rs:748-957,
src/types.rs:329-339, src/mapping.rs:445-495, src/shmap/seeding.rs:221-245
and src/io/mod.rs:435-580."""
import oracle as O


# ---------------------------------------------------------------- buckets.rs:748-957
def test_begin_end_bucket_boundaries():
    b = O.Buckets(100)
    b.set_halflen(10)
    assert (b.begin(0, 0), b.end(0, 0)) == (0, 20)
    assert (b.begin(0, 1), b.end(0, 1)) == (10, 30)


def test_add_to_pos_touches_bucket_and_predecessor():
    b = O.Buckets(100)
    b.set_halflen(10)
    b.add_to_pos(25, 25, 0, 1, 0, 1, 25, 25)  # tpos 25: bucket 2 and its predecessor 1
    s = b.sorted()
    assert sorted((x[0], x[1]) for x in s) == [(0, 1), (0, 2)]
    assert all(x[2] == 1 for x in s)


def test_add_to_pos_at_bucket_zero_does_not_touch_predecessor():
    b = O.Buckets(100)
    b.set_halflen(10)
    b.add_to_pos(5, 5, 0, 1, 0, 1, 5, 5)
    s = b.sorted()
    assert len(s) == 1 and (s[0][0], s[0][1]) == (0, 0)


def test_get_sorted_buckets_dedups_and_orders_by_matches_descending():
    b = O.Buckets(200)
    b.set_halflen(10)
    b.add_to_pos(50, 50, 0, 1, 0, 1, 50, 50)
    b.add_to_pos(51, 51, 0, 1, 0, 1, 51, 51)
    b.add_to_pos(150, 150, 0, 1, 0, 1, 150, 150)
    s = b.sorted()
    assert s[0][2] >= s[-1][2]
    locs = [(x[0], x[1]) for x in s]
    assert len(set(locs)) == len(locs)
    # matches descending, ties by (segm_id, b) ascending (buckets.rs:697-704)
    assert [(-x[2], x[0], x[1]) for x in s] == sorted((-x[2], x[0], x[1]) for x in s)


def test_clear_resets_touched_buckets():
    b = O.Buckets(100)
    b.set_halflen(10)
    b.add_to_pos(25, 25, 0, 1, 0, 1, 25, 25)
    assert b.sorted()
    b.clear()
    assert not b.sorted()


def test_abs_pos_flag_selects_r_vs_tpos_for_bucket_index():
    bt = O.Buckets(1000)
    ba = O.Buckets(1000, ap=True)
    bt.set_halflen(10)
    ba.set_halflen(10)
    bt.add_to_pos(99, 3, 0, 1, 0, 1, 99, 99)  # r = 99 -> bucket 9; tpos = 3 -> bucket 0
    ba.add_to_pos(99, 3, 0, 1, 0, 1, 99, 99)
    assert (0, 0) in [(x[0], x[1]) for x in bt.sorted()]
    assert (0, 9) in [(x[0], x[1]) for x in ba.sorted()]


def test_dense_and_sparse_paths_agree():
    sparse = O.Buckets(1 << 30, n_kmers=0, ap=True)  # the slot count passes the dense cap
    dense = O.Buckets(4000, ap=True)
    assert sparse.set_halflen(10) and dense.set_halflen(10)
    assert not sparse.dense_on and dense.dense_on
    for span in (3900, 150):
        sparse.clear()
        dense.clear()
        assert sparse.set_halflen(10) and dense.set_halflen(10)
        rng = 0x9E3779B97F4A7C15
        for _ in range(5000):
            rng = (rng * 6364136223846793005 + 1) & 0xFFFFFFFFFFFFFFFF
            r = (rng >> 33) % span
            cd = 1 if r % 3 == 0 else -1
            sparse.add_to_pos(r, r, 0, 1, 0, cd, r, r)
            dense.add_to_pos(r, r, 0, 1, 0, cd, r, r)
        sparse.propagate()
        dense.propagate()
        a, b = sparse.sorted(), dense.sorted()
        assert a and a == b, span


def test_an_abandoned_read_does_not_leak_into_the_next_dense_read():
    b = O.Buckets(1 << 24, n_kmers=0, ap=True)
    b.clear()
    assert b.set_halflen(10) and b.dense_on
    b.add_to_pos(500, 500, 0, 1, 0, 1, 500, 500)  # added to, never extracted
    b.clear()
    assert b.set_halflen(5) and not b.dense_on  # over the dense cap
    b.propagate()
    assert not b.sorted()
    b.clear()
    assert b.set_halflen(10) and b.dense_on
    b.add_to_pos(500, 500, 0, 1, 0, 1, 500, 500)
    b.propagate()
    out = b.sorted()
    assert len(out) == 2 and all(x[2] == 1 for x in out)


def test_bucket_content_add_assign_merges_ranges_and_sums():
    """src/types.rs:329-339, through the accumulator: two contents in one bucket."""
    b = O.Buckets(100)
    b.set_halflen(10)
    b.add_to_pos(12, 12, 0, 2, 1, 1, 10, 20)
    b.add_to_pos(15, 15, 0, 3, 2, -1, 5, 15)
    b.propagate()
    for seg, bb, matches, codir, rmin, rmax in b.sorted():  # bucket 1 and its predecessor 0
        assert (matches, codir, rmin, rmax) == (5, 0, 5, 20)


# ---------------------------------------------------------------- mapping.rs:445-495
def test_update_only_overwrites_on_improvement():
    m = O.Mapping()
    assert m.state()[0] == -1.0
    m.update(0, 9, 100, 200, 0, 1000, 5, 0.5, 3, 101)
    assert m.state() == (0.5, 100, "+")
    m.update(0, 9, 300, 400, 0, 1000, 2, 0.2, -1, 101)  # worse: ignored
    assert m.state() == (0.5, 100, "+")
    m.update(0, 9, 300, 400, 0, 1000, 8, 0.9, -1, 101)  # better: overwrites
    assert m.state() == (0.9, 300, "-")


def test_overlap_disjoint_segments_is_negative_zero():
    import math

    a, b = O.Mapping(), O.Mapping()
    a.update(0, 9, 0, 100, 0, 1000, 5, 0.5, 1, 101)
    b.update(0, 9, 0, 100, 1, 1000, 5, 0.5, 1, 101)
    ov = O.Mapping.overlap(a, b)
    assert ov == 0.0 and math.copysign(1.0, ov) == -1.0


def test_overlap_same_segment_fraction():
    a, b = O.Mapping(), O.Mapping()
    a.update(0, 9, 0, 100, 0, 1000, 5, 0.5, 1, 101)
    b.update(0, 9, 50, 150, 0, 1000, 5, 0.5, 1, 101)
    assert abs(O.Mapping.overlap(a, b) - 50.0 / 150.0) < 1e-9


def test_calc_mapq_uses_integer_division_for_strand_check():
    m = O.Mapping()
    m.update(0, 9, 0, 100, 0, 1000, 5, 0.9, 3, 101)  # intersection 5: 5 / 2 == 2; |3| is not < 2
    assert m.calc_mapq(0.5, 0.02) in (60, 0)
    assert m.calc_mapq(0.5, 0.02) == 60  # frac = 1 - 0.5 / 0.9 > 0.02


# ---------------------------------------------------------------- seeding.rs:221-245
def test_unique_elements_groups_by_hash_and_collects_pmatches():
    p = [(60, 0x111111, False), (70, 0x222222, False), (10, 0x111111, True), (20, 0x222222, True),
         (30, 0x111111, True), (40, 0x444444, False), (50, 0x555555, False)]
    seeds = O.seed_groups(p)
    got = {tuple(pm) for _, _, pm in seeds}
    assert got == {(60, 30, 10), (70, 20), (40,), (50,)}
    assert sorted(occ for _, occ, _ in seeds) == [1, 1, 2, 3]


# ---------------------------------------------------------------- io/mod.rs:435-580
def _synthetic_fasta(n_segments, seed):
    """The reference test's generator (src/io/mod.rs:457-482), restated: names,
    lengths and line widths from its LCG, bases (i * 7 + s) % 4 of ACGT."""
    state = seed

    def rnd():
        nonlocal state
        state = (state * 6364136223846793005 + 1442695040888963407) & 0xFFFFFFFFFFFFFFFF
        return state >> 33

    text, expect = bytearray(), []
    for s in range(n_segments):
        name = f"chr{s}_" + "x" * (rnd() % 40)
        length = 1 + rnd() % 900
        width = 1 + rnd() % 97
        seq = bytes(b"ACGT"[(i * 7 + s) % 4] for i in range(length))
        text += f">{name} some description here\n".encode()
        for j in range(0, length, width):
            text += seq[j:j + width] + b"\n"
        expect.append((name, seq))
    return bytes(text), expect


def _readers(tmp_path, data):
    from shmap_b200 import fasta

    p = tmp_path / "t.fa"
    p.write_bytes(data)
    return fasta.read_fastx(str(p)), O.read_fasta(str(p))


def test_reads_records_and_truncates_id_at_whitespace(tmp_path):
    for got in _readers(tmp_path, b">read1 some description\nACGT\n>read2\nGGGG\n"):
        assert got == [("read1", b"ACGT"), ("read2", b"GGGG")]


def test_crlf_and_a_missing_final_newline(tmp_path):
    for got in _readers(tmp_path, b">a desc\r\nACGT\r\nGGTT\r\n>b\r\nTTTT"):
        assert got == [("a", b"ACGTGGTT"), ("b", b"TTTT")]


def test_synthetic_files_of_the_reference(tmp_path):
    for n, seed in ((24, 0xC0FFEE), (6, 42)):
        data, expect = _synthetic_fasta(n, seed)
        for got in _readers(tmp_path, data):
            assert got == expect, (n, seed)


# ---------------------------------------------------------------- shmap/mod.rs:1033-1047
def test_all_eight_const_generic_combinations_run():
    """Every (NBP, OS, AP) combination, under every metric, maps the golden
    fixture's reads, and the same call twice gives the same records."""
    import itertools
    import os

    from helpers import pack
    from shmap_b200 import fasta

    here = os.path.join(os.path.dirname(__file__), "golden")
    refs = fasta.read_fastx(os.path.join(here, "tiny_ref.fa"))
    reads = fasta.read_fastx(os.path.join(here, "tiny_reads.fa"))
    idx = O.Index.from_records(refs, 8, 1.0)
    seq, offs = pack([s for _, s in reads])
    for nbp, os_, ap in itertools.product((False, True), repeat=3):
        for metric in ("Containment", "Jaccard", "bucket_SH", "bucket_LCS"):
            p = O.params(k=8, h_frac=1.0, theta=0.1, metric=metric, no_bucket_pruning=nbp, one_sweep=os_,
                         abs_pos=ap)
            a = idx.map_reads(p, seq, offs)
            b = idx.map_reads(p, seq, offs, threads=3)
            assert a.tobytes() == b.tobytes(), (nbp, os_, ap, metric)
            assert (a["status"] == 0).any(), (nbp, os_, ap, metric)
    # the reference test's own inputs: a tandem ACGT reference and reads
    tand = O.Index.from_records([("ref", b"ACGT" * 50)], 8, 1.0)
    tseq, toffs = pack([b"ACGT" * 14, b"CGTA" * 14])
    for nbp, os_, ap in itertools.product((False, True), repeat=3):
        for metric in ("Containment", "Jaccard", "bucket_SH", "bucket_LCS"):
            p = O.params(k=8, h_frac=1.0, theta=0.1, metric=metric, no_bucket_pruning=nbp, one_sweep=os_,
                         abs_pos=ap)
            assert tand.map_reads(p, tseq, toffs).tobytes() == tand.map_reads(p, tseq, toffs, threads=2).tobytes()
