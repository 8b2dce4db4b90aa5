"""Test data generators restated from the reference's own tests, plus small
comparison helpers. Used by both the oracle tests and the GPU parity tests."""
from __future__ import annotations

import numpy as np

M64 = (1 << 64) - 1


def xorshift_dna(seed: int, n: int) -> bytes:
    """tests/multithreaded_parity.rs:14-25 (and nthash_equivalence.rs:15-26)."""
    s = seed & M64
    out = bytearray(n)
    for i in range(n):
        s ^= (s << 13) & M64
        s ^= s >> 7
        s ^= (s << 17) & M64
        out[i] = b"ACGT"[s % 4]
    return bytes(out)


def lcg_dna(seed: int, n: int) -> bytes:
    """src/sketch.rs:239-245."""
    r = seed & M64
    out = bytearray(n)
    for i in range(n):
        r = (r * 6364136223846793005 + 1) & M64
        out[i] = b"ACGT"[(r >> 60) % 4]
    return bytes(out)


def floor_reference() -> bytes:
    """tests/short_read_sketch_floor.rs:39-56: 4000 xorshift bases from 0x2545F4914F6CDD1D."""
    x = 0x2545F4914F6CDD1D
    out = bytearray()
    for _ in range(4000):
        x ^= (x << 13) & M64
        x ^= x >> 7
        x ^= (x << 17) & M64
        out.append(b"ACGT"[x % 4])
    return bytes(out)


def floor_reads(ref: bytes, lens):
    """tests/short_read_sketch_floor.rs:58-61."""
    return [(f"len{l}_{i}", ref[100 + i * 7:100 + i * 7 + l]) for i, l in enumerate(lens)]


def thread_parity_workload():
    """tests/multithreaded_parity.rs:60-82: 20 kb reference, 60 real substrings
    of varying length and 15 unrelated reads, interleaved."""
    ref = xorshift_dna(42, 20_000)
    reads = []
    for i in range(60):
        start = (i * 137) % 19_000
        ln = 200 + (i % 5) * 50
        reads.append((f"mapped_{i}", ref[start:start + ln]))
        if i % 4 == 0:
            reads.append((f"unmapped_{i}", xorshift_dna(9000 + i, 150)))
    return [("chr1", ref)], reads


def pack(seqs):
    offs = np.zeros(len(seqs) + 1, np.int64)
    if seqs:
        offs[1:] = np.cumsum([len(s) for s in seqs])
    buf = np.frombuffer(b"".join(seqs), np.uint8) if seqs else np.zeros(0, np.uint8)
    return np.ascontiguousarray(buf), offs


def strip_t(paf: str) -> str:
    """tests/golden_paf.rs:13-23."""
    return "\n".join("\t".join(f for f in ln.split("\t") if not f.startswith("t:f:")) for ln in paf.splitlines())


def nthash_direct(seq: bytes, k: int):
    """tests/nthash_equivalence.rs:31-61: per-window (fw, rc) from the definition."""
    A, C, G, T = 0x3C8BFBB395C60474, 0x3193C18562A02B4C, 0x20323ED082572324, 0x295549F54BE24456
    fwt = {ord("A"): A, ord("a"): A, ord("C"): C, ord("c"): C, ord("G"): G, ord("g"): G, ord("T"): T, ord("t"): T}
    rct = {ord("A"): T, ord("a"): T, ord("C"): G, ord("c"): G, ord("G"): C, ord("g"): C, ord("T"): A, ord("t"): A}

    def rotl(x, n):
        n &= 63
        return ((x << n) | (x >> (64 - n))) & M64 if n else x

    out = []
    for i in range(len(seq) - k + 1):
        f = r = 0
        for j in range(k):
            f ^= rotl(fwt.get(seq[i + j], 0), k - 1 - j)
            r ^= rotl(rct.get(seq[i + j], 0), j)
        out.append((f, r))
    return out


RECORD_FIELDS = ("status", "read_len", "sketch_size", "seeds", "p_start", "p_end", "segm_id", "t_l", "t_r",
                 "same_strand", "intersection", "s_sz", "bucket_seg", "bucket_b", "has_second", "intersection2",
                 "bucket2_seg", "bucket2_b", "total_matches", "max_seed_matches", "seed_matches", "seeded_buckets",
                 "final_buckets", "score", "sh", "score2")


def record_mismatches(a: np.ndarray, b: np.ndarray, limit: int = 10):
    """Field-by-field differences of two record arrays (bit-exact, floats included)."""
    out = []
    for f in RECORD_FIELDS:
        x, y = a[f], b[f]
        if x.dtype.kind == "f":
            bad = np.nonzero(x.view(np.int64) != y.view(np.int64))[0]
        else:
            bad = np.nonzero(x != y)[0]
        for i in bad[:limit]:
            out.append((int(i), f, x[i], y[i]))
    return out
