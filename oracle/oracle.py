"""TEST INFRASTRUCTURE ONLY: ctypes wrapper of the CPU oracle (liboracle.so).

Only tests/, __graft_entry__.smoke() and bench.py's CPU baseline use this, as
the checker. It restates shmap-rs's mapping path sequentially in C++ (see
oracle.hpp); the product never imports it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from typing import Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
CLI = os.path.join(HERE, "shmap_oracle")

METRICS = {"Containment": 0, "Jaccard": 1, "bucket_SH": 2, "bucket_LCS": 3}


def build() -> None:
    subprocess.run(["make", "-s", "-C", HERE], check=True)


class OParams(ctypes.Structure):
    _fields_ = [("k", ctypes.c_int32), ("h_frac", ctypes.c_double), ("max_matches", ctypes.c_int32),
                ("theta", ctypes.c_double), ("min_diff", ctypes.c_double), ("max_overlap", ctypes.c_double),
                ("metric", ctypes.c_int32), ("no_bucket_pruning", ctypes.c_int32), ("one_sweep", ctypes.c_int32),
                ("abs_pos", ctypes.c_int32), ("rarity_weight", ctypes.c_double), ("rarity_tiebreak", ctypes.c_double),
                ("rarity_alpha", ctypes.c_double)]


RECORD_DTYPE = np.dtype(
    [("score", "<f8"), ("sh", "<f8"), ("score2", "<f8")]
    + [(n, "<i4") for n in (
        "status", "read_len", "sketch_size", "seeds", "p_start", "p_end", "segm_id", "t_l", "t_r",
        "same_strand", "intersection", "s_sz", "bucket_seg", "bucket_b", "has_second", "intersection2",
        "bucket2_seg", "bucket2_b", "total_matches", "max_seed_matches", "seed_matches",
        "seeded_buckets", "final_buckets", "reserved")],
    align=True,
)

_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = ctypes.CDLL(LIB)
        P, i32, i64, u64, dbl = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_uint64, ctypes.c_double
        for name, res, args in [
            ("orc_sketch", i64, [P, i64, i32, dbl, i32, P, P, P, i64]),
            ("orc_h_thres", u64, [i32, dbl]),
            ("orc_lcs", i32, [P, P, i32, i32, i32, P, P, P, i32]),
            ("orc_buckets_new", P, [i32, i32, i32]),
            ("orc_buckets_free", None, [P]),
            ("orc_buckets_set_halflen", i32, [P, i32]),
            ("orc_buckets_dense_on", i32, [P]),
            ("orc_buckets_begin", i32, [P, i32, i32]),
            ("orc_buckets_end", i32, [P, i32, i32]),
            ("orc_buckets_add_to_pos", None, [P, i32, i32, i32, i32, i32, i32, i32, i32]),
            ("orc_buckets_propagate", None, [P]),
            ("orc_buckets_clear", None, [P]),
            ("orc_buckets_sorted", i64, [P, P, i64]),
            ("orc_mapping_new", P, []),
            ("orc_mapping_free", None, [P]),
            ("orc_mapping_update", None, [P, i32, i32, i32, i32, i32, i32, i32, dbl, i32, i32]),
            ("orc_mapping_get", None, [P, P, P, P]),
            ("orc_mapping_overlap", dbl, [P, P]),
            ("orc_mapping_calc_mapq", i32, [P, dbl, dbl]),
            ("orc_seed_groups", i64, [P, P, P, i32, P, P, P, P]),
            ("orc_read_fasta", i32, [ctypes.c_char_p, P, P, P, P, P, P]),
            ("orc_index_build", P, [P, P, i32, ctypes.c_char_p, i32, dbl, i32, i32]),
            ("orc_index_free", None, [P]),
            ("orc_index_stats", None, [P, P]),
            ("orc_index_count", None, [P, P, i64, P]),
            ("orc_index_hits", i64, [P, u64, P, P, P, P, i64]),
            ("orc_segment_sketch", i64, [P, i32, P, P, P, i64]),
            ("orc_map", i32, [P, P, P, P, i32, i32, P]),
            ("orc_paf", i64, [P, P, P, P, ctypes.c_char_p, i32, i32, P, i64]),
            ("orc_time_map", dbl, [P, P, P, P, i32, i32]),
            ("orc_map_paf", dbl, [P, P, P, P, ctypes.c_char_p, i32, i32, P, P]),
            ("orc_take_text", i64, [P, i64]),
        ]:
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _p(a: np.ndarray) -> int:
    return a.ctypes.data if a.size else 0


def params(k=15, h_frac=0.05, max_matches=None, theta=0.9, min_diff=0.02, max_overlap=0.5, metric="Containment",
           no_bucket_pruning=False, one_sweep=False, abs_pos=False, rarity_weight=0.0, rarity_tiebreak=0.0,
           rarity_alpha=0.0) -> OParams:
    return OParams(k, h_frac, -1 if max_matches is None else max_matches, theta, min_diff, max_overlap,
                   METRICS[metric], int(no_bucket_pruning), int(one_sweep), int(abs_pos), rarity_weight,
                   rarity_tiebreak, rarity_alpha)


def sketch(seq: bytes, k: int, h_frac: float, offset: int = 0):
    buf = np.frombuffer(seq, np.uint8)
    cap = max(0, len(seq) - k + 1)
    r = np.zeros(cap, np.int32)
    h = np.zeros(cap, np.uint64)
    st = np.zeros(cap, np.uint8)
    n = lib().orc_sketch(_p(buf), len(seq), k, h_frac, offset, _p(r), _p(h), _p(st), cap)
    return r[:n], h[:n], st[:n]


def lcs(t, bgn: int, end: int, seeds) -> int:
    """bucket_LCS's count over window [bgn, end) of the sketch t = [(r, h), ...]
    for a read whose seeds are {hash: [positions, in pmatches order]}."""
    t_r = np.array([r for r, _ in t], np.int32)
    t_h = np.array([h for _, h in t], np.uint64)
    sh = np.array(list(seeds), np.uint64)
    lens = [len(v) for v in seeds.values()]
    off = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    pos = np.array([x for v in seeds.values() for x in v] + [0], np.int32)
    return int(lib().orc_lcs(_p(t_r), _p(t_h), len(t), bgn, end, _p(sh), _p(off), _p(pos), len(sh)))


class Buckets:
    """The bucket accumulator (src/buckets.rs:305-724) over one segment 'seg0'
    of sz bases holding n_kmers k-mers (test hook)."""

    def __init__(self, sz: int, n_kmers: Optional[int] = None, ap: bool = False):
        self.h = lib().orc_buckets_new(sz, sz if n_kmers is None else n_kmers, int(ap))

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_buckets_free(self.h)

    def set_halflen(self, h: int) -> bool:
        return bool(lib().orc_buckets_set_halflen(self.h, h))

    @property
    def dense_on(self) -> bool:
        return bool(lib().orc_buckets_dense_on(self.h))

    def begin(self, segm: int, b: int) -> int:
        return lib().orc_buckets_begin(self.h, segm, b)

    def end(self, segm: int, b: int) -> int:
        return lib().orc_buckets_end(self.h, segm, b)

    def add_to_pos(self, r: int, tpos: int, segm: int, matches: int, seeds: int, codir: int, rmin: int, rmax: int):
        lib().orc_buckets_add_to_pos(self.h, r, tpos, segm, matches, seeds, codir, rmin, rmax)

    def propagate(self):
        lib().orc_buckets_propagate(self.h)

    def clear(self):
        lib().orc_buckets_clear(self.h)

    def sorted(self):
        """[(segm_id, b, matches, codirection, r_min, r_max)] in get_sorted_buckets order."""
        n = lib().orc_buckets_sorted(self.h, None, 0)
        out = np.zeros(6 * max(n, 1), np.int32)
        lib().orc_buckets_sorted(self.h, _p(out), n)
        return [tuple(int(x) for x in out[6 * i:6 * i + 6]) for i in range(n)]


class Mapping:
    """A Mapping (src/mapping.rs:299-420) driven directly (test hook)."""

    def __init__(self):
        self.h = lib().orc_mapping_new()

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_mapping_free(self.h)

    def update(self, p_start, p_end, t_l, t_r, seg_id, seg_sz, intersection, score, same_strand, sz):
        lib().orc_mapping_update(self.h, p_start, p_end, t_l, t_r, seg_id, seg_sz, intersection, score,
                                 same_strand, sz)

    def state(self):
        sc, tl, st = ctypes.c_double(), ctypes.c_int32(), ctypes.c_char()
        lib().orc_mapping_get(self.h, ctypes.byref(sc), ctypes.byref(tl), ctypes.byref(st))
        return sc.value, tl.value, st.value.decode()

    @staticmethod
    def overlap(a: "Mapping", b: "Mapping") -> float:
        return lib().orc_mapping_overlap(a.h, b.h)

    def calc_mapq(self, theta2: float, min_diff: float) -> int:
        return lib().orc_mapping_calc_mapq(self.h, theta2, min_diff)


def seed_groups(kmers):
    """unique_elements_with_info (src/shmap/seeding.rs:26-77) of [(r, h, strand)]
    against an empty index: [(hash, occurrences, pmatches)] in seed order."""
    n = len(kmers)
    r = np.array([k[0] for k in kmers], np.int32)
    h = np.array([k[1] for k in kmers], np.uint64)
    st = np.array([int(k[2]) for k in kmers], np.uint8)
    oh = np.zeros(max(n, 1), np.uint64)
    occ = np.zeros(max(n, 1), np.int32)
    off = np.zeros(n + 1, np.int32)
    pm = np.zeros(max(n, 1), np.int32)
    m = lib().orc_seed_groups(_p(r), _p(h), _p(st), n, _p(oh), _p(occ), _p(off), _p(pm))
    return [(int(oh[i]), int(occ[i]), [int(x) for x in pm[off[i]:off[i + 1]]]) for i in range(m)]


def read_fasta(path: str):
    """The oracle's read_fasta (src/io/mod.rs:383-427): [(name, bases)]."""
    n, nb, sb_ = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
    if lib().orc_read_fasta(os.fsencode(path), ctypes.byref(n), ctypes.byref(nb), ctypes.byref(sb_), None, None,
                            None) != 0:
        raise ValueError(f"invalid FASTA record in {path}")
    names = ctypes.create_string_buffer(nb.value + 1)
    seq = np.zeros(max(sb_.value, 1), np.uint8)
    offs = np.zeros(n.value + 1, np.int64)
    lib().orc_read_fasta(os.fsencode(path), ctypes.byref(n), ctypes.byref(nb), ctypes.byref(sb_), names, _p(seq),
                         _p(offs))
    nm = names.raw[:nb.value].decode().split("\n") if n.value else []
    return [(nm[i], seq[offs[i]:offs[i + 1]].tobytes()) for i in range(n.value)]


def h_thres(h_frac: float, k: int = 15) -> int:
    return int(lib().orc_h_thres(k, h_frac))


class Index:
    STATS = ("segments", "total_nucls", "indexed_hits", "indexed_kmers", "highest_freq_kmer",
             "blacklisted_kmers", "blacklisted_hits", "sketched_kmers")

    def __init__(self, names: Sequence[str], seq: np.ndarray, seg_off: np.ndarray, k: int, h_frac: float,
                 max_matches: Optional[int] = None, threads: int = 1):
        self.seq = np.ascontiguousarray(seq, np.uint8)
        self.seg_off = np.ascontiguousarray(seg_off, np.int64)
        self.names = list(names)
        self.h = lib().orc_index_build(_p(self.seq), _p(self.seg_off), len(self.names),
                                       "\n".join(self.names).encode(), k, h_frac,
                                       -1 if max_matches is None else max_matches, threads)

    @classmethod
    def from_records(cls, records, k, h_frac, max_matches=None, threads=1):
        seqs = [s for _, s in records]
        off = np.zeros(len(seqs) + 1, np.int64)
        off[1:] = np.cumsum([len(s) for s in seqs])
        buf = np.frombuffer(b"".join(seqs), np.uint8) if seqs else np.zeros(0, np.uint8)
        return cls([n for n, _ in records], buf, off, k, h_frac, max_matches, threads)

    def __del__(self):
        try:
            lib().orc_index_free(self.h)
        except Exception:
            pass

    def stats(self) -> dict:
        out = np.zeros(8, np.int64)
        lib().orc_index_stats(self.h, _p(out))
        return dict(zip(self.STATS, (int(x) for x in out)))

    def count(self, hashes) -> np.ndarray:
        hashes = np.ascontiguousarray(hashes, np.uint64)
        out = np.zeros(len(hashes), np.int32)
        lib().orc_index_count(self.h, _p(hashes), len(hashes), _p(out))
        return out

    def hits(self, h: int):
        n = lib().orc_index_hits(self.h, h, 0, 0, 0, 0, 0)
        seg, tpos, r = (np.zeros(n, np.int32) for _ in range(3))
        st = np.zeros(n, np.uint8)
        lib().orc_index_hits(self.h, h, _p(seg), _p(tpos), _p(r), _p(st), n)
        return seg, tpos, r, st

    def segment(self, i: int):
        n = lib().orc_segment_sketch(self.h, i, 0, 0, 0, 0)
        r = np.zeros(n, np.int32)
        h = np.zeros(n, np.uint64)
        st = np.zeros(n, np.uint8)
        lib().orc_segment_sketch(self.h, i, _p(r), _p(h), _p(st), n)
        return r, h, st

    def map_reads(self, p: OParams, seq: np.ndarray, offs: np.ndarray, threads: int = 1) -> np.ndarray:
        seq = np.ascontiguousarray(seq, np.uint8)
        offs = np.ascontiguousarray(offs, np.int64)
        out = np.zeros(len(offs) - 1, RECORD_DTYPE)
        lib().orc_map(self.h, ctypes.byref(p), _p(seq), _p(offs), len(offs) - 1, threads, _p(out))
        return out

    def paf(self, p: OParams, seq: np.ndarray, offs: np.ndarray, names: Sequence[str], threads: int = 1) -> str:
        seq = np.ascontiguousarray(seq, np.uint8)
        offs = np.ascontiguousarray(offs, np.int64)
        joined = "\n".join(names).encode()
        n = lib().orc_paf(self.h, ctypes.byref(p), _p(seq), _p(offs), joined, len(offs) - 1, threads, 0, 0)
        buf = ctypes.create_string_buffer(n + 1)
        lib().orc_paf(self.h, ctypes.byref(p), _p(seq), _p(offs), joined, len(offs) - 1, threads, buf, n)
        return buf.raw[:n].decode()

    def map_paf(self, p: OParams, seq: np.ndarray, offs: np.ndarray, names: Sequence[str], threads: int,
                records: bool = True):
        """Maps the reads with `threads` host threads and renders their PAF text
        in input order (t:f: as 0): (records or None, text bytes, seconds of
        mapping and rendering)."""
        seq = np.ascontiguousarray(seq, np.uint8)
        offs = np.ascontiguousarray(offs, np.int64)
        n = len(offs) - 1
        out = np.zeros(n, RECORD_DTYPE) if records else None
        tl = ctypes.c_int64()
        joined = "\n".join(names).encode()
        secs = lib().orc_map_paf(self.h, ctypes.byref(p), _p(seq), _p(offs), joined, n, threads,
                                 _p(out) if records else None, ctypes.byref(tl))
        buf = np.empty(max(tl.value, 1), np.uint8)
        lib().orc_take_text(_p(buf), tl.value)
        return out, buf[:tl.value].tobytes(), float(secs)

    def time_map(self, p: OParams, seq: np.ndarray, offs: np.ndarray, threads: int) -> float:
        seq = np.ascontiguousarray(seq, np.uint8)
        offs = np.ascontiguousarray(offs, np.int64)
        return float(lib().orc_time_map(self.h, ctypes.byref(p), _p(seq), _p(offs), len(offs) - 1, threads))


def run_cli(args: Sequence[str]) -> subprocess.CompletedProcess:
    if not os.path.exists(CLI):
        build()
    return subprocess.run([CLI, *args], capture_output=True, text=True)
