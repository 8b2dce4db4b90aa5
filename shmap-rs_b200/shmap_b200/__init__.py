"""Python binding of the B200 mapping path (ctypes over lib/libshmapgpu.so).

The library is the product: CUDA kernels for sm_100a behind the C ABI of
include/shmap_gpu.h. This module only marshals arguments; it never computes a
mapping itself, and it raises if the library is missing instead of falling
back to anything.

The API mirrors the reference crate's entry points for this path:
``FracMinHash.sketch`` (src/sketch.rs), ``SketchIndex.build_index`` /
``count`` (src/index.rs), ``Mapper.map_reads`` (src/mapper.rs,
src/shmap/mod.rs) and the PAF writer (src/mapping.rs).
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

PKG_ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_DIR = os.path.join(PKG_ROOT, "lib")
LIB_PATH = os.path.join(LIB_DIR, "libshmapgpu.so")
SYNTH_PATH = os.path.join(LIB_DIR, "libshmapsynth.so")
CLI_PATH = os.path.join(PKG_ROOT, "bin", "shmap")

SHM_OK = 0
SHM_ERR_INVALID, SHM_ERR_CUDA, SHM_ERR_NOMEM, SHM_ERR_CAPACITY, SHM_ERR_TIMEOUT = -1, -2, -3, -4, -5
CONTAINMENT, JACCARD, BUCKET_SH, BUCKET_LCS = 0, 1, 2, 3
METRICS = {"Containment": CONTAINMENT, "Jaccard": JACCARD, "bucket_SH": BUCKET_SH, "bucket_LCS": BUCKET_LCS}

# shm_map_record (include/shmap_gpu.h)
RECORD_DTYPE = np.dtype(
    [("score", "<f8"), ("sh", "<f8"), ("score2", "<f8")]
    + [(n, "<i4") for n in (
        "status", "read_len", "sketch_size", "seeds", "p_start", "p_end", "segm_id", "t_l", "t_r",
        "same_strand", "intersection", "s_sz", "bucket_seg", "bucket_b", "has_second", "intersection2",
        "bucket2_seg", "bucket2_b", "total_matches", "max_seed_matches", "seed_matches",
        "seeded_buckets", "final_buckets", "reserved")],
    align=True,
)
assert RECORD_DTYPE.itemsize == 120  # sizeof(shm_map_record)


class ShmError(RuntimeError):
    """A non-zero status from the C ABI, with the library's message."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"shmap-b200 error {code}: {msg}")
        self.code = code


class CParams(ctypes.Structure):
    _fields_ = [("k", ctypes.c_int32), ("h_frac", ctypes.c_double), ("max_matches", ctypes.c_int32),
                ("theta", ctypes.c_double), ("min_diff", ctypes.c_double), ("max_overlap", ctypes.c_double),
                ("metric", ctypes.c_int32), ("no_bucket_pruning", ctypes.c_int32), ("one_sweep", ctypes.c_int32),
                ("abs_pos", ctypes.c_int32), ("rarity_weight", ctypes.c_double), ("rarity_tiebreak", ctypes.c_double),
                ("rarity_alpha", ctypes.c_double)]


class CServerConfig(ctypes.Structure):
    _fields_ = [("slots", ctypes.c_int32), ("max_batch_reads", ctypes.c_int32), ("max_batch_bases", ctypes.c_int64),
                ("hbm_budget", ctypes.c_size_t)]


class CRequestStats(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int32), ("reads", ctypes.c_int32), ("batch_reads", ctypes.c_int32),
                ("batch_requests", ctypes.c_int32), ("queued_ms", ctypes.c_double), ("mapped_ms", ctypes.c_double),
                ("total_ms", ctypes.c_double)]


class CIndexStats(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int64) for n in (
        "segments", "total_nucls", "indexed_hits", "indexed_kmers", "highest_freq_kmer",
        "blacklisted_kmers", "blacklisted_hits", "sketched_kmers")]


_lib = None


def lib() -> ctypes.CDLL:
    """Loads libshmapgpu.so (raises if it was not built: there is no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing; build it with `make -C {PKG_ROOT}`")
    L = ctypes.CDLL(LIB_PATH)
    P, i32, i64, u64, dbl, sz = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_uint64, ctypes.c_double, ctypes.c_size_t
    sig = {
        "shm_last_error": (ctypes.c_char_p, []),
        "shm_params_default": (None, [P]),
        "shm_params_validate": (ctypes.c_int, [P]),
        "shm_h_thres": (u64, [dbl]),
        "shm_ctx_create": (ctypes.c_int, [ctypes.c_int, sz, P]),
        "shm_ctx_destroy": (ctypes.c_int, [P]),
        "shm_ctx_launches": (i64, [P]),
        "shm_sketch": (ctypes.c_int, [P, P, i64, i32, dbl, i32, P, P, P, i64, P]),
        "shm_index_build": (ctypes.c_int, [P, P, P, i32, ctypes.c_char_p, i32, dbl, i32, P]),
        "shm_index_destroy": (ctypes.c_int, [P]),
        "shm_index_save": (ctypes.c_int, [P, ctypes.c_char_p]),
        "shm_index_load": (ctypes.c_int, [P, ctypes.c_char_p, P]),
        "shm_index_info": (ctypes.c_int, [P, P, P, P]),
        "shm_index_file_check": (ctypes.c_int, [ctypes.c_char_p]),
        "shm_tuning_get": (ctypes.c_int, [ctypes.c_char_p, P]),
        "shm_tuning_set": (ctypes.c_int, [ctypes.c_char_p, i64]),
        "shm_tuning_load": (ctypes.c_int, [ctypes.c_char_p]),
        "shm_tuning_source": (ctypes.c_char_p, []),
        "shm_index_stats_get": (ctypes.c_int, [P, P]),
        "shm_index_count": (ctypes.c_int, [P, P, P, i64, P]),
        "shm_index_hits": (ctypes.c_int, [P, P, u64, P, P, P, P, i64, P]),
        "shm_index_segment": (ctypes.c_int, [P, P, i32, P, P, P, i64, P, ctypes.c_char_p, i32, P]),
        "shm_map_batch": (ctypes.c_int, [P, P, P, P, P, i32, P]),
        "shm_map_plain": (ctypes.c_int, [P, P, P, P, P, i32, P]),
        "shm_map_multi": (ctypes.c_int, [P, P, i32, P, P, P, i32, P, P]),
        "shm_map_batch_device": (ctypes.c_int, [P, P, P, P, P, P, i32, P]),
        "shm_map_paf": (ctypes.c_int, [P, P, P, P, P, i32, ctypes.c_char_p, P, P, i64, P]),
        "shm_format_paf": (ctypes.c_int, [P, P, P, i32, ctypes.c_char_p, P, P, i64, P]),
        "shm_ctx_stream": (P, [P]),
        "shm_ctx_set_timing": (ctypes.c_int, [P, ctypes.c_int]),
        "shm_ctx_stage_times": (ctypes.c_int, [P, P, P, ctypes.c_int]),
        "shm_stage_name": (ctypes.c_char_p, [ctypes.c_int]),
        "shm_ctx_work_stats": (ctypes.c_int, [P, P, ctypes.c_int]),
        "shm_work_stat_name": (ctypes.c_char_p, [ctypes.c_int]),
        "shm_sketch_device_noalloc": (ctypes.c_int, [P, i64, i32, dbl, i32, P, P, i64, P, P]),
        "shm_format_paf_device": (ctypes.c_int, [P, P, P, P, i32, ctypes.c_char_p, P, P, i64, P]),
        "shm_fasta_parse_device": (ctypes.c_int, [P, P, i64, P]),
        "shm_fasta_records": (ctypes.c_int, [P, P, P, P]),
        "shm_fasta_copy_seq": (ctypes.c_int, [P, P]),
        "shm_fasta_destroy": (ctypes.c_int, [P]),
        "shm_index_build_fasta": (ctypes.c_int, [P, P, i32, dbl, i32, P]),
        "shm_map_fasta": (ctypes.c_int, [P, P, P, P, i32, i32, P]),
        "shm_server_config_default": (None, [P]),
        "shm_server_create": (ctypes.c_int, [P, P, P, P, P]),
        "shm_submit": (ctypes.c_int, [P, P, P, i32, P, P]),
        "shm_poll": (ctypes.c_int, [P, u64, i32, P]),
        "shm_server_destroy": (ctypes.c_int, [P]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def _check(rc: int) -> None:
    if rc != SHM_OK:
        raise ShmError(rc, lib().shm_last_error().decode(errors="replace"))


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data if a.size else 0


@dataclass
class Params:
    """The CLI parameters the mapping path reads (src/params.rs:20-186)."""
    k: int = 15
    h_frac: float = 0.05
    max_matches: Optional[int] = None
    theta: float = 0.9
    min_diff: float = 0.02
    max_overlap: float = 0.5
    metric: str = "Containment"
    no_bucket_pruning: bool = False
    one_sweep: bool = False
    abs_pos: bool = False
    rarity_weight: float = 0.0
    rarity_tiebreak: float = 0.0
    rarity_alpha: float = 0.0

    def c(self) -> CParams:
        if self.metric not in METRICS:
            raise ValueError(f"metric {self.metric!r} is not on the device path")
        return CParams(self.k, self.h_frac, -1 if self.max_matches is None else self.max_matches, self.theta,
                       self.min_diff, self.max_overlap, METRICS[self.metric], int(self.no_bucket_pruning),
                       int(self.one_sweep), int(self.abs_pos), self.rarity_weight, self.rarity_tiebreak,
                       self.rarity_alpha)

    def validate(self) -> None:
        """Params::validate (src/params.rs:191-263); raises ShmError with the reference's message."""
        cp = self.c()
        _check(lib().shm_params_validate(ctypes.byref(cp)))


def h_thres(h_frac: float) -> int:
    return int(lib().shm_h_thres(h_frac))


def pack(seqs: Sequence[bytes]) -> tuple[np.ndarray, np.ndarray]:
    """Concatenates sequences into (bytes, offsets[n+1])."""
    offs = np.zeros(len(seqs) + 1, dtype=np.int64)
    if seqs:
        offs[1:] = np.cumsum([len(s) for s in seqs])
    buf = np.frombuffer(b"".join(seqs), dtype=np.uint8) if seqs else np.zeros(0, np.uint8)
    return np.ascontiguousarray(buf), offs


class Context:
    """A device context (one GPU, one stream, grow-only scratch)."""

    def __init__(self, device: int = 0, hbm_budget: int = 0):
        h = ctypes.c_void_p()
        _check(lib().shm_ctx_create(device, hbm_budget, ctypes.byref(h)))
        self.h = h

    def close(self) -> None:
        if self.h:
            lib().shm_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def launches(self) -> int:
        return int(lib().shm_ctx_launches(self.h))

    @property
    def stream(self) -> int:
        """The cudaStream_t (as an int) every call of this context runs on."""
        return int(lib().shm_ctx_stream(self.h) or 0)

    def set_timing(self, on: bool) -> None:
        _check(lib().shm_ctx_set_timing(self.h, int(on)))

    def stage_times(self) -> dict:
        """{stage: (milliseconds, timed launches)} accumulated since timing was switched on."""
        ms = np.zeros(16, np.float64)
        cnt = np.zeros(16, np.int64)
        n = lib().shm_ctx_stage_times(self.h, _ptr(ms), _ptr(cnt), 16)
        return {lib().shm_stage_name(i).decode(): (float(ms[i]), int(cnt[i])) for i in range(n)}

    def work_stats(self) -> dict:
        """Work counters of every mapping call since the last reset (set_timing(False))."""
        out = np.zeros(32, np.int64)
        n = lib().shm_ctx_work_stats(self.h, _ptr(out), 32)
        return {lib().shm_work_stat_name(i).decode(): int(out[i]) for i in range(n)}

    def sketch(self, seq: bytes, k: int, h_frac: float, offset: int = 0):
        """FracMinHash::sketch_slice_into: arrays (r, h, strand) in sequence order."""
        buf = np.frombuffer(seq, dtype=np.uint8)
        cap = max(0, len(seq) - k + 1)
        r = np.zeros(cap, np.int32)
        h = np.zeros(cap, np.uint64)
        st = np.zeros(cap, np.uint8)
        n = ctypes.c_int64()
        _check(lib().shm_sketch(self.h, _ptr(buf), len(seq), k, h_frac, offset, _ptr(r), _ptr(h), _ptr(st), cap,
                                ctypes.byref(n)))
        return r[:n.value], h[:n.value], st[:n.value]


class SketchIndex:
    """The reference index on the device (SketchIndex, src/index.rs)."""

    def __init__(self, ctx: Context, names: Sequence[str], seq: np.ndarray, seg_off: np.ndarray, k: int,
                 h_frac: float, max_matches: Optional[int] = None):
        self.ctx = ctx
        self.names = list(names)
        self.k, self.h_frac = k, h_frac
        seq = np.ascontiguousarray(seq, dtype=np.uint8)
        seg_off = np.ascontiguousarray(seg_off, dtype=np.int64)
        h = ctypes.c_void_p()
        joined = "\n".join(self.names).encode()
        _check(lib().shm_index_build(ctx.h, _ptr(seq), _ptr(seg_off), len(self.names), joined, k, h_frac,
                                     -1 if max_matches is None else max_matches, ctypes.byref(h)))
        self.h = h

    @classmethod
    def from_records(cls, ctx: Context, records: Sequence[tuple[str, bytes]], k: int, h_frac: float,
                     max_matches: Optional[int] = None) -> "SketchIndex":
        seq, off = pack([s for _, s in records])
        return cls(ctx, [n for n, _ in records], seq, off, k, h_frac, max_matches)

    @classmethod
    def from_device_fasta(cls, ctx: Context, fa: "DeviceFasta", k: int, h_frac: float,
                          max_matches: Optional[int] = None) -> "SketchIndex":
        """The index of a FASTA parsed on the device (shm_index_build_fasta)."""
        obj = cls.__new__(cls)
        obj.ctx = ctx
        obj.h = None
        obj.names = list(fa.names)
        obj.k, obj.h_frac = k, h_frac
        h = ctypes.c_void_p()
        _check(lib().shm_index_build_fasta(ctx.h, fa.h, k, h_frac, -1 if max_matches is None else max_matches,
                                           ctypes.byref(h)))
        obj.h = h
        return obj

    def map_device_fasta(self, params: Params, fa: "DeviceFasta", first: int = 0,
                         n: Optional[int] = None) -> np.ndarray:
        """Records of reads [first, first + n) of a FASTA parsed on the device (shm_map_fasta)."""
        n = fa.n - first if n is None else n
        out = np.zeros(n, RECORD_DTYPE)
        cp = params.c()
        _check(lib().shm_map_fasta(self.ctx.h, self.h, ctypes.byref(cp), fa.h, first, n, _ptr(out)))
        return out

    def save(self, path: str) -> None:
        """Writes the index to a file (shm_index_save)."""
        _check(lib().shm_index_save(self.h, os.fsencode(path)))

    @classmethod
    def load(cls, ctx: Context, path: str) -> "SketchIndex":
        """Reads an index written by save onto ctx's device (shm_index_load)."""
        obj = cls.__new__(cls)
        obj.ctx = ctx
        obj.h = None
        h = ctypes.c_void_p()
        _check(lib().shm_index_load(ctx.h, os.fsencode(path), ctypes.byref(h)))
        obj.h = h
        k, hf, mm = ctypes.c_int32(), ctypes.c_double(), ctypes.c_int32()
        _check(lib().shm_index_info(h, ctypes.byref(k), ctypes.byref(hf), ctypes.byref(mm)))
        obj.k, obj.h_frac = k.value, hf.value
        # the segment names, from the file's header (layout in shm_index.cu)
        with open(path, "rb") as f:
            head = f.read(8 + 4 + 4 + 8 + 4 + 4 + 12 + 64)
            n_seg = int(np.frombuffer(head, np.int32, 1, 28)[0])
            names = []
            for _ in range(n_seg):
                ln = int(np.frombuffer(f.read(4), np.uint32)[0])
                names.append(f.read(ln).decode())
                f.read(4)
        obj.names = names
        return obj

    def close(self) -> None:
        if self.h:
            lib().shm_index_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def stats(self) -> dict:
        st = CIndexStats()
        _check(lib().shm_index_stats_get(self.h, ctypes.byref(st)))
        return {n: getattr(st, n) for n, _ in CIndexStats._fields_}

    def count(self, hashes: np.ndarray) -> np.ndarray:
        """SketchIndex::count for every hash."""
        hashes = np.ascontiguousarray(hashes, dtype=np.uint64)
        out = np.zeros(len(hashes), np.int32)
        _check(lib().shm_index_count(self.ctx.h, self.h, _ptr(hashes), len(hashes), _ptr(out)))
        return out

    def hits(self, h: int):
        """The hit list of a hash in (segm_id, r) order: arrays (segm_id, tpos, r, strand)."""
        n = ctypes.c_int64()
        lib().shm_index_hits(self.ctx.h, self.h, h, 0, 0, 0, 0, 0, ctypes.byref(n))
        cap = n.value
        seg, tpos, r = (np.zeros(cap, np.int32) for _ in range(3))
        st = np.zeros(cap, np.uint8)
        _check(lib().shm_index_hits(self.ctx.h, self.h, h, _ptr(seg), _ptr(tpos), _ptr(r), _ptr(st), cap,
                                    ctypes.byref(n)))
        return seg, tpos, r, st

    def segment(self, i: int):
        """A segment's sketch (r, h, strand), its name and length."""
        n = ctypes.c_int64()
        nm = ctypes.create_string_buffer(4096)
        ln = ctypes.c_int32()
        lib().shm_index_segment(self.ctx.h, self.h, i, 0, 0, 0, 0, ctypes.byref(n), nm, 4096, ctypes.byref(ln))
        cap = n.value
        r = np.zeros(cap, np.int32)
        h = np.zeros(cap, np.uint64)
        st = np.zeros(cap, np.uint8)
        _check(lib().shm_index_segment(self.ctx.h, self.h, i, _ptr(r), _ptr(h), _ptr(st), cap, ctypes.byref(n), nm,
                                       4096, ctypes.byref(ln)))
        return r, h, st, nm.value.decode(), ln.value

    def map_reads(self, params: Params, seq: np.ndarray, offs: np.ndarray, plain: bool = False) -> np.ndarray:
        """Mapper::map_reads for reads packed as (bytes, offsets): one record per read, in input order."""
        seq = np.ascontiguousarray(seq, dtype=np.uint8)
        offs = np.ascontiguousarray(offs, dtype=np.int64)
        n = len(offs) - 1
        out = np.zeros(n, RECORD_DTYPE)
        cp = params.c()
        f = lib().shm_map_plain if plain else lib().shm_map_batch
        _check(f(self.ctx.h, self.h, ctypes.byref(cp), _ptr(seq), _ptr(offs), n, _ptr(out)))
        return out

    def map_reads_device(self, params: Params, d_seq_ptr: int, h_offs: np.ndarray, d_out_ptr: int) -> None:
        """The device-resident form: reads and records already in device memory."""
        h_offs = np.ascontiguousarray(h_offs, dtype=np.int64)
        cp = params.c()
        _check(lib().shm_map_batch_device(self.ctx.h, self.h, ctypes.byref(cp), d_seq_ptr, 0, _ptr(h_offs),
                                          len(h_offs) - 1, d_out_ptr))

    def map_paf(self, params: Params, seq: np.ndarray, offs: np.ndarray, names: Sequence[str],
                with_records: bool = True):
        """Mapper.map_reads as the command line runs it (shm_map_paf): reads
        in, the PAF text of the mapped ones out, rendered on the device batch
        by batch (t:f: as 0). Returns (text, records or None)."""
        seq = np.ascontiguousarray(seq, dtype=np.uint8)
        offs = np.ascontiguousarray(offs, dtype=np.int64)
        n = len(offs) - 1
        joined = "\n".join(names).encode()
        out = np.zeros(n, RECORD_DTYPE) if with_records else None
        cp = params.c()
        need = ctypes.c_int64()
        cap = 640 * n + len(joined) + 1  # a line is about 480 bytes plus its names
        buf = ctypes.create_string_buffer(cap)
        rc = lib().shm_map_paf(self.ctx.h, self.h, ctypes.byref(cp), _ptr(seq), _ptr(offs), n, joined,
                               0 if out is None else _ptr(out), buf, cap, ctypes.byref(need))
        if rc == SHM_ERR_CAPACITY:
            cap = need.value + 1
            buf = ctypes.create_string_buffer(cap)
            rc = lib().shm_map_paf(self.ctx.h, self.h, ctypes.byref(cp), _ptr(seq), _ptr(offs), n, joined,
                                   0 if out is None else _ptr(out), buf, cap, ctypes.byref(need))
        _check(rc)
        return ctypes.string_at(buf, need.value).decode(), out

    def format_paf(self, params: Params, records: np.ndarray, names: Sequence[str],
                   map_time: Optional[np.ndarray] = None) -> str:
        """PAF lines of the mapped reads (src/mapping.rs Display impls)."""
        records = np.ascontiguousarray(records, dtype=RECORD_DTYPE)
        joined = "\n".join(names).encode()
        cp = params.c()
        mt = None if map_time is None else np.ascontiguousarray(map_time, dtype=np.float64)
        need = ctypes.c_int64()
        _check(lib().shm_format_paf(self.h, ctypes.byref(cp), _ptr(records), len(records), joined,
                                    0 if mt is None else _ptr(mt), 0, 0, ctypes.byref(need)))
        buf = ctypes.create_string_buffer(need.value + 1)
        _check(lib().shm_format_paf(self.h, ctypes.byref(cp), _ptr(records), len(records), joined,
                                    0 if mt is None else _ptr(mt), buf, need.value, ctypes.byref(need)))
        return buf.raw[:need.value].decode()


class DeviceFasta:
    """A FASTA file's bytes parsed on the device (shm_fasta_parse_device): the
    sequences stay in device memory; names and offsets come back."""

    def __init__(self, ctx: Context, data: bytes):
        buf = np.frombuffer(data, np.uint8)
        h = ctypes.c_void_p()
        _check(lib().shm_fasta_parse_device(ctx.h, _ptr(buf), len(buf), ctypes.byref(h)))
        self.h = h
        n = ctypes.c_int32()
        offs = ctypes.POINTER(ctypes.c_int64)()
        names = ctypes.c_char_p()
        _check(lib().shm_fasta_records(h, ctypes.byref(n), ctypes.byref(offs), ctypes.byref(names)))
        self.n = n.value
        self.offs = np.ctypeslib.as_array(offs, (self.n + 1,)).copy()
        self.names = names.value.decode(errors="replace").split("\n") if self.n else []

    def seq(self) -> np.ndarray:
        out = np.zeros(int(self.offs[-1]), np.uint8)
        if out.size:
            _check(lib().shm_fasta_copy_seq(self.h, _ptr(out)))
        return out

    def close(self) -> None:
        if self.h:
            lib().shm_fasta_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Serving with continuous batching (shm_server_create / shm_submit /
    shm_poll): the index stays resident and requests submitted from any thread
    are mapped in batches that device slots take as they free up. A request's
    arrays are kept alive here until it is polled done."""

    def __init__(self, ctx: "Context", index: "SketchIndex", params: Params, slots: int = 2,
                 max_batch_reads: int = 16384, max_batch_bases: int = 1 << 28, hbm_budget: int = 0):
        cfg = CServerConfig(slots, max_batch_reads, max_batch_bases, hbm_budget)
        self._cp = params.c()
        h = ctypes.c_void_p()
        _check(lib().shm_server_create(ctx.h, index.h, ctypes.byref(self._cp), ctypes.byref(cfg), ctypes.byref(h)))
        self.h = h
        self._live = {}

    def submit(self, seq: np.ndarray, offs: np.ndarray, out: Optional[np.ndarray] = None) -> int:
        """Queues reads (bytes and n+1 offsets, as map_reads takes them); returns a ticket."""
        seq = np.ascontiguousarray(seq, dtype=np.uint8)
        offs = np.ascontiguousarray(offs, dtype=np.int64)
        n = len(offs) - 1
        if out is None:
            out = np.zeros(n, RECORD_DTYPE)
        t = ctypes.c_uint64()
        _check(lib().shm_submit(self.h, _ptr(seq), _ptr(offs), n, _ptr(out), ctypes.byref(t)))
        self._live[t.value] = (seq, offs, out)
        return t.value

    def poll(self, ticket: int, wait_ms: int = -1):
        """(records, stats dict) once the request is done; None while it is not
        (wait_ms >= 0); raises ShmError if its batch failed."""
        st = CRequestStats()
        rc = lib().shm_poll(self.h, ticket, wait_ms, ctypes.byref(st))
        if rc == SHM_ERR_TIMEOUT:
            return None
        arrays = self._live.pop(ticket, None)
        _check(rc)
        stats = {f: getattr(st, f) for f, _ in CRequestStats._fields_}
        return arrays[2], stats

    def close(self) -> None:
        if self.h:
            _check(lib().shm_server_destroy(self.h))
            self.h = None
            self._live.clear()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def map_reads_multi(indexes: Sequence["SketchIndex"], params: Params, seq: np.ndarray, offs: np.ndarray):
    """shm_map_multi: the reads cut into contiguous shares, one per index
    replica (each on its own context's device), mapped at the same time;
    returns (records in read order, reads per share)."""
    seq = np.ascontiguousarray(seq, dtype=np.uint8)
    offs = np.ascontiguousarray(offs, dtype=np.int64)
    n = len(offs) - 1
    k = len(indexes)
    ctxs = (ctypes.c_void_p * k)(*[ix.ctx.h.value if hasattr(ix.ctx.h, "value") else ix.ctx.h for ix in indexes])
    idxs = (ctypes.c_void_p * k)(*[ix.h.value if hasattr(ix.h, "value") else ix.h for ix in indexes])
    out = np.zeros(n, RECORD_DTYPE)
    shares = np.zeros(k, np.int32)
    cp = params.c()
    _check(lib().shm_map_multi(ctxs, idxs, k, ctypes.byref(cp), _ptr(seq), _ptr(offs), n, _ptr(out),
                               _ptr(shares)))
    return out, shares


def format_paf_device(index: "SketchIndex", params: Params, records: np.ndarray, names: Sequence[str],
                      map_time: Optional[np.ndarray] = None) -> str:
    """SketchIndex.format_paf's text, rendered on the index's device (shm_format_paf_device)."""
    records = np.ascontiguousarray(records, dtype=RECORD_DTYPE)
    joined = "\n".join(names).encode()
    cp = params.c()
    mt = None if map_time is None else np.ascontiguousarray(map_time, dtype=np.float64)
    need = ctypes.c_int64()
    f = lib().shm_format_paf_device
    cap = 640 * len(records) + len(joined) + 1  # a line is about 480 bytes plus its names
    buf = ctypes.create_string_buffer(cap)
    rc = f(index.ctx.h, index.h, ctypes.byref(cp), _ptr(records), len(records), joined,
           0 if mt is None else _ptr(mt), buf, cap, ctypes.byref(need))
    if rc == SHM_ERR_CAPACITY:  # very long numbers: once more with the exact size
        cap = need.value + 1
        buf = ctypes.create_string_buffer(cap)
        rc = f(index.ctx.h, index.h, ctypes.byref(cp), _ptr(records), len(records), joined,
               0 if mt is None else _ptr(mt), buf, cap, ctypes.byref(need))
    _check(rc)
    return ctypes.string_at(buf, need.value).decode()


def strip_timing(paf: str) -> str:
    """Drops the wall-clock t:f: tag, as the reference's own golden test does (tests/golden_paf.rs:13-23)."""
    return "\n".join("\t".join(f for f in line.split("\t") if not f.startswith("t:f:"))
                     for line in paf.splitlines())


from . import synth  # noqa: E402  (seeded workloads)
from . import fasta  # noqa: E402
