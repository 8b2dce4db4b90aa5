"""Seeded synthetic workloads with the shapes of the benchmark configurations
(lib/libshmapsynth.so does the work; every base is a pure function of the seed).

Presets (sizes as the benchmark configurations state them):
  uniform5m      4 uniform contigs, 5 Mbp; 2,000 x 10 kb reads, 1% errors 60/20/20
  human31        24 contigs of 50-250 Mbp, 3.1 Gbp, 3% tandem satellite arrays
                 (171 bp / 2 kb monomers, 1-3% copy divergence), 5% interspersed
                 6 kb repeats at 10% divergence
  hifi           150,000 lognormal(23 kb, 6 kb) reads clipped 1-60 kb, 0.5% errors 60/20/20
  ont            92,000 lognormal(24 kb, 15 kb) reads clipped 0.5-200 kb, 7% errors 40/30/30
  dense          125,000 reads of mean 15 kb, 1% errors, 20% started in satellite arrays
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, replace
from typing import List, Tuple

import numpy as np

from . import SYNTH_PATH


class RefCfg(ctypes.Structure):
    _fields_ = [("seed", ctypes.c_uint64), ("total_bases", ctypes.c_int64), ("n_contigs", ctypes.c_int32),
                ("min_contig", ctypes.c_int64), ("satellite_frac", ctypes.c_double),
                ("repeat_frac", ctypes.c_double), ("repeat_len", ctypes.c_int32), ("repeat_div", ctypes.c_double),
                ("sat_div_lo", ctypes.c_double), ("sat_div_hi", ctypes.c_double),
                ("sat_array_lo", ctypes.c_int64), ("sat_array_hi", ctypes.c_int64)]


class ReadCfg(ctypes.Structure):
    _fields_ = [("seed", ctypes.c_uint64), ("n_reads", ctypes.c_int32), ("len_mean", ctypes.c_double),
                ("len_sd", ctypes.c_double), ("len_min", ctypes.c_int64), ("len_max", ctypes.c_int64),
                ("err_rate", ctypes.c_double), ("sub_w", ctypes.c_double), ("ins_w", ctypes.c_double),
                ("del_w", ctypes.c_double), ("satellite_read_frac", ctypes.c_double)]


@dataclass
class RefSpec:
    seed: int = 1
    total_bases: int = 5_000_000
    n_contigs: int = 4
    min_contig: int = 500_000
    satellite_frac: float = 0.0
    repeat_frac: float = 0.0
    repeat_len: int = 6000
    repeat_div: float = 0.10
    sat_div_lo: float = 0.01
    sat_div_hi: float = 0.03
    sat_array_lo: int = 200_000
    sat_array_hi: int = 3_000_000


@dataclass
class ReadSpec:
    seed: int = 2
    n_reads: int = 2000
    len_mean: float = 10_000
    len_sd: float = 0.0
    len_min: int = 10_000
    len_max: int = 10_000
    err_rate: float = 0.01
    sub_w: float = 0.6
    ins_w: float = 0.2
    del_w: float = 0.2
    satellite_read_frac: float = 0.0


REFS = {
    "uniform5m": RefSpec(seed=11, total_bases=5_000_000, n_contigs=4, min_contig=500_000),
    "human31": RefSpec(seed=31, total_bases=3_100_000_000, n_contigs=24, min_contig=50_000_000,
                       satellite_frac=0.03, repeat_frac=0.05),
}
READS = {
    "fixed10k": ReadSpec(seed=12, n_reads=2000, len_mean=10_000, len_sd=0, len_min=10_000, len_max=10_000,
                         err_rate=0.01, sub_w=0.6, ins_w=0.2, del_w=0.2),
    "hifi": ReadSpec(seed=23, n_reads=150_000, len_mean=23_000, len_sd=6_000, len_min=1_000, len_max=60_000,
                     err_rate=0.005, sub_w=0.6, ins_w=0.2, del_w=0.2),
    "ont": ReadSpec(seed=24, n_reads=92_000, len_mean=24_000, len_sd=15_000, len_min=500, len_max=200_000,
                    err_rate=0.07, sub_w=0.4, ins_w=0.3, del_w=0.3),
    "dense": ReadSpec(seed=15, n_reads=125_000, len_mean=15_000, len_sd=6_000, len_min=1_000, len_max=60_000,
                      err_rate=0.01, sub_w=0.6, ins_w=0.2, del_w=0.2, satellite_read_frac=0.2),
}

_lib = None


def _synth():
    global _lib
    if _lib is None:
        if not os.path.exists(SYNTH_PATH):
            raise ImportError(f"{SYNTH_PATH} is missing; run make")
        L = ctypes.CDLL(SYNTH_PATH)
        P = ctypes.c_void_p
        for name, res, args in [
            ("synth_ref_create", P, [P]), ("synth_ref_free", None, [P]), ("synth_ref_total", ctypes.c_int64, [P]),
            ("synth_ref_nseg", ctypes.c_int32, [P]), ("synth_ref_num_sat_arrays", ctypes.c_int64, [P]),
            ("synth_ref_segments", None, [P, P, ctypes.c_char_p, ctypes.c_int64]),
            ("synth_ref_fill", None, [P, P, ctypes.c_int32]), ("synth_reads_create", P, [P, P]),
            ("synth_reads_free", None, [P]), ("synth_reads_total", ctypes.c_int64, [P, P, P, ctypes.c_int32]),
            ("synth_reads_fill", None, [P, P, P, P, P, ctypes.c_int32]),
            ("synth_read_name", None, [P, P, ctypes.c_int32, ctypes.c_char_p, ctypes.c_int32]),
        ]:
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _threads() -> int:
    return max(1, min(64, os.cpu_count() or 1))


class Genome:
    """A seeded synthetic reference: names, bases (uint8) and segment byte offsets."""

    def __init__(self, spec: RefSpec, threads: int = 0):
        L = _synth()
        self.spec = spec
        c = RefCfg(spec.seed, spec.total_bases, spec.n_contigs, spec.min_contig, spec.satellite_frac,
                   spec.repeat_frac, spec.repeat_len, spec.repeat_div, spec.sat_div_lo, spec.sat_div_hi,
                   spec.sat_array_lo, spec.sat_array_hi)
        self.h = L.synth_ref_create(ctypes.byref(c))
        n = L.synth_ref_nseg(self.h)
        self.seg_off = np.zeros(n + 1, np.int64)
        names = ctypes.create_string_buffer(64 * n + 64)
        L.synth_ref_segments(self.h, self.seg_off.ctypes.data, names, len(names))
        self.names = names.value.decode().split("\n")
        self.seq = np.empty(int(self.seg_off[-1]) + 32, np.uint8)
        L.synth_ref_fill(self.h, self.seq.ctypes.data, threads or _threads())
        self.seq = self.seq[: int(self.seg_off[-1])]

    def __del__(self):
        try:
            _synth().synth_ref_free(self.h)
        except Exception:
            pass

    def records(self) -> List[Tuple[str, bytes]]:
        return [(self.names[i], self.seq[self.seg_off[i]:self.seg_off[i + 1]].tobytes())
                for i in range(len(self.names))]

    def reads(self, spec: ReadSpec, threads: int = 0):
        """(names, bytes, offsets) of a seeded read set drawn from this genome."""
        L = _synth()
        c = ReadCfg(spec.seed, spec.n_reads, spec.len_mean, spec.len_sd, spec.len_min, spec.len_max, spec.err_rate,
                    spec.sub_w, spec.ins_w, spec.del_w, spec.satellite_read_frac)
        rs = L.synth_reads_create(self.h, ctypes.byref(c))
        try:
            t = threads or _threads()
            total = L.synth_reads_total(self.h, rs, self.seq.ctypes.data, t)
            seq = np.empty(total + 32, np.uint8)
            offs = np.zeros(spec.n_reads + 1, np.int64)
            L.synth_reads_fill(self.h, rs, self.seq.ctypes.data, seq.ctypes.data, offs.ctypes.data, t)
            nb = ctypes.create_string_buffer(128)
            names = []
            for i in range(spec.n_reads):
                L.synth_read_name(self.h, rs, i, nb, 128)
                names.append(nb.value.decode())
        finally:
            L.synth_reads_free(rs)
        return names, seq[:total], offs


def scaled(spec, factor: float, **kw):
    """A smaller version of a preset (same shape) for tests."""
    if isinstance(spec, RefSpec):
        return replace(spec, total_bases=int(spec.total_bases * factor),
                       min_contig=int(spec.min_contig * factor),
                       sat_array_lo=max(4000, int(spec.sat_array_lo * factor)),
                       sat_array_hi=max(8000, int(spec.sat_array_hi * factor)), **kw)
    return replace(spec, n_reads=max(1, int(spec.n_reads * factor)), **kw)
