#!/usr/bin/env python
"""Throughput of the B200 long-read mapping path (reads/s), one JSON line.

Workload (default): the human-scale HiFi-like configuration - a seeded 3.1 Gbp
synthetic reference in 24 contigs of 50-250 Mbp with 3% tandem satellite
arrays and 5% interspersed 6 kb repeats, and 150,000 lognormal(23 kb, 6 kb)
reads clipped to 1-60 kb with 0.5% errors; k=25, r=0.01, t=0.4, Containment.
A step maps every read of the workload once. The index is built on the device
before timing. Inputs (3.4 GB of reads, a 1 GB index) are larger than L2.
--workload ont / dense run the ONT-like (Containment, then Jaccard) and the
r=0.10 dense (Containment, then bucket_SH) configurations.

  value     reads/s with the reads already resident in HBM (device events,
            max over ranks)
  e2e       the same through shm_map_paf from pinned host buffers: reads in,
            PAF text out. The host->device copy of the reads and the
            device->host copy of the records and the PAF text are inside the
            timed region (e2e.records_only: shm_map_batch, records out)
  parity    every read of the workload mapped by the CPU oracle (the C++
            restatement of the reference path): its records must equal the
            device's bit for bit and its PAF text the e2e text byte for byte
            (t:f: aside); any difference ends the run with status 1
  roofline  the stage that takes the most device time, its algorithmic
            bytes per launch over its average launch time (CUDA events on the
            library's stream during the timed steps), against the measured
            HBM copy bandwidth; the sketch, bound by integer issue, also
            reports its warp-instruction issue rate against the SMs' peak
  cpu_baseline  that oracle run, every read mapped and its PAF rendered with
            every host core; cpu_baseline_1t: a bounded sample with one
            thread (the reference's -@1)

Side measurements (rank 0, outside the timed steps; a failure is reported
under its key): index_file (shm_index_save / shm_index_load of the built
index), paf_text (shm_format_paf against shm_format_paf_device on the step's
records, same bytes), fasta_parse (shm_fasta_parse_device on the first 20,000
reads as FASTA), serving (shm_server_* under Poisson arrivals: achieved
reads/s and per-read p50/p99 latency, records checked against the step's),
plain_form (one read per launch on a sample), other_metrics (the workload's
second -m, timed and checked the same way). --metric maps with another -m.

--impl reference times that CPU implementation alone (rank 0) on the same
workload, each step a bounded sample, with every host core and with one.
Multi-GPU: one process per GPU, each builds its own replica of the index and
maps its own read set (weak scaling); no collective on the data path.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import re
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "shmap-rs_b200"))

import numpy as np  # noqa: E402

# the workload's further -m, timed and checked after the first
EXTRA_METRICS = {"hifi": [], "uniform": [], "ont": ["Jaccard"], "dense": ["bucket_SH"]}

WORKLOADS = {
    # name: (reference preset, read preset, k, r, theta, metric, description)
    "hifi": ("human31", "hifi", 25, 0.01, 0.4, "Containment",
             "3.1 Gbp human-scale reference (24 contigs, 3% satellites, 5% repeats), 150,000 HiFi-like reads "
             "(lognormal 23+-6 kb, 0.5% errors), k=25 r=0.01 t=0.4 Containment"),
    "uniform": ("uniform5m", "fixed10k", 25, 0.01, 0.4, "Containment",
                "5 Mbp uniform reference in 4 contigs, 2,000 x 10 kb reads with 1% errors, k=25 r=0.01 t=0.4"),
    # at 7% errors only about 0.93^25 = 16% of a read's 25-mers survive, so no
    # read clears -t 0.4: the ONT-like workload maps at -t 0.1
    "ont": ("human31", "ont", 25, 0.01, 0.1, "Containment",
            "3.1 Gbp human-scale reference, 92,000 ONT-like reads (lognormal 24+-15 kb, 7% errors), k=25 r=0.01 "
            "t=0.1"),
    "dense": ("human31", "dense", 25, 0.10, 0.4, "Containment",
              "3.1 Gbp human-scale reference at r=0.10, 125,000 reads of 15 kb (1% errors, 20% satellite)"),
}


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def load_traffic():
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f)
    return {}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def start(self):
        """Starts sampling and returns once the first sample is written: nvidia-smi's
        own start-up stays out of the timed region."""
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                       "--format=csv,noheader,nounits", "-lms", "100"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None
            return
        t0 = time.time()
        while time.time() - t0 < 10 and self.p.poll() is None and os.path.getsize(self.f.name) == 0:
            time.sleep(0.02)

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        self.f.seek(0)
        rows = [r.split(",") for r in self.f.read().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm = [float(r[1]) for r in rows if len(r) > 8 and r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if len(r) > 8 and r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in rows:
            if len(r) > 8:
                for i, n in enumerate(names):
                    if r[5 + i].strip().lower() == "active":
                        reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(rows)}


def _extra(name: str, fn):
    """Runs one of the side measurements (index file, PAF text, FASTA parse,
    serving); a failure is reported under its key in the JSON line instead of
    ending the run."""
    try:
        return fn()
    except Exception as e:  # noqa: BLE001 - reported, not hidden
        log(f"[bench] {name} failed: {e!r}")
        return {"error": f"{type(e).__name__}: {e}"}


def make_workload(name: str, rank: int, scale: float, metric_override: str | None = None):
    from shmap_b200 import synth

    rp, qp, k, r, theta, metric, desc = WORKLOADS[name]
    if metric_override and metric_override != metric:
        desc = f"{desc}; -m {metric_override} in place of {metric}"
        metric = metric_override
    rspec = synth.REFS[rp]
    qspec = synth.READS[qp]
    if scale != 1.0:
        rspec = synth.scaled(rspec, scale)
        qspec = synth.scaled(qspec, scale)
    qspec = synth.replace(qspec, seed=qspec.seed + 1000 * rank) if rank else qspec
    t0 = time.time()
    gen = synth.Genome(rspec)
    t1 = time.time()
    names, seq, offs = gen.reads(qspec)
    t2 = time.time()
    log(f"[bench] rank {rank}: reference {len(gen.seq) / 1e9:.3f} Gbp in {t1 - t0:.1f}s, "
        f"{len(names)} reads / {len(seq) / 1e9:.3f} Gbp in {t2 - t1:.1f}s")
    return gen, names, seq, offs, dict(k=k, r=r, theta=theta, metric=metric, desc=desc)


def algorithmic_bytes(stage: str, w: dict, seq_bytes: float) -> tuple[float, str]:
    """Bytes a stage must move at the least over the counted work: its inputs
    read once and its outputs written once. seq_bytes is the reads' sum of
    ceil(L/4) + ceil(L/8) (2-bit codes and a 1-bit non-ACGT mask)."""
    if stage == "sketch":
        return (seq_bytes + 16.0 * w["kmers"],
                "sum over reads of ceil(L/4) + ceil(L/8) (2-bit codes, 1-bit non-ACGT mask) in + 16 B per "
                "selected k-mer out")
    if stage == "seedprep":
        return (16.0 * w["kmers"] + 32.0 * w["distinct_seeds"],
                "16 B per read k-mer in + 32 B (one sector) per count() probe")
    if stage in ("contrib", "extend", "bscan"):
        return (12.0 * (w["seed_hits"] + w["extension_seeds"]),
                "12 B per hit touched (match_seeds and matches_in_bucket hits)")
    if stage == "refine":
        return 12.0 * w["refine_kmers"], "12 B per reference k-mer of every refined window (8 B hash + 4 B r)"
    return 0.0, "n/a"


def packed_bytes(offs: np.ndarray) -> float:
    lens = np.diff(offs)
    return float(((lens + 3) // 4).sum() + ((lens + 7) // 8).sum())


def workload_config(args, wk: dict, n: int, nbytes: int, world: int) -> dict:
    """The config object of both arms' JSON lines (the same keys and values)."""
    return {"workload": args.workload, "description": wk["desc"], "reads_per_gpu": n, "bases_per_gpu": nbytes,
            "k": wk["k"], "r": wk["r"], "theta": wk["theta"], "metric": wk["metric"],
            "l2": "inputs larger than L2 (reads and index are GB-sized), no flush",
            "parallelism": f"replicas x{world}" if world > 1 else "1 GPU", "scale": args.scale}


def time_device(ctx, idx, p, d_seq, offs, d_out, stream, steps: int, warmup: int, world: int, local: int,
                clocks=None):
    """W untimed steps, then K steps of the device-resident path between CUDA
    events on the library's stream (barrier + synchronize on both sides; max
    over ranks). Returns (ms, launches, stage times, work counters, clocks)."""
    import torch

    def step():
        idx.map_reads_device(p, d_seq.data_ptr(), offs, d_out.data_ptr())

    for _ in range(warmup):
        step()
    torch.cuda.synchronize()
    ctx.set_timing(False)
    ctx.set_timing(True)
    if clocks:
        clocks.start()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    launches0 = ctx.launches
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(steps):
        step()
    ev1.record(stream)
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    launches = ctx.launches - launches0
    clk = clocks.stop() if clocks else None
    stages = ctx.stage_times()
    work = ctx.work_stats()
    ctx.set_timing(False)
    if world > 1:
        t = torch.tensor([ms], device=f"cuda:{local}")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms = float(t.item())
    return ms, launches, stages, work, clk


def time_e2e(ctx, idx, p, h_seq_np, offs, joined, h_out, h_text, steps: int, world: int, local: int,
             with_paf: bool = True):
    """K steps through the public C ABI from pinned host memory: shm_map_paf
    (reads in, records and PAF text out) or shm_map_batch (records out).
    Every step's host->device and device->host copies are inside the timed
    region. Returns (ms, h2d bytes per step, d2h bytes per step, text length)."""
    import torch

    import shmap_b200 as sb

    n = len(offs) - 1
    cp = p.c()
    need = ctypes.c_int64()

    def step():
        if with_paf:
            sb._check(sb.lib().shm_map_paf(ctx.h, idx.h, ctypes.byref(cp), h_seq_np.ctypes.data, offs.ctypes.data,
                                           n, joined, h_out.ctypes.data, h_text.ctypes.data, len(h_text),
                                           ctypes.byref(need)))
        else:
            sb._check(sb.lib().shm_map_batch(ctx.h, idx.h, ctypes.byref(cp), h_seq_np.ctypes.data,
                                             offs.ctypes.data, n, h_out.ctypes.data))

    step()  # grows the buffers of this call shape
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    stream = torch.cuda.ExternalStream(ctx.stream, device=f"cuda:{local}")
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    io0 = ctx.work_stats()  # bytes copied between host and device, counted by the library
    w0 = time.perf_counter()
    e0.record(stream)
    for _ in range(steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    ms = max(e0.elapsed_time(e1), (time.perf_counter() - w0) * 1e3)
    io1 = ctx.work_stats()
    h2d = (io1.get("h2d_bytes", 0) - io0.get("h2d_bytes", 0)) // max(1, steps)
    d2h = (io1.get("d2h_bytes", 0) - io0.get("d2h_bytes", 0)) // max(1, steps)
    if world > 1:
        t = torch.tensor([ms], device=f"cuda:{local}")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms = float(t.item())
    return ms, int(h2d), int(d2h), int(need.value) if with_paf else 0


_T_TAG = re.compile(rb"\tt:f:[^\t\n]*")


def oracle_check(oi, wk: dict, metric: str, names, seq, offs, rec, text: bytes, threads: int) -> tuple[dict, float]:
    """Every read mapped by the CPU oracle with `threads` host threads, its PAF
    rendered: records compared with the device's bit for bit, PAF text with
    the e2e text byte for byte (the wall-clock t:f: tag removed from both, as
    the reference's own golden test does). Returns (parity, oracle seconds)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O  # the checker, never the measured product

    op = O.params(k=wk["k"], h_frac=wk["r"], theta=wk["theta"], metric=metric)
    orec, otext, secs = oi.map_paf(op, seq, offs, names, threads)
    same_rec = orec.tobytes() == rec.tobytes()
    bad_fields, bad_reads = {}, np.zeros(len(rec), bool)
    if not same_rec:
        for f in rec.dtype.names:
            x, y = rec[f], orec[f]
            d = (x.view(np.int64) != y.view(np.int64)) if x.dtype.kind == "f" else (x != y)
            if d.any():
                bad_fields[f] = int(d.sum())
                bad_reads |= d
    a, b = _T_TAG.sub(b"", text), _T_TAG.sub(b"", otext)
    res = {"reads": int(len(rec)), "mapped": int((rec["status"] == 0).sum()),
           "record_mismatches": int(bad_reads.sum()), "mismatched_fields": bad_fields,
           "first_mismatched_reads": [int(i) for i in np.nonzero(bad_reads)[0][:5]],
           "records_equal": bool(same_rec),
           "paf_bytes": len(text), "paf_lines": text.count(b"\n"), "paf_bytes_equal": a == b,
           "against": "CPU oracle (C++ restatement of the reference path), every read of the workload; PAF "
                      "compared without the wall-clock t:f: tag"}
    return res, secs


def cpu_one_thread(oi, wk: dict, names, seq, offs, target_s: float, rate_all: float, threads_all: int) -> dict:
    """The oracle with one host thread (the reference's -@1) on a bounded
    sample of the workload's reads sized to about target_s seconds."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    op = O.params(k=wk["k"], h_frac=wk["r"], theta=wk["theta"], metric=wk["metric"])
    n = len(offs) - 1
    m = int(max(16, min(n, rate_all / max(1, threads_all) * target_s)))
    a = (n - m) // 2
    sub = offs[a:a + m + 1] - offs[a]
    _, _, secs = oi.map_paf(op, seq[offs[a]:offs[a + m]], sub, names[a:a + m], 1, records=False)
    return {"value": round(m / secs, 1), "unit": "reads/s", "cores": 1, "kind": "port",
            "sample": f"reads {a}..{a + m} of the workload's {n}, mapped and PAF rendered by the C++ oracle "
                      f"with one thread ({secs:.1f} s)"}


def oracle_index(gen, wk: dict, threads: int):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    t0 = time.time()
    oi = O.Index(gen.names, gen.seq, gen.seg_off, wk["k"], wk["r"], threads=threads)
    log(f"[bench] CPU oracle index in {time.time() - t0:.1f}s with {threads} threads")
    return oi


def run_ours(args, rank, world, local):
    import torch

    import shmap_b200 as sb

    torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    gen, names, seq, offs, wk = make_workload(args.workload, rank, args.scale, args.metric)
    ctx = sb.Context(local)
    t0 = time.time()
    idx = sb.SketchIndex(ctx, gen.names, gen.seq, gen.seg_off, wk["k"], wk["r"])
    torch.cuda.synchronize()
    index_s = time.time() - t0
    st = idx.stats()
    log(f"[bench] rank {rank}: index on device in {index_s:.2f}s: {st}")
    def _index_file():  # the index written to a file and read back (shm_index_save / shm_index_load)
        with tempfile.TemporaryDirectory() as td:
            path = os.path.join(td, "ref.shmapidx")
            t0 = time.time()
            idx.save(path)
            save_s = time.time() - t0
            t0 = time.time()
            back = sb.SketchIndex.load(ctx, path)
            torch.cuda.synchronize()
            load_s = time.time() - t0
            if back.stats() != st:
                raise RuntimeError("the index read back differs from the one built")
            res = {"bytes": os.path.getsize(path), "save_s": round(save_s, 3), "load_s": round(load_s, 3)}
            back.close()
            return res

    index_file = _extra("index_file", _index_file) if rank == 0 and args.side else None

    p = sb.Params(k=wk["k"], h_frac=wk["r"], theta=wk["theta"], metric=wk["metric"])
    n = len(names)
    nbytes = int(offs[-1])
    joined = "\n".join(names).encode()

    # device-resident inputs
    d_seq = torch.empty(nbytes + 32, dtype=torch.uint8, device=f"cuda:{local}")
    d_seq[:nbytes].copy_(torch.from_numpy(np.ascontiguousarray(seq)))
    d_seq[nbytes:].zero_()
    d_out = torch.empty(n * sb.RECORD_DTYPE.itemsize, dtype=torch.uint8, device=f"cuda:{local}")
    stream = torch.cuda.ExternalStream(ctx.stream, device=f"cuda:{local}")

    clocks = ClockSampler(local)
    ms, launches, stages, work, clk = time_device(ctx, idx, p, d_seq, offs, d_out, stream, args.steps, args.warmup,
                                                  world, local, clocks)
    rec = d_out.cpu().numpy().view(sb.RECORD_DTYPE).copy()
    mapped = float((rec["status"] == 0).mean())

    # end to end through the public C ABI, from pinned host memory: reads in, PAF text out
    h_seq = torch.empty(nbytes + 32, dtype=torch.uint8).pin_memory()
    h_seq[:nbytes].copy_(torch.from_numpy(np.ascontiguousarray(seq)))
    h_out_t = torch.empty(n * sb.RECORD_DTYPE.itemsize, dtype=torch.uint8).pin_memory()
    h_seq_np = h_seq.numpy()
    h_out = h_out_t.numpy().view(sb.RECORD_DTYPE)
    h_text = torch.empty(640 * n + len(joined) + 64, dtype=torch.uint8).pin_memory().numpy()
    e2e_ms, h2d_step, d2h_step, text_len = time_e2e(ctx, idx, p, h_seq_np, offs, joined, h_out, h_text,
                                                    args.steps, world, local, True)
    if not np.array_equal(h_out.view(np.uint8), rec.view(np.uint8)):
        raise RuntimeError("e2e records differ from the device-resident records")
    text = h_text[:text_len].tobytes()
    if rank == 0 and text != idx.format_paf(p, rec, names).encode():
        raise RuntimeError("e2e PAF text differs from the host formatter's text over the same records")
    rec_ms, rec_h2d, rec_d2h, _ = time_e2e(ctx, idx, p, h_seq_np, offs, joined, h_out, h_text, args.steps, world,
                                           local, False)
    if not np.array_equal(h_out.view(np.uint8), rec.view(np.uint8)):
        raise RuntimeError("e2e (records only) records differ from the device-resident records")

    def _paf():  # the PAF text of the step's records: shm_format_paf (host) and shm_format_paf_device
        cp = p.c()
        need = ctypes.c_int64()
        _ = sb.lib().shm_format_paf(idx.h, ctypes.byref(cp), rec.ctypes.data, n, joined, None, None, 0,
                                    ctypes.byref(need))
        cap = need.value
        buf_h = np.empty(cap, np.uint8)
        buf_d = torch.empty(cap, dtype=torch.uint8).pin_memory().numpy()
        t0 = time.perf_counter()
        sb._check(sb.lib().shm_format_paf(idx.h, ctypes.byref(cp), rec.ctypes.data, n, joined, None,
                                          buf_h.ctypes.data, cap, ctypes.byref(need)))
        t_h = time.perf_counter() - t0
        ts = []
        for _ in range(3):  # the first call grows the device buffers
            t0 = time.perf_counter()
            sb._check(sb.lib().shm_format_paf_device(ctx.h, idx.h, ctypes.byref(cp), rec.ctypes.data, n, joined,
                                                     None, buf_d.ctypes.data, cap, ctypes.byref(need)))
            ts.append(time.perf_counter() - t0)
        if not np.array_equal(buf_h, buf_d):
            raise RuntimeError("PAF text rendered on the device differs from the host's")
        res = {"bytes": cap, "lines": int((rec["status"] == 0).sum()), "host_s": round(t_h, 4),
               "device_s": round(min(ts[1:]), 4), "host_over_device": round(t_h / min(ts[1:]), 1)}
        log(f"[bench] PAF text: {res}")
        return res

    paf = _extra("paf", _paf) if rank == 0 and args.side else None

    def _fasta_parse():  # reads as FASTA bytes (pinned host memory), parsed on the device
        m = min(n, 20000)
        parts = []
        for i in range(m):
            parts.append(b">read%d\n" % i)
            parts.append(seq[offs[i]:offs[i + 1]].tobytes())
            parts.append(b"\n")
        raw = b"".join(parts)
        del parts
        pin = torch.empty(len(raw), dtype=torch.uint8).pin_memory()
        pin.copy_(torch.frombuffer(bytearray(raw), dtype=torch.uint8))
        pin_np = pin.numpy()
        sb.DeviceFasta(ctx, pin_np).close()  # warm-up
        t0 = time.perf_counter()
        fa = sb.DeviceFasta(ctx, pin_np)
        t_fa = time.perf_counter() - t0
        if fa.n != m or not np.array_equal(fa.offs, offs[: m + 1] - offs[0]):
            raise RuntimeError("reads parsed on the device differ from the workload's")
        fa.close()
        res = {"reads": m, "bytes": len(raw), "s": round(t_fa, 4), "gb_per_s": round(len(raw) / t_fa / 1e9, 1),
               "what": "shm_fasta_parse_device from pinned host memory, upload included"}
        log(f"[bench] FASTA parse: {res}")
        return res

    fasta_parse = _extra("fasta_parse", _fasta_parse) if rank == 0 and args.side else None

    def _serving():
        # the configuration's mix: HiFi-like requests from the workload's reads and
        # ONT-like ones from a second read set of the same genome
        from shmap_b200 import synth

        sets = [("hifi" if args.workload == "hifi" else args.workload, h_seq_np, offs, rec)]
        if args.workload == "hifi":
            qs = synth.READS["ont"]
            if args.scale != 1.0:
                qs = synth.scaled(qs, args.scale)
            qs = synth.scaled(qs, min(1.0, 20_000 / qs.n_reads))
            o_names, o_seq, o_offs = gen.reads(qs)
            o_h = torch.empty(int(o_offs[-1]) + 32, dtype=torch.uint8).pin_memory()
            o_h[: int(o_offs[-1])].copy_(torch.from_numpy(np.ascontiguousarray(o_seq)))
            o_h_np = o_h.numpy()
            o_rec = idx.map_reads(p, o_h_np[: int(o_offs[-1])], o_offs)
            sets.append(("ont", o_h_np, o_offs, o_rec))
        res = serve_load(ctx, idx, p, sets, [10_000, 50_000, 200_000, 1_000_000], args.serve_seconds, 11)
        log(f"[bench] serving: {res}")
        return res

    serving = _extra("serving", _serving) if rank == 0 and args.serve_seconds > 0 and args.side else None

    # plain one-read-per-launch form on a sample
    plain = None
    if rank == 0 and args.plain_sample > 0:
        m = min(n, args.plain_sample)
        sub_offs = offs[: m + 1].copy()
        sub_seq = np.ascontiguousarray(seq[: sub_offs[-1]])
        t0 = time.perf_counter()
        prec = idx.map_reads(p, sub_seq, sub_offs, plain=True)
        pt = time.perf_counter() - t0
        if not np.array_equal(prec.view(np.uint8), rec[:m].view(np.uint8)):
            raise RuntimeError("plain records differ from the batched records")
        plain = {"reads_per_s": m / pt, "sample_reads": m}

    # the workload's further metrics, timed the same way (device-resident and e2e with PAF)
    others = {}
    for om in EXTRA_METRICS.get(args.workload, []) if args.metric is None else []:
        po = sb.Params(k=wk["k"], h_frac=wk["r"], theta=wk["theta"], metric=om)
        oms, olaunch, ostages, _, _ = time_device(ctx, idx, po, d_seq, offs, d_out, stream, args.steps,
                                                  args.warmup, world, local)
        orec = d_out.cpu().numpy().view(sb.RECORD_DTYPE).copy()
        oe_ms, oh2d, od2h, olen = time_e2e(ctx, idx, po, h_seq_np, offs, joined, h_out, h_text, args.steps, world,
                                           local, True)
        if not np.array_equal(h_out.view(np.uint8), orec.view(np.uint8)):
            raise RuntimeError(f"{om}: e2e records differ from the device-resident records")
        others[om] = {"value": round(n * world * args.steps / (oms / 1e3), 1), "unit": "reads/s",
                      "ms_per_step": round(oms / args.steps, 3), "gpu_launches": int(olaunch),
                      "stages_ms": {k: round(v[0] / args.steps, 3) for k, v in ostages.items()},
                      "mapped_fraction": round(float((orec["status"] == 0).mean()), 4),
                      "e2e": {"value": round(n * world * args.steps / (oe_ms / 1e3), 1), "unit": "reads/s",
                              "ms_per_step": round(oe_ms / args.steps, 3), "h2d_bytes_per_step": oh2d,
                              "d2h_bytes_per_step": od2h},
                      "_rec": orec, "_text": h_text[:olen].tobytes()}
        log(f"[bench] -m {om}: {others[om]['value']:.0f} reads/s device-resident, "
            f"{others[om]['e2e']['value']:.0f} e2e")

    result = None
    if rank == 0:
        reads_total = n * world
        value = reads_total * args.steps / (ms / 1e3)
        mbp = float(nbytes) * world * args.steps / (ms / 1e3) / 1e6
        peak, peak_kind = load_peaks()
        traffic = load_traffic()
        top = max((s for s in stages if s != "aux"), key=lambda s: stages[s][0])
        top_ms, top_calls = stages[top]
        per_launch_s = top_ms / 1e3 / max(1, top_calls)
        alg, alg_desc = algorithmic_bytes(top, work, packed_bytes(offs) * args.steps)
        alg_per_launch = alg / max(1, top_calls)
        achieved = alg_per_launch / per_launch_s / 1e9 if per_launch_s > 0 else 0.0
        tr = None
        tinfo = traffic.get(args.workload, {}).get(top)
        if tinfo and tinfo.get("unit") in work:
            tr = round(tinfo["bytes_per_unit"] * work[tinfo["unit"]] / max(1, top_calls))
        roof = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "traffic": tr, "kernel": top,
                "peak_source": f"{peak_kind} MEASURED_PEAKS.json hbm_gbs" if peak_kind == "measured" else "fallback",
                "avg_launch_ms": round(per_launch_s * 1e3, 4), "launches": top_calls,
                "algorithmic_bytes_per_launch": round(alg_per_launch), "algorithmic_bytes": alg_desc}
        if top == "sketch":
            # integer-issue bound: warp instructions per base (ncu's smsp__inst_executed on a
            # one-kernel capture, profiles/traffic.json) times the bases of a launch, over the
            # launch time, against four warp instructions per clock on each of the 148 SMs
            ipb = traffic.get(args.workload, {}).get("sketch_warp_inst_per_base")
            mhz = (clk or {}).get("sm_mhz") or 1965.0
            roof["bound"] = "int_issue"
            if ipb:
                inst = ipb * work["bases"] / max(1, top_calls)
                ach_i = inst / per_launch_s / 1e12
                pk_i = 148 * 4 * mhz * 1e6 / 1e12
                roof["issue"] = {"achieved": round(ach_i, 4), "peak": round(pk_i, 4), "unit": "T warp-inst/s",
                                 "frac": round(ach_i / pk_i, 4), "warp_inst_per_base": ipb,
                                 "peak_def": f"148 SMs x 4 warp instructions per clock at the sampled {mhz:.0f} MHz"}
            roof["note"] = ("bound by integer instruction issue, not HBM: its HBM fraction is small by "
                            "construction; reaching 60% of HBM at this instruction count would need several "
                            "times the SMs' issue rate")
        e2e_value = reads_total * args.steps / (e2e_ms / 1e3)
        rec_value = reads_total * args.steps / (rec_ms / 1e3)
        result = {
            "metric": "reads/s (mapping, byte-identical PAF records)", "value": round(value, 1), "unit": "reads/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
            "data": "synthetic (seeded generator, shapes of the benchmark configuration)",
            "config": workload_config(args, wk, n, nbytes, world),
            "mbp_per_s": round(mbp, 1),
            "mapped_fraction": round(mapped, 4),
            "index_build_s": round(index_s, 3),
            "index_file": index_file,
            "index": st,
            "stages_ms": {k: round(v[0] / args.steps, 3) for k, v in stages.items()},
            "work_per_step": {k: v // max(1, args.steps) for k, v in work.items()},
            "roofline": roof,
            # h2d/d2h: the bytes the call copied (the reads go up packed: 2-bit codes, the nonzero
            # words of the non-ACGT mask, the batch plans, the names; records and PAF text come
            # down); ascii_gb_per_s: the reads' own bytes taken in per second
            "e2e": {"value": round(e2e_value, 1), "unit": "reads/s", "h2d_bytes_per_step": h2d_step,
                    "d2h_bytes_per_step": d2h_step, "ms_per_step": round(e2e_ms / args.steps, 3),
                    "ascii_gb_per_s": round(nbytes * args.steps / (e2e_ms / 1e3) / 1e9, 1),
                    "paf_bytes_per_step": text_len,
                    "what": "shm_map_paf: reads from pinned host memory in, records and PAF text out",
                    "records_only": {"value": round(rec_value, 1), "unit": "reads/s",
                                     "ms_per_step": round(rec_ms / args.steps, 3), "h2d_bytes_per_step": rec_h2d,
                                     "d2h_bytes_per_step": rec_d2h, "what": "shm_map_batch: records out"}},
            "gpu_launches": int(launches),
            "clocks": clk,
        }
        if serving:
            result["serving"] = serving
        if paf:
            result["paf_text"] = paf
        if fasta_parse:
            result["fasta_parse"] = fasta_parse
        if plain:
            result["plain_form"] = {"reads_per_s": round(plain["reads_per_s"], 1), "sample_reads": plain["sample_reads"],
                                    "batched_e2e_over_plain": round(e2e_value / plain["reads_per_s"], 1)}
        if others:
            result["other_metrics"] = others
    if world > 1:
        torch.distributed.barrier()
    idx.close()
    ctx.close()
    return result, (gen, names, seq, offs, wk, rec, text)



def serve_load(ctx, idx, p, sets, rates, seconds: float, seed: int):
    """Serving (shm_server_*): requests of 1-4,096 reads (uniform), each a run
    of reads of one of the read sets (HiFi-like or ONT-like, chosen at random
    per request) read in place from pinned memory, arrive as a Poisson process
    at each offered rate (reads/s) for `seconds`. Reports the achieved rate,
    the per-read latency percentiles (a read's latency is its request's,
    submit to records written), how many requests a batch carried, and
    checks every request's records against the same reads mapped alone in
    one call. sets: [(name, pinned bytes, offsets, records alone)]."""
    import threading

    import shmap_b200 as sb

    rng = np.random.default_rng(seed)
    out = []
    same = True

    def draw():
        si = int(rng.integers(0, len(sets)))
        _, _, o, _ = sets[si]
        n = len(o) - 1
        size = int(rng.integers(1, min(4096, n) + 1))
        a = int(rng.integers(0, n - size + 1))
        return si, a, size

    with sb.Server(ctx, idx, p, slots=2) as srv:
        # warm-up: full batches on both slots, so that their buffers are grown
        warm = []
        for _ in range(8):
            si = len(warm) % len(sets)
            _, hs, o, _ = sets[si]
            size = min(4096, len(o) - 1)
            warm.append(srv.submit(hs, o[:size + 1]))
        for t in warm:
            if srv.poll(t, 120_000) is None:
                raise RuntimeError("a serving warm-up request did not finish within 120 s")
        for rate in rates:
            plan, t = [], 0.0
            while True:
                t += rng.exponential(2048.5 / rate)
                if t > seconds:
                    break
                plan.append((t,) + draw())
            tickets = [None] * len(plan)
            ready = threading.Semaphore(0)

            def submitter():
                t0 = time.perf_counter()
                for i, (at, si, a, size) in enumerate(plan):
                    delay = at - (time.perf_counter() - t0)
                    if delay > 0:
                        time.sleep(delay)
                    _, hs, o, _ = sets[si]
                    tickets[i] = srv.submit(hs, o[a:a + size + 1])
                    ready.release()

            w0 = time.perf_counter()
            th = threading.Thread(target=submitter)
            th.start()
            lat, sizes, batch_req, kinds = [], [], [], []
            for i, (at, si, a, size) in enumerate(plan):
                ready.acquire()
                done = srv.poll(tickets[i], 120_000)
                if done is None:
                    raise RuntimeError("a serving request did not finish within 120 s")
                got, stt = done
                lat.append(stt["total_ms"])
                sizes.append(size)
                batch_req.append(stt["batch_requests"])
                kinds.append(si)
                if not np.array_equal(got.view(np.uint8), sets[si][3][a:a + size].view(np.uint8)):
                    same = False
            wall = time.perf_counter() - w0
            th.join()
            per_read = np.repeat(np.array(lat), np.array(sizes))
            br = np.array(batch_req)
            out.append({"offered_reads_per_s": rate, "arrived_reads_per_s": round(sum(sizes) / seconds, 1),
                        "achieved_reads_per_s": round(sum(sizes) / wall, 1),
                        "requests": len(plan), "reads": int(sum(sizes)),
                        "requests_by_kind": {sets[j][0]: int(sum(1 for x in kinds if x == j)) for j in range(len(sets))},
                        "p50_ms": round(float(np.percentile(per_read, 50)), 3),
                        "p99_ms": round(float(np.percentile(per_read, 99)), 3),
                        "mean_requests_per_batch": round(float(br.mean()), 2) if len(br) else 0.0,
                        "requests_in_merged_batches": round(float((br > 1).mean()), 3) if len(br) else 0.0})
    return {"arrivals": f"Poisson, requests of 1-4,096 reads (uniform) of one kind each "
                        f"({' or '.join(x[0] for x in sets)}, at random), {seconds:g} s per offered rate",
            "slots": 2, "rates": out, "records_same_as_alone": same}


def cpu_reference(gen, names, seq, offs, wk, target_s: float, threads: int, steps: int = 1, oi=None):
    """The CPU oracle on bounded samples, mapping and rendering PAF: returns
    (reads/s per step, sample description)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O  # the checker / CPU baseline, never the measured product

    if oi is None:
        oi = oracle_index(gen, wk, threads)
    p = O.params(k=wk["k"], h_frac=wk["r"], theta=wk["theta"], metric=wk["metric"])
    n = len(names)
    m = min(n, max(threads * 8, 256))
    _, _, t = oi.map_paf(p, seq, offs[: m + 1], names[:m], threads, records=False)
    rate = m / max(t, 1e-6)
    m = int(min(n, max(m, rate * target_s)))
    rates = []
    for s in range(steps):
        a = (s * m) % max(1, n - m + 1)
        sub = offs[a: a + m + 1] - offs[a]
        _, _, t = oi.map_paf(p, seq[offs[a]:offs[a + m]], sub, names[a:a + m], threads, records=False)
        rates.append(m / t)
    return rates, (f"{m} of the workload's {n} reads per step, mapped and PAF rendered by the C++ oracle "
                   f"with {threads} threads")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="hifi")
    ap.add_argument("--scale", type=float, default=1.0, help="shrink the workload (tests and profiling)")
    ap.add_argument("--metric", choices=["Containment", "Jaccard", "bucket_SH", "bucket_LCS"], default=None,
                    help="map with this -m instead of the workload's (its further -m are then not run)")
    ap.add_argument("--cpu-seconds", type=float, default=10.0,
                    help="one-thread CPU baseline sample size, in seconds of work")
    ap.add_argument("--plain-sample", type=int, default=400)
    ap.add_argument("--no-cpu-baseline", action="store_true",
                    help="skip the oracle runs (and with them the full-size parity check)")
    ap.add_argument("--no-side", dest="side", action="store_false",
                    help="skip the side measurements (index file, PAF formatter, FASTA, serving)")
    ap.add_argument("--serve-seconds", type=float, default=2.0,
                    help="seconds of Poisson arrivals per offered rate in the serving measurement (0 skips it)")
    args = ap.parse_args()
    rank, world, local = dist_env()
    threads = os.cpu_count() or 1

    if args.impl == "reference":
        if rank != 0:
            return
        gen, names, seq, offs, wk = make_workload(args.workload, 0, args.scale, args.metric)
        oi = oracle_index(gen, wk, threads)
        per_step = max(2.0, 150.0 / max(1, args.steps + args.warmup))
        rates, sample = cpu_reference(gen, names, seq, offs, wk, per_step, threads, steps=args.warmup + args.steps,
                                      oi=oi)
        timed = rates[args.warmup:] or rates
        v = statistics.mean(timed)
        one = cpu_one_thread(oi, wk, names, seq, offs, args.cpu_seconds, v, threads)
        line = {"metric": "reads/s (mapping, byte-identical PAF records)", "value": round(v, 1), "unit": "reads/s",
                "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": round(len(names) / v * 1e3, 3), "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "u64", "data": "synthetic (seeded generator, shapes of the benchmark "
                                                             "configuration)", "impl": "reference",
                "config": workload_config(args, wk, len(names), int(offs[-1]), args.gpus),
                "host_cores": threads,
                "cpu_baseline": {"value": round(v, 1), "unit": "reads/s", "cores": threads, "kind": "port",
                                 "sample": sample},
                "cpu_baseline_1t": one,
                "e2e": {"value": round(v, 1), "unit": "reads/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
                "note": "the reference is Rust and no Rust toolchain exists on this image; this arm times the C++ "
                        "restatement of its mapping path (oracle/), reads in and PAF text out, with every host core "
                        "(value) and with one (cpu_baseline_1t)"}
        print(json.dumps(line), flush=True)
        return

    result, data = run_ours(args, rank, world, local)
    failed = False
    if rank == 0:
        result["host_cores"] = threads
        if world == 1 and not args.no_cpu_baseline:
            gen, names, seq, offs, wk, rec, text = data
            oi = oracle_index(gen, wk, threads)
            parity, secs = oracle_check(oi, wk, wk["metric"], names, seq, offs, rec, text, threads)
            rate = len(names) / secs
            result["parity"] = parity
            result["cpu_baseline"] = {"value": round(rate, 1), "unit": "reads/s", "cores": threads, "kind": "port",
                                      "sample": f"all {len(names)} reads of the workload, mapped and PAF rendered "
                                                f"by the C++ oracle with {threads} threads ({secs:.1f} s)",
                                      "e2e_speedup": round(result["e2e"]["value"] / rate, 2)}
            result["cpu_baseline_1t"] = cpu_one_thread(oi, wk, names, seq, offs, args.cpu_seconds, rate, threads)
            result["cpu_baseline_1t"]["e2e_speedup"] = round(result["e2e"]["value"] /
                                                             result["cpu_baseline_1t"]["value"], 1)
            failed = not (parity["records_equal"] and parity["paf_bytes_equal"])
            for om, o in result.get("other_metrics", {}).items():
                par, osecs = oracle_check(oi, wk, om, names, seq, offs, o.pop("_rec"), o.pop("_text"), threads)
                o["parity"] = par
                o["cpu_baseline"] = {"value": round(len(names) / osecs, 1), "unit": "reads/s", "cores": threads,
                                     "kind": "port", "sample": f"all {len(names)} reads, oracle with {threads} threads"}
                failed = failed or not (par["records_equal"] and par["paf_bytes_equal"])
        for o in result.get("other_metrics", {}).values():
            o.pop("_rec", None)
            o.pop("_text", None)
        print(json.dumps(result), flush=True)
    if failed:
        log("[bench] PARITY FAILED: the device's records or PAF differ from the CPU oracle's")
        sys.exit(1)


if __name__ == "__main__":
    main()
