"""The project's autotuner: measures the launch and batch shapes of
shm_tuning_* on a workload and writes the settings file the library reads
(tuning.conf beside lib/, or --out).

    python -m shmap_b200.autotune [--workload hifi|ont|dense] [--scale S] [--out PATH]

One setting at a time (coordinate descent, two rounds), each candidate value
timed over a few mapping steps with CUDA events on the library's stream after
warm-up steps: the device-resident path for the device settings, the
host-buffer path (pinned reads in, records out) for the host batch settings.
Every run's records are compared with the first run's: a setting that
changed a result would be a bug, and the tuner stops on it. The chosen
values and every measurement go into the file, the measurements as comments.
"""
from __future__ import annotations

import argparse
import ctypes
import os
import statistics
import sys

import numpy as np

from . import Context, Params, RECORD_DTYPE, SketchIndex, _check, lib, synth

PRESETS = {  # reference preset, read preset, k, r, theta, metric
    "hifi": ("human31", "hifi", 25, 0.01, 0.4, "Containment"),
    "ont": ("human31", "ont", 25, 0.01, 0.1, "Containment"),
    "dense": ("human31", "dense", 25, 0.10, 0.4, "Containment"),
    "uniform": ("uniform5m", "fixed10k", 25, 0.01, 0.4, "Containment"),
}

DEVICE_KNOBS = [
    ("device_pack", [0, 1]),
    ("sketch_ctas_per_sm", [2, 4, 6, 8]),
    ("wide_ctas_per_sm", [2, 4, 6, 8]),
    ("refine_warps_per_sm", [16, 32, 48, 64]),
    ("dev_batch_reads", [16384, 32768, 65536, 131072, 262144]),
    ("dev_first_batch_reads", [1024, 4096, 16384, 65536]),
    ("bt_fast_slots", [64, 128, 256, 512]),
]
HOST_KNOBS = [
    ("host_batch_reads", [8192, 16384, 32768, 65536]),
    ("host_batch_bases", [1 << 26, 1 << 27, 1 << 28, 1 << 29]),
    ("host_first_batch_reads", [1024, 4096, 16384]),
    ("host_raw_share", [0, 10, 20, 30]),
    ("host_pack_task_kib", [0, 256, 1024, 4096]),
    ("host_stream", [0, 1, 2]),
    ("host_stream_piece_kib", [1024, 2048, 4096]),
    ("host_stream_ring", [2, 4]),
    ("host_stream_first_kib", [32768, 65536, 131072]),
    ("host_stream_last_kib", [131072, 262144, 524288]),
    ("plan_mapped", [0, 1]),
]


def get(key: str) -> int:
    v = ctypes.c_int64()
    _check(lib().shm_tuning_get(key.encode(), ctypes.byref(v)))
    return v.value


def put(key: str, value: int) -> None:
    _check(lib().shm_tuning_set(key.encode(), int(value)))


def main(argv=None) -> int:
    import torch

    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", choices=sorted(PRESETS), default="hifi")
    ap.add_argument("--scale", type=float, default=1.0)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=2)
    ap.add_argument("--rounds", type=int, default=2)
    ap.add_argument("--out", default=os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                                                  "tuning.conf"))
    a = ap.parse_args(argv)
    rp, qp, k, r, theta, metric = PRESETS[a.workload]
    rs, qs = synth.REFS[rp], synth.READS[qp]
    if a.scale != 1.0:
        rs, qs = synth.scaled(rs, a.scale), synth.scaled(qs, a.scale)
    gen = synth.Genome(rs)
    names, seq, offs = gen.reads(qs)
    ctx = Context(0)
    idx = SketchIndex(ctx, gen.names, gen.seq, gen.seg_off, k, r)
    p = Params(k=k, h_frac=r, theta=theta, metric=metric)
    n, nb = len(names), int(offs[-1])
    d_seq = torch.zeros(nb + 32, dtype=torch.uint8, device="cuda")
    d_seq[:nb].copy_(torch.from_numpy(np.ascontiguousarray(seq)))
    d_out = torch.empty(n * RECORD_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
    h_seq = torch.empty(nb + 32, dtype=torch.uint8).pin_memory()
    h_seq[:nb].copy_(torch.from_numpy(np.ascontiguousarray(seq)))
    h_seq_np = h_seq.numpy()
    h_out = torch.empty(n * RECORD_DTYPE.itemsize, dtype=torch.uint8).pin_memory().numpy().view(RECORD_DTYPE)
    stream = torch.cuda.ExternalStream(ctx.stream, device="cuda:0")
    cp = p.c()
    want = None

    def run_device():
        idx.map_reads_device(p, d_seq.data_ptr(), offs, d_out.data_ptr())

    def run_host():
        _check(lib().shm_map_batch(ctx.h, idx.h, ctypes.byref(cp), h_seq_np.ctypes.data, offs.ctypes.data, n,
                                   h_out.ctypes.data))

    def measure(fn, host: bool) -> float:
        nonlocal want
        for _ in range(a.warmup):
            fn()
        torch.cuda.synchronize()
        ts = []
        for _ in range(a.steps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn()
            e1.record(stream)
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
        rec = (h_out.copy() if host else d_out.cpu().numpy().view(RECORD_DTYPE).copy())
        if want is None:
            want = rec
        elif rec.tobytes() != want.tobytes():
            raise RuntimeError("records changed under a tuning setting")
        return statistics.median(ts)

    log = []
    for rnd in range(a.rounds):
        for knobs, fn, host in ((DEVICE_KNOBS, run_device, False), (HOST_KNOBS, run_host, True)):
            for key, values in knobs:
                res = {}
                for v in values:
                    put(key, v)
                    res[v] = measure(fn, host)
                    print(f"[autotune] round {rnd} {key}={v}: {res[v]:.3f} ms", file=sys.stderr, flush=True)
                best = min(res, key=res.get)
                put(key, best)
                log.append((rnd, key, res, best))
    keys = [k2 for k2, _ in DEVICE_KNOBS + HOST_KNOBS]
    with open(a.out, "w") as f:
        f.write("# Launch and batch shapes measured by shmap_b200.autotune (python -m shmap_b200.autotune "
                f"--workload {a.workload} --scale {a.scale:g}): {n} reads, {nb} bases, k={k} r={r} -m {metric}.\n")
        f.write("# Each value was timed (median ms a mapping step, CUDA events) with the others held; the "
                "fastest was kept.\n")
        for rnd, key, res, best in log:
            f.write(f"# round {rnd} {key}: " + ", ".join(f"{v}={ms:.3f}" for v, ms in res.items()) + "\n")
        for key in keys:
            f.write(f"{key} = {get(key)}\n")
    print(f"[autotune] wrote {a.out}", file=sys.stderr)
    idx.close()
    ctx.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
