"""The measured launch and batch shapes (shm_tuning_*): every setting reads
back what was set, values out of range and unknown keys are refused, a
settings file is read with its comments and refused (nothing changed) when a
line is malformed. The settings change how work is cut, never a result: the
GPU test maps one read set under very different settings and compares."""
import ctypes

import numpy as np
import pytest

import shmap_b200 as sb

KEYS = ["dev_batch_reads", "dev_batch_bases", "dev_first_batch_reads", "host_batch_reads", "host_batch_bases",
        "host_first_batch_reads", "sketch_ctas_per_sm", "wide_ctas_per_sm", "refine_warps_per_sm", "device_pack",
        "host_raw_share", "bt_fast_slots", "host_pack_task_kib", "host_stream", "host_stream_bases",
        "host_stream_chunk_kib", "host_stream_first_kib", "host_stream_piece_kib", "host_stream_ring",
        "host_stream_last_kib", "host_stream_raw_share", "plan_mapped"]


def _get(k):
    v = ctypes.c_int64()
    assert sb.lib().shm_tuning_get(k.encode(), ctypes.byref(v)) == 0
    return v.value


@pytest.fixture
def saved():
    before = {k: _get(k) for k in KEYS}
    yield before
    for k, v in before.items():
        assert sb.lib().shm_tuning_set(k.encode(), v) == 0


def test_get_set_and_ranges(saved):
    L = sb.lib()
    assert all(v >= 0 for v in saved.values())
    assert L.shm_tuning_set(b"sketch_ctas_per_sm", 3) == 0 and _get("sketch_ctas_per_sm") == 3
    assert L.shm_tuning_set(b"sketch_ctas_per_sm", 0) == sb.SHM_ERR_INVALID
    assert L.shm_tuning_set(b"sketch_ctas_per_sm", 99) == sb.SHM_ERR_INVALID
    assert _get("sketch_ctas_per_sm") == 3
    assert L.shm_tuning_set(b"no_such_knob", 1) == sb.SHM_ERR_INVALID
    assert b"unknown tuning setting" in L.shm_last_error()
    assert isinstance(L.shm_tuning_source(), bytes)


def test_settings_file(saved, tmp_path):
    L = sb.lib()
    good = tmp_path / "t.conf"
    good.write_text("# measured\nwide_ctas_per_sm = 4   # contrib\n\nhost_batch_reads=20000\n")
    assert L.shm_tuning_load(str(good).encode()) == 0
    assert _get("wide_ctas_per_sm") == 4 and _get("host_batch_reads") == 20000
    assert L.shm_tuning_source() == str(good).encode()
    bad = tmp_path / "b.conf"
    bad.write_text("wide_ctas_per_sm = 2\nbogus line\n")
    assert L.shm_tuning_load(str(bad).encode()) == sb.SHM_ERR_INVALID
    assert b"not a 'key = value' line" in L.shm_last_error()
    assert _get("wide_ctas_per_sm") == 4  # nothing of a refused file applies
    (tmp_path / "c.conf").write_text("refine_warps_per_sm = 1000\n")
    assert L.shm_tuning_load(str(tmp_path / "c.conf").encode()) == sb.SHM_ERR_INVALID


@pytest.mark.gpu
def test_results_do_not_depend_on_the_settings(gpu_ctx, saved):
    from helpers import record_mismatches
    from shmap_b200 import synth

    gen = synth.Genome(synth.REFS["uniform5m"])
    names, seq, offs = gen.reads(synth.READS["fixed10k"])
    g = sb.SketchIndex.from_records(gpu_ctx, gen.records(), 25, 0.01)
    p = sb.Params(k=25, h_frac=0.01, theta=0.4)
    want = g.map_reads(p, seq, offs)
    L = sb.lib()
    for k, v in [("dev_batch_reads", 1024), ("dev_first_batch_reads", 64), ("host_batch_reads", 1024),
                 ("host_first_batch_reads", 100), ("sketch_ctas_per_sm", 1), ("wide_ctas_per_sm", 1),
                 ("refine_warps_per_sm", 8), ("device_pack", 1), ("bt_fast_slots", 16), ("plan_mapped", 1)]:
        assert L.shm_tuning_set(k.encode(), v) == 0
    got = g.map_reads(p, seq, offs)
    assert not record_mismatches(got, want)
    import torch

    d_seq = torch.zeros(len(seq) + 32, dtype=torch.uint8, device="cuda")
    d_seq[: len(seq)].copy_(torch.from_numpy(np.ascontiguousarray(seq)))
    d_out = torch.empty(len(names) * sb.RECORD_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
    g.map_reads_device(p, d_seq.data_ptr(), offs, d_out.data_ptr())
    torch.cuda.synchronize()
    assert not record_mismatches(d_out.cpu().numpy().view(sb.RECORD_DTYPE), want)
    # reads in pinned host memory, a share of the batches sent up as ASCII
    pin = torch.zeros(len(seq) + 32, dtype=torch.uint8).pin_memory()
    pin[: len(seq)].copy_(torch.from_numpy(np.ascontiguousarray(seq)))
    offs64 = np.ascontiguousarray(offs, dtype=np.int64)
    cp = p.c()
    for share in (40, 100):
        assert L.shm_tuning_set(b"host_raw_share", share) == 0
        out = np.zeros(len(names), sb.RECORD_DTYPE)
        sb._check(L.shm_map_batch(gpu_ctx.h, g.h, ctypes.byref(cp), pin.data_ptr(), offs64.ctypes.data, len(names),
                                  out.ctypes.data))
        assert not record_mismatches(out, want), share
    # about 20 batches of 1 MiB: a third or two thirds of them sent up as bytes beside the packed
    # ones (raw batches in a row, each raw buffer reused), packing cut into tasks of 1 KiB to 64 KiB
    assert L.shm_tuning_set(b"host_batch_bases", 1 << 20) == 0
    for share, task_kib in ((34, 1), (67, 0), (0, 64)):
        assert L.shm_tuning_set(b"host_raw_share", share) == 0
        assert L.shm_tuning_set(b"host_pack_task_kib", task_kib) == 0
        out = np.zeros(len(names), sb.RECORD_DTYPE)
        sb._check(L.shm_map_batch(gpu_ctx.h, g.h, ctypes.byref(cp), pin.data_ptr(), offs64.ctypes.data, len(names),
                                  out.ctypes.data))
        assert not record_mismatches(out, want), (share, task_kib)
    # one packing stream a call: in parts of 16 MiB (two parts), chunks of 256 KiB (more chunks than
    # mask-list slots), device batches from 256 KiB up and back down; with the defaults; pieces sent
    # by the packing threads (64 KiB pieces, two buffers a thread; and the defaults); and the
    # batch-by-batch form
    assert L.shm_tuning_set(b"host_raw_share", 0) == 0
    # (and with a third or all of the pieces sent up as bytes, packed on the device)
    for stream, bases, chunk, first, task, raw in ((1, 1 << 24, 256, 256, 64, 0), (1, 1 << 32, 32768, 32768, 256, 0),
                                                   (2, 1 << 24, 256, 256, 64, 0), (2, 1 << 32, 32768, 32768, 2048, 0),
                                                   (2, 1 << 24, 256, 256, 64, 34), (2, 1 << 32, 32768, 32768, 64, 100),
                                                   (0, 1 << 32, 32768, 32768, 256, 0)):
        for k, x in (("host_stream", stream), ("host_stream_bases", bases), ("host_stream_chunk_kib", chunk),
                     ("host_stream_raw_share", raw),
                     ("host_stream_first_kib", first), ("host_stream_last_kib", first), ("host_pack_task_kib", task),
                     ("host_stream_piece_kib", task), ("host_stream_ring", 2 if task == 64 else 4)):
            assert L.shm_tuning_set(k.encode(), x) == 0
        out = np.zeros(len(names), sb.RECORD_DTYPE)
        sb._check(L.shm_map_batch(gpu_ctx.h, g.h, ctypes.byref(cp), pin.data_ptr(), offs64.ctypes.data, len(names),
                                  out.ctypes.data))
        assert not record_mismatches(out, want), (stream, bases, chunk, first, task, raw)
