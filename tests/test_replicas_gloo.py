"""The multi-GPU replica logic (shard, map, gather in order) on two CPU ranks
over gloo. The CPU oracle stands in for the per-rank mapper, so the test
checks the host logic alone: two ranks must produce exactly the records of
one process mapping everything."""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out_path):
    for p in (os.path.join(ROOT, "shmap-rs_b200"), os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")):
        sys.path.insert(0, p)
    import torch.distributed as dist

    import oracle as O
    from helpers import pack, thread_parity_workload
    from shmap_b200 import replicas

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    refs, reads = thread_parity_workload()
    idx = O.Index.from_records(refs, 12, 0.5)
    p = O.params(k=12, h_frac=0.5, theta=0.2)
    seq, offs = pack([s for _, s in reads])
    got = replicas.map_replicated(lambda s, o: idx.map_reads(p, s, o), seq, offs, rank, world)
    if rank == 0:
        np.save(out_path, got)
    dist.barrier()
    dist.destroy_process_group()


def test_shard_bounds_cover_everything_once():
    from shmap_b200 import replicas

    for n in (0, 1, 5, 76, 1001):
        for world in (1, 2, 3, 8):
            spans = [replicas.shard_bounds(n, r, world) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == n
            assert all(spans[i][1] == spans[i + 1][0] for i in range(world - 1))
            assert max(b - a for a, b in spans) - min(b - a for a, b in spans) <= 1


def test_two_gloo_ranks_equal_one_process(tmp_path):
    import oracle as O
    from helpers import pack, thread_parity_workload

    out = str(tmp_path / "rec.npy")
    port = _free_port()
    mp.start_processes(_worker, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
    got = np.load(out)
    refs, reads = thread_parity_workload()
    idx = O.Index.from_records(refs, 12, 0.5)
    seq, offs = pack([s for _, s in reads])
    want = idx.map_reads(O.params(k=12, h_frac=0.5, theta=0.2), seq, offs)
    assert got.dtype == want.dtype and np.array_equal(got.view(np.uint8), want.view(np.uint8))
