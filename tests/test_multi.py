"""shm_map_multi: one read set over several device contexts, each with its own
index replica, mapped at the same time and merged in read order. This run has
one GPU, so the replicas are two contexts on device 0 (their work is
independent: nothing waits on the other); the records must equal a
single-context call, shares must cover the reads in order, and a context
given twice or an index on another context's device is refused."""
import numpy as np
import pytest

import shmap_b200 as sb
from helpers import record_mismatches
from shmap_b200 import synth

pytestmark = pytest.mark.gpu


def test_shares_over_two_replicas_equal_one_call(gpu_ctx):
    gen = synth.Genome(synth.REFS["uniform5m"])
    names, seq, offs = gen.reads(synth.scaled(synth.READS["fixed10k"], 1.5))
    p = sb.Params(k=25, h_frac=0.01, theta=0.4)
    g0 = sb.SketchIndex.from_records(gpu_ctx, gen.records(), 25, 0.01)
    want = g0.map_reads(p, seq, offs)
    c1 = sb.Context(0)
    g1 = sb.SketchIndex.from_records(c1, gen.records(), 25, 0.01)
    for k in (1, 2):
        got, shares = sb.map_reads_multi([g0, g1][:k], p, seq, offs)
        assert not record_mismatches(got, want)
        assert shares.sum() == len(names) and (shares > 0).all()
    got, shares = sb.map_reads_multi([g0, g1], p, seq[: offs[3]], offs[:4])
    assert not record_mismatches(got, want[:3]) and shares.sum() == 3
    with pytest.raises(sb.ShmError):
        sb.map_reads_multi([g0, g0], p, seq, offs)
    g1.close()
    c1.close()
