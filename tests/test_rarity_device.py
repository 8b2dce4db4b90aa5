"""The rarity flags on the device (--rarity-weight, --rarity-tiebreak,
--rarity-alpha; src/params.rs:76-112, src/shmap/mod.rs:694-723,
src/shmap/scoring.rs:214-281, 409-481) against the CPU oracle, record for
record (the f64 support is a running sum in the reference's order, so the
scores and the tie-break decisions must be bit-exact) and PAF line for line:
a repeat-rich reference where near-equal copies compete, the human-like
genome at 1% scale, Containment and Jaccard, the bucket metric (no support:
the band only lowers the admission bar), absolute positions, no pruning.
CPU: the validation messages of the flags (src/params.rs:223-242)."""
import numpy as np
import pytest

import oracle as O
import shmap_b200 as sb
from helpers import pack, record_mismatches, strip_t
from shmap_b200 import synth
from test_oracle_golden import _rarity_workload


def test_flag_validation():
    p = sb.Params(k=15, h_frac=0.1, rarity_weight=5.0)
    with pytest.raises(sb.ShmError) as e:
        p.validate()
    assert "The rarity weight (--rarity-weight) should be between 0 and 4. You provided 5." in str(e.value)
    p = sb.Params(k=15, h_frac=0.1, rarity_weight=1.0, metric="Jaccard")
    with pytest.raises(sb.ShmError) as e:
        p.validate()
    assert "--rarity-weight is only defined for -m Containment (got Jaccard)." in str(e.value)
    sb.Params(k=15, h_frac=0.1, rarity_tiebreak=0.05, rarity_alpha=3.0, metric="Jaccard").validate()


def _compare(g, o, names, seq, offs, **kw):
    gp, op = sb.Params(**kw), O.params(**kw)
    rec = g.map_reads(gp, seq, offs)
    want = o.map_reads(op, seq, offs, threads=8)
    mm = record_mismatches(rec, want)
    assert not mm, (kw, mm)
    text, rec2 = g.map_paf(gp, seq, offs, names)
    assert rec2.tobytes() == rec.tobytes()
    assert strip_t(text) == strip_t(o.paf(op, seq, offs, names, threads=8))
    return rec


CASES = [dict(rarity_weight=1.0), dict(rarity_weight=0.5, rarity_alpha=2.0), dict(rarity_tiebreak=0.01),
         dict(rarity_tiebreak=0.05, rarity_alpha=0.5), dict(rarity_tiebreak=0.2, rarity_alpha=2.0),
         dict(rarity_weight=1.0, rarity_tiebreak=0.02), dict(rarity_tiebreak=0.05, metric="Jaccard"),
         dict(rarity_tiebreak=0.05, metric="bucket_SH"), dict(rarity_weight=0.5, abs_pos=True, theta=0.05),
         dict(rarity_tiebreak=0.03, no_bucket_pruning=True), dict(rarity_weight=1.0, one_sweep=True)]


@pytest.mark.gpu
@pytest.mark.parametrize("kw", CASES)
def test_rarity_on_repeats(gpu_ctx, kw):
    _, ref_rep, reads = _rarity_workload()
    g = sb.SketchIndex.from_records(gpu_ctx, [("r", ref_rep)], 15, 0.2)
    o = O.Index.from_records([("r", ref_rep)], 15, 0.2, threads=4)
    seq, offs = pack(reads)
    names = [f"q{i}" for i in range(len(reads))]
    rec = _compare(g, o, names, seq, offs, **{"k": 15, "h_frac": 0.2, "theta": 0.3, **kw})
    # under -F the windows are read lengths of bases: few reads reach -t there
    assert (rec["status"] == 0).mean() > (0.0 if kw.get("abs_pos") else 0.5)


@pytest.mark.gpu
@pytest.mark.parametrize("kw", [dict(rarity_weight=1.0), dict(rarity_tiebreak=0.02),
                                dict(rarity_tiebreak=0.05, rarity_alpha=2.0, metric="Jaccard")])
def test_rarity_human_like(gpu_ctx, kw):
    gen = synth.Genome(synth.scaled(synth.REFS["human31"], 0.01))
    names, seq, offs = gen.reads(synth.scaled(synth.READS["dense"], 400 / synth.READS["dense"].n_reads))
    g = sb.SketchIndex(gpu_ctx, gen.names, gen.seq, gen.seg_off, 25, 0.05)
    o = O.Index(gen.names, gen.seq, gen.seg_off, 25, 0.05, threads=8)
    rec = _compare(g, o, names, seq, offs, k=25, h_frac=0.05, theta=0.4, **kw)
    assert (rec["status"] == 0).mean() > 0.5
