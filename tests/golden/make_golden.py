"""Regenerates the committed golden fixtures of this directory from the
reference checkout (run in a container that has it; the GPU box does not).

  tiny_ref.fa, tiny_reads.fa, tiny.golden.paf
      copied verbatim from the reference's tests/fixtures/ (its golden PAF
      test, tests/golden_paf.rs:25-53, runs `-k 8 -r 1.0 -t 0.1` on them).
  known_answers.json
      the constants the reference's unit tests assert, each with the test it
      comes from, read from the test sources as text.

Usage: python tests/golden/make_golden.py /path/to/reference
"""
from __future__ import annotations

import json
import os
import re
import shutil
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def main(ref: str) -> None:
    fx = os.path.join(ref, "tests", "fixtures")
    for name in ("tiny_ref.fa", "tiny_reads.fa", "tiny.golden.paf"):
        shutil.copyfile(os.path.join(fx, name), os.path.join(HERE, name))

    idx_src = open(os.path.join(ref, "src", "index.rs")).read()
    sk_src = open(os.path.join(ref, "src", "sketch.rs")).read()

    def grab(pattern: str, text: str) -> str:
        m = re.search(pattern, text, re.S)
        if not m:
            raise SystemExit(f"pattern not found: {pattern}")
        return m.group(1)

    known = {
        "source": "shmap-rs v1.4.3 unit tests",
        "ntHash_seeds": {  # src/sketch.rs:60-63
            "A": grab(r"const A: Hash = (0x[0-9a-f_]+);", sk_src).replace("_", ""),
            "C": grab(r"const C: Hash = (0x[0-9a-f_]+);", sk_src).replace("_", ""),
            "G": grab(r"const G: Hash = (0x[0-9a-f_]+);", sk_src).replace("_", ""),
            "T": grab(r"const TN: Hash = (0x[0-9a-f_]+);", sk_src).replace("_", ""),
        },
        # src/index.rs:715-741
        "single_segment": {
            "fasta": ">ref\nACCAGTACCA\n", "k": 4, "r": 1.0,
            "counts": json.loads(grab(r"single_segment_indexing.*?let expected = (\[[0-9, ]+\]);", idx_src)),
            "indexed_hits": int(grab(r"single_segment_indexing.*?count\(\"indexed_hits\"\), (\d+)\)", idx_src)),
            "indexed_kmers": int(grab(r"single_segment_indexing.*?count\(\"indexed_kmers\"\), (\d+)\)", idx_src)),
        },
        # src/index.rs:743-769
        "two_segments": {
            "fasta": ">segm1\nACCAGTACCA\n>segm2\nGGACCA\n", "k": 4, "r": 1.0,
            "counts": json.loads(grab(r"two_segments_share.*?let expected = (\[[0-9, ]+\]);", idx_src)),
            "indexed_hits": int(grab(r"two_segments_share.*?count\(\"indexed_hits\"\), (\d+)\)", idx_src)),
            "indexed_kmers": int(grab(r"two_segments_share.*?count\(\"indexed_kmers\"\), (\d+)\)", idx_src)),
        },
        # src/index.rs:783-855: 10 segments with a shared prefix, k=6, r=1, -M 3
        "max_matches_case": {"k": 6, "r": 1.0, "max_matches": 3, "repeated": "ACGTACGTACGTACGTACGT",
                             "suffix": "TTTTGGGGCCCCAAAA"},
        # src/sketch.rs:272-296
        "rc_symmetry": {"k": 4, "s": "ACGGT", "s_rc": "ACCGT"},
        # src/sketch.rs:225-230
        "shorter_than_k": {"k": 4, "s": "ACC"},
        # tests/short_read_sketch_floor.rs
        "sketch_floor": {"k": 8, "below": [8, 9, 10, 11], "above": [12, 20, 48], "mixed": [28, 8, 28, 9, 28],
                         "mixed_mapped": 3, "seed": "0x2545F4914F6CDD1D", "ref_len": 4000,
                         "params": ["-k", "8", "-r", "1.0", "-t", "0.4", "-m", "Containment"]},
        # tests/multithreaded_parity.rs
        "thread_parity": {"k": 12, "r": 0.5, "t": 0.2, "ref_seed": 42, "ref_len": 20000, "n_mapped": 60},
        # tests/integration_paf.rs
        "integration": {"lines": 2, "target": "ref", "strand": "+", "invalid_k_message": "K-mer length"},
    }
    with open(os.path.join(HERE, "known_answers.json"), "w") as f:
        json.dump(known, f, indent=1)
        f.write("\n")
    print("wrote", sorted(os.listdir(HERE)))


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
