"""The device command line (shmap-rs_b200/bin/shmap, the reference's
src/main.rs:16-70 over the B200 path): the golden PAF of
tests/golden_paf.rs:25-53 straight from FASTA, after writing the index with
--index-out, and from that file with --index-in (whose k and -r replace the
command line's); missing arguments are refused before any device is touched."""
import os
import subprocess

import pytest

import shmap_b200 as sb
from helpers import strip_t


def _run(args):
    return subprocess.run([sb.CLI_PATH] + args, capture_output=True, text=True, timeout=300)


def _golden(golden_dir):
    return strip_t(open(os.path.join(golden_dir, "tiny.golden.paf")).read().rstrip("\n"))


@pytest.mark.parametrize("args,missing", [(["-p", "x.fa"], "--text"), (["-s", "x.fa"], "--pattern"),
                                          (["-k", "8"], "--pattern, --text"), (["--index-out", "o"], "--pattern, --text")])
def test_missing_arguments(args, missing):
    r = _run(args)
    assert r.returncode == 1
    assert r.stderr.strip() == f"ERROR: the following required arguments were not provided: {missing}"


@pytest.mark.gpu
def test_cli_golden_and_index_files(golden_dir, tmp_path):
    ref, reads = os.path.join(golden_dir, "tiny_ref.fa"), os.path.join(golden_dir, "tiny_reads.fa")
    want = _golden(golden_dir)
    r = _run(["-s", ref, "-p", reads, "-k", "8", "-r", "1.0", "-t", "0.1"])
    assert r.returncode == 0, r.stderr
    assert strip_t(r.stdout.rstrip("\n")) == want
    ix = str(tmp_path / "tiny.shmapidx")
    r = _run(["-s", ref, "-p", reads, "-k", "8", "-r", "1.0", "-t", "0.1", "--index-out", ix])
    assert r.returncode == 0, r.stderr
    assert strip_t(r.stdout.rstrip("\n")) == want and os.path.getsize(ix) > 0
    # the file's k = 8 and r = 1.0 win over the command line's
    r = _run(["--index-in", ix, "-p", reads, "-k", "15", "-r", "0.1", "-t", "0.1"])
    assert r.returncode == 0, r.stderr
    assert strip_t(r.stdout.rstrip("\n")) == want
    r = _run(["--index-in", str(tmp_path / "absent.shmapidx"), "-p", reads])
    assert r.returncode == 1 and "failed to load index from" in r.stderr
