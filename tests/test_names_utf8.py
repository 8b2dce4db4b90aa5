"""Record names as the reference turns header bytes into a String
(String::from_utf8_lossy, src/io/mod.rs:408-410): every maximal subpart of an
ill-formed UTF-8 sequence becomes one U+FFFD. The oracle's reader and the
package reader agree on headers with Latin-1 bytes, truncated and overlong
sequences and surrogates, and both equal Python's own lossy decoding; the
device parser is checked against them in test_fasta_device.py."""
import ctypes

import numpy as np
import pytest

import oracle as O
from shmap_b200 import fasta

HEADERS = [b"plain", b"caf\xe9", b"\xff\xfe", b"a\xe0\x80b", b"\xf0\x90\x80", b"\xed\xa0\x80x", b"\xc0\xaf",
           b"ok\xe2\x82\xac", b"\xf4\x90\x80\x80", b"\xe2\x82", b"tab\x85\tcomment", b"mix\xf0\x9f\x98\x80\x80"]


def _file(tmp_path):
    p = tmp_path / "names.fa"
    with open(p, "wb") as f:
        for i, h in enumerate(HEADERS):
            f.write(b">" + h + b" desc\n" + b"ACGT" * (i + 1) + b"\n")
    return str(p)


def test_oracle_and_package_readers_decode_names_lossily(tmp_path):
    p = _file(tmp_path)
    want = [h.split(b"\t")[0].decode("utf-8", errors="replace") for h in HEADERS]
    a = [n for n, _ in O.read_fasta(p)]
    b = [n for n, _ in fasta.read_fastx(p)]
    assert a == want and b == want
    rng = np.random.default_rng(4)
    for _ in range(300):
        h = bytes(rng.integers(0x21, 256, int(rng.integers(1, 12)), dtype=np.uint8))
        q = tmp_path / "r.fa"
        q.write_bytes(b">" + h + b"\nACGT\n")
        w = h.split(b" ")[0].split(b"\t")[0].decode("utf-8", errors="replace")
        assert [n for n, _ in O.read_fasta(str(q))] == [w], h


@pytest.mark.gpu
def test_device_parser_names_are_lossy_utf8(gpu_ctx, tmp_path):
    """The device FASTA parser hands back the same names, already valid UTF-8
    (strict decoding of the raw bytes succeeds)."""
    import shmap_b200 as sb

    data = open(_file(tmp_path), "rb").read()
    fa = sb.DeviceFasta(gpu_ctx, data)
    n = ctypes.c_int32()
    offs = ctypes.POINTER(ctypes.c_int64)()
    names = ctypes.c_char_p()
    assert sb.lib().shm_fasta_records(fa.h, ctypes.byref(n), ctypes.byref(offs), ctypes.byref(names)) == 0
    got = names.value.decode("utf-8").split("\n")  # strict
    assert got == [h.split(b"\t")[0].decode("utf-8", errors="replace") for h in HEADERS]
    fa.close()

