"""Index files are checked on the host before any of their arrays reaches a
device (shm_index_file_check makes the checks of shm_index_load without a
device). A file is written here in the library's format from the CPU oracle's
index of a small reference (segments, every reference k-mer, the hash CSR),
so this runs without a GPU: the library accepts it, and refuses it with
SHM_ERR_INVALID after one corrupted byte anywhere (checksum) and after each
hand-made inconsistency with a recomputed checksum: segment offsets out of
order, a hash above the threshold, a position outside its segment or out of
order, keys out of order, hit-list offsets out of order, a hit that is no
reference k-mer or out of order in its list, header counts that cannot be,
a negative segment length and a wrong byte count. The device test in
test_index_file.py loads a file from this writer and compares it with the
index built on the device."""
import struct

import numpy as np
import pytest

import oracle as O
import shmap_b200 as sb
from helpers import xorshift_dna

M64 = (1 << 64) - 1


def idx_sum(data: bytes) -> int:
    """The file's checksum: 8-byte words round-robin into four multiply-rotate
    lanes, then the tail word and the length."""
    lanes = [0x9E3779B97F4A7C15, 0xBF58476D1CE4E5B9, 0x94D049BB133111EB, 0x2545F4914F6CDD1D]
    rotl = lambda x, r: ((x << r) | (x >> (64 - r))) & M64  # noqa: E731
    words = 0

    def word(w):
        nonlocal words
        i = words & 3
        lanes[i] = (rotl(lanes[i] ^ ((w * 0xFF51AFD7ED558CCD) & M64), 29) * 0xC4CEB9FE1A85EC53) & M64
        words += 1

    n8 = len(data) // 8
    for w in np.frombuffer(data[: 8 * n8], "<u8").tolist():
        word(w)
    tail = data[8 * n8:]
    part = int.from_bytes(tail, "little") if tail else 0
    word(part ^ (len(tail) << 56))
    word(len(data))
    h = lanes[0]
    for i in range(1, 4):
        h = rotl(h, 17) ^ ((lanes[i] * 0x9E3779B97F4A7C15) & M64)
    return h ^ (h >> 31)


def index_sections(records, k, h_frac):
    """The file's sections from the oracle's index: header values, segments,
    seg_off, ref_h, ref_rs (r << 1 | strand), keys, key_off, hits."""
    o = O.Index.from_records(records, k, h_frac)
    rs, hs = [], []
    seg_off = [0]
    for i in range(len(records)):
        r, h, st = o.segment(i)
        rs.append((r.astype(np.uint32) << 1) | st.astype(np.uint32))
        hs.append(h)
        seg_off.append(seg_off[-1] + len(h))
    ref_h = np.concatenate(hs) if hs else np.zeros(0, np.uint64)
    ref_rs = np.concatenate(rs) if rs else np.zeros(0, np.uint32)
    order = np.lexsort((np.arange(len(ref_h)), ref_h))  # by hash, then by k-mer id
    keys, counts = np.unique(ref_h[order], return_counts=True)
    key_off = np.concatenate([[0], np.cumsum(counts)]).astype(np.uint32)
    st = o.stats()
    return dict(k=k, h_frac=h_frac, mm=-1, names=[n for n, _ in records], lens=[len(s) for _, s in records],
                stats=[st[n] for n in O.Index.STATS], seg_off=np.array(seg_off, np.uint32), ref_h=ref_h,
                ref_rs=ref_rs, keys=keys.astype(np.uint64), key_off=key_off, hits=order.astype(np.uint32))


def write_index(path, d, n_keys=None, fix_sum=True, count_delta=0):
    body = bytearray(b"SHMAPIX1")
    body += struct.pack("<Iidiiiii", 2, d["k"], d["h_frac"], d["mm"], len(d["names"]),
                        len(d["keys"]) if n_keys is None else n_keys, len(d["ref_h"]), len(d["hits"]))
    body += struct.pack("<8q", *d["stats"])
    for nm, ln in zip(d["names"], d["lens"]):
        b = nm.encode()
        body += struct.pack("<I", len(b)) + b + struct.pack("<i", ln)
    for key in ("seg_off", "ref_h", "ref_rs", "keys", "key_off", "hits"):
        body += np.ascontiguousarray(d[key]).tobytes()
    body = bytes(body)
    s = idx_sum(body) if fix_sum else idx_sum(body) ^ 1
    with open(path, "wb") as f:
        f.write(body + struct.pack("<QQ", len(body) + count_delta, s))


def _records():
    rep = b"ACGTACGTACGTACGTACGT"
    recs = [(f"chr{i}", xorshift_dna(100 + i, 20000 + 977 * i)) for i in range(4)]
    return recs + [("repeats", (rep + b"TTGGCCAA") * 100), ("empty", b""), ("short", b"ACG")]


def _check(path):
    rc = sb.lib().shm_index_file_check(path.encode())
    return rc, sb.lib().shm_last_error().decode()


@pytest.fixture(scope="module")
def sections():
    return index_sections(_records(), 12, 0.2)


def test_a_written_index_file_is_accepted(tmp_path, sections):
    p = str(tmp_path / "ok.shmapidx")
    write_index(p, sections)
    assert _check(p) == (0, _check(p)[1])
    assert len(sections["keys"]) > 100 and (np.diff(sections["key_off"]) > 1).any()


def _corrupt(d, what):
    d = {k: (v.copy() if isinstance(v, np.ndarray) else list(v) if isinstance(v, list) else v) for k, v in d.items()}
    kw = {}
    if what == "seg_off":
        d["seg_off"][1], d["seg_off"][2] = d["seg_off"][2], d["seg_off"][1]
    elif what == "ref_h":
        d["ref_h"][5] = np.uint64(M64)
    elif what == "ref_rs_range":
        d["ref_rs"][3] = np.uint32((d["lens"][0] + 5) << 1)
    elif what == "ref_rs_order":
        d["ref_rs"][3], d["ref_rs"][4] = d["ref_rs"][4], d["ref_rs"][3]
    elif what == "keys":
        d["keys"][7], d["keys"][8] = d["keys"][8], d["keys"][7]
    elif what == "key_off":
        d["key_off"][10] = d["key_off"][11]
    elif what == "hits_range":
        d["hits"][9] = np.uint32(len(d["ref_h"]))
    elif what == "hits_order":
        i = int(np.nonzero(np.diff(d["key_off"]) > 1)[0][0])
        a = int(d["key_off"][i])
        d["hits"][a], d["hits"][a + 1] = d["hits"][a + 1], d["hits"][a]
    elif what == "header":
        kw["n_keys"] = len(d["hits"]) + 1
    elif what == "seg_len":
        d["lens"][1] = -5
    elif what == "byte_count":
        kw["count_delta"] = 8
    elif what == "checksum":
        kw["fix_sum"] = False
    return d, kw


@pytest.mark.parametrize("what,msg", [("checksum", "checksum"), ("seg_off", "segment offsets"),
                                      ("ref_h", "threshold"), ("ref_rs_range", "position"),
                                      ("ref_rs_order", "position"), ("keys", "keys"),
                                      ("key_off", "hit-list offsets"), ("hits_range", "hits"),
                                      ("hits_order", "hits"), ("header", "header"), ("seg_len", "segment length"),
                                      ("byte_count", "truncated")])
def test_inconsistent_index_files_are_refused(tmp_path, sections, what, msg):
    p = str(tmp_path / f"{what}.shmapidx")
    d, kw = _corrupt(sections, what)
    write_index(p, d, **kw)
    rc, err = _check(p)
    assert rc == sb.SHM_ERR_INVALID and msg in err, (what, err)


def test_one_flipped_byte_anywhere_is_refused(tmp_path, sections):
    p = str(tmp_path / "ok.shmapidx")
    write_index(p, sections)
    blob = open(p, "rb").read()
    rng = np.random.default_rng(3)
    for pos in list(rng.integers(0, len(blob), 40)) + [0, 9, 20, len(blob) - 1, len(blob) - 9]:
        bad = bytearray(blob)
        bad[int(pos)] ^= 0x10
        q = str(tmp_path / "bad.shmapidx")
        open(q, "wb").write(bytes(bad))
        assert _check(q)[0] == sb.SHM_ERR_INVALID, pos
    assert _check(str(tmp_path / "missing.shmapidx"))[0] == sb.SHM_ERR_INVALID
