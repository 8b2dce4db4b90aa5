"""FASTA/FASTQ reading with the reference's record semantics (src/io/mod.rs:383-427):
the id is the header up to the first space or tab, sequence lines are joined
with their line ends (and a trailing '\\r') removed."""
from __future__ import annotations

from typing import List, Tuple


def read_fastx(path: str) -> List[Tuple[str, bytes]]:
    with open(path, "rb") as f:
        data = f.read()
    out: List[Tuple[str, bytes]] = []
    name = None
    parts: List[bytes] = []
    lines = data.split(b"\n")
    i = 0
    while i < len(lines):
        line = lines[i]
        if line.endswith(b"\r"):
            line = line[:-1]
        i += 1
        if line.startswith(b">"):
            if name is not None:
                out.append((name, b"".join(parts)))
            name = line[1:].split(b" ")[0].split(b"\t")[0].decode(errors="replace")
            parts = []
        elif line.startswith(b"@") and name is None:
            # FASTQ: header, sequence, '+', quality
            hdr = line[1:].split(b" ")[0].split(b"\t")[0].decode(errors="replace")
            seq = lines[i].rstrip(b"\r") if i < len(lines) else b""
            i += 3
            out.append((hdr, seq))
        elif name is not None:
            parts.append(line)
        elif line:
            raise ValueError(f"invalid FASTA record in {path}")
    if name is not None:
        out.append((name, b"".join(parts)))
    return out


def write_fasta(path: str, records, width: int = 0) -> None:
    with open(path, "wb") as f:
        for name, seq in records:
            f.write(b">" + name.encode() + b"\n")
            if width:
                for j in range(0, len(seq), width):
                    f.write(seq[j:j + width] + b"\n")
            else:
                f.write(seq + b"\n")
