"""ORACLE (test infrastructure only): CPU restatement of the reference's BGZF
writer, fq2bam-meth/python/bam_emit.py (_bgzf_block L77-98, _BgzfWriter
L101-186, _BGZF_EOF L21-23, _MAX_UNCOMPRESSED L24): the uncompressed stream
is cut every 65280 bytes, each piece is raw-deflated by zlib at the given
level and framed as a gzip member with the BC extra subfield; the EOF member
closes the file.  Also a member reader for the tests."""
from __future__ import annotations

import struct
import zlib

BLOCK = 65280
EOF_MEMBER = bytes.fromhex("1f8b08040000000000ff0600424302001b0003000000000000000000")


def member(chunk: bytes, level: int) -> bytes:
    c = zlib.compressobj(level, zlib.DEFLATED, -15)
    payload = c.compress(chunk) + c.flush()
    head = struct.pack("<BBBBLBBHBBHH", 31, 139, 8, 4, 0, 0, 255, 6, 66, 67, 2, 25 + len(payload))
    return head + payload + struct.pack("<II", zlib.crc32(chunk) & 0xFFFFFFFF, len(chunk) & 0xFFFFFFFF)


def compress(stream: bytes, level: int = 1, eof: bool = True) -> bytes:
    parts = [member(stream[i:i + BLOCK], level) for i in range(0, len(stream), BLOCK)]
    return b"".join(parts) + (EOF_MEMBER if eof else b"")


def members(data: bytes) -> list[dict]:
    """Splits a BGZF file into members: header fields, deflate payload,
    CRC-32 and ISIZE as stored."""
    out, off = [], 0
    while off < len(data):
        id1, id2, cm, flg, mtime, xfl, os_, xlen = struct.unpack_from("<BBBBLBBH", data, off)
        si1, si2, slen, bsize = struct.unpack_from("<BBHH", data, off + 12)
        size = bsize + 1
        payload = data[off + 18:off + size - 8]
        crc, isize = struct.unpack_from("<II", data, off + size - 8)
        out.append({"off": off, "size": size, "fixed": (id1, id2, cm, flg, mtime, xfl, os_, xlen, si1, si2, slen),
                    "payload": payload, "crc": crc, "isize": isize})
        off += size
    return out


def inflate(payload: bytes) -> bytes:
    d = zlib.decompressobj(-15)
    out = d.decompress(payload) + d.flush()
    if not d.eof or d.unused_data:
        raise ValueError("deflate stream not terminated where the member says")
    return out
