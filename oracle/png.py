"""PNG writer restated from src/png.zig:10-117 (test infrastructure).

Pure Python, byte for byte the reference's stream: signature, IHDR, one
IDAT chunk holding a zlib stream of stored (uncompressed) DEFLATE blocks of
at most 65535 bytes over rows that each start with filter byte 0, the
Adler-32 of the raw rows, and IEND.  The CRC-32 and Adler-32 are computed
here from their definitions (bitwise CRC over the reflected polynomial
0xEDB88320; Adler's two sums modulo 65521), independently of zlib, so the
tests can also check both against Python's zlib.
"""
from __future__ import annotations

import struct

MAX_STORED_BLOCK = 65535  # png.zig:8
SIGNATURE = b"\x89PNG\r\n\x1a\n"  # png.zig:7


class PngError(ValueError):
    pass


def crc32(data: bytes, crc: int = 0) -> int:
    """CRC-32 as PNG uses it (register preset to ones, result complemented)."""
    c = crc ^ 0xFFFFFFFF
    for byte in data:
        c ^= byte
        for _ in range(8):
            c = (c >> 1) ^ 0xEDB88320 if c & 1 else c >> 1
    return c ^ 0xFFFFFFFF


def adler32(data: bytes) -> int:
    a, b = 1, 0
    for byte in data:
        a = (a + byte) % 65521
        b = (b + a) % 65521
    return (b << 16) | a


def _chunk(kind: bytes, data: bytes) -> bytes:  # png.zig:60-70
    return struct.pack(">I", len(data)) + kind + data + struct.pack(">I", crc32(kind + data))


def write_png(width: int, height: int, rgb: bytes) -> bytes:
    """png.writePng (png.zig:10-58)."""
    assert len(rgb) == width * height * 3
    if width == 0 or height == 0 or width > 2**31 - 1 or height > 2**31 - 1:
        raise PngError("InvalidDimensions")
    raw_len = (width * 3 + 1) * height
    blocks = -(-raw_len // MAX_STORED_BLOCK)
    zlib_len = 2 + raw_len + 5 * blocks + 4
    if zlib_len > 2**31 - 1:
        raise PngError("ImageTooLarge")
    out = bytearray(SIGNATURE)
    out += _chunk(b"IHDR", struct.pack(">IIBBBBB", width, height, 8, 2, 0, 0, 0))
    raw = bytearray()
    row = width * 3
    for y in range(height):
        raw += b"\x00" + rgb[y * row:(y + 1) * row]
    z = bytearray(b"\x78\x01")
    pos = 0
    while pos < raw_len:  # StoredDeflate, png.zig:85-112
        n = min(MAX_STORED_BLOCK, raw_len - pos)
        final = 1 if pos + n == raw_len else 0
        z += bytes([final]) + struct.pack("<HH", n, n ^ 0xFFFF) + raw[pos:pos + n]
        pos += n
    z += struct.pack(">I", adler32(bytes(raw)))
    assert len(z) == zlib_len
    out += struct.pack(">I", zlib_len) + b"IDAT" + z + struct.pack(">I", crc32(b"IDAT" + bytes(z)))
    out += _chunk(b"IEND", b"")
    return bytes(out)
