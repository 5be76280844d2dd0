"""The .fds v1 sample file (crates/fd-samples/src/{header,write,wire}.rs of the reference):
little-endian header (magic FDSAMPLE, major 1, minor, column bits, grid, iteration cap,
escape radius, rotation, the view strings and the kernel id, padded to 8 bytes), then each
present column in bit order, each padded to 8 bytes. Columns the route fills: class (u8),
nu (f64), de (f32), normal (u16), bound (f32), stripe (f32; crates/fd-samples/src/
column.rs:18-22)."""
import struct

import numpy as np

MAGIC = b"FDSAMPLE"
MAJOR, MINOR = 1, 1
BITS = {"class": 1, "nu": 2, "de": 4, "normal": 8, "bound": 16, "stripe": 32}


def _pad8(b: bytearray):
    b.extend(b"\0" * (-len(b) % 8))


def _str(b: bytearray, s: str):
    e = s.encode()
    if len(e) > 65535:
        raise ValueError("string longer than 65535 bytes")
    b += struct.pack("<H", len(e)) + e


def encode(header, samples, minor=MINOR) -> bytes:
    """Header::encode (header.rs:62-81) + write (write.rs:8-53)."""
    cols = ("class",) + tuple(c for c in ("nu", "de", "normal", "bound", "stripe") if c in header.columns)
    n = header.nx * header.ny
    b = bytearray(MAGIC)
    b += struct.pack("<HHIIIII", MAJOR, minor, sum(BITS[c] for c in cols), header.nx, header.ny, header.ss, 0)
    b += struct.pack("<Qdd", header.max_iter, header.escape_radius, header.view.rotation)
    for s in (header.view.center_re, header.view.center_im, header.view.width, header.kernel):
        _str(b, s)
    _pad8(b)
    arrays = {"class": (samples.cls, np.uint8), "nu": (samples.nu, "<f8"), "de": (samples.de, "<f4"),
              "normal": (samples.normal, "<u2"), "bound": (samples.bound, "<f4"),
              "stripe": (samples.stripe, "<f4")}
    for c in cols:
        a, dt = arrays[c]
        if a is None or len(a) != n:
            raise ValueError(f"column {c} does not match nx * ny")
        b += np.ascontiguousarray(a, dtype=dt).tobytes()
        _pad8(b)
    return bytes(b)


def write(path, header, samples):
    with open(path, "wb") as f:
        f.write(encode(header, samples))
