"""Packing of Python strings / byte strings into CSR buffers (bytes + offsets)."""

from __future__ import annotations

import numpy as np


def pack_strings(strings, offset_dtype=np.int32):
    """list[str | bytes] -> (uint8 data, offsets[B+1]).

    ``str`` items are encoded latin-1 (one byte per character, as in the
    reference bridges, src/gpu_bridge_monoid_batch.py:89-101); a character
    above U+00FF raises ``UnicodeEncodeError``."""
    B = len(strings)
    if B and isinstance(strings[0], (bytes, bytearray, memoryview)):
        blob = b"".join(strings)
        lens = np.fromiter((len(s) for s in strings), dtype=np.int64, count=B)
    else:
        blob = "".join(strings).encode("latin-1")
        lens = np.fromiter((len(s) for s in strings), dtype=np.int64, count=B)
    offsets = np.zeros(B + 1, dtype=np.int64)
    np.cumsum(lens, out=offsets[1:])
    if offset_dtype == np.int32 and B and offsets[-1] > np.iinfo(np.int32).max:
        raise OverflowError("batch larger than 2 GiB needs 64-bit offsets")
    data = np.frombuffer(blob, dtype=np.uint8).copy() if blob else np.zeros(1, dtype=np.uint8)
    return data, offsets.astype(offset_dtype), int(offsets[-1]) if B else 0
