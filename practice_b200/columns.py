"""On-disk column and validity formats of the reference's data directory.

Restates include/crystal/utils.h:98-253:
* a column is raw little-endian int32, one value per row (loadColumn :242-253);
* an optional validity file sits beside it, tried in this order per base name:
  ``.valid64 .valid .validity .valid_bitmap`` (uint64 words, bit = 1 valid),
  ``.valid8`` (one byte per row, non-zero valid), ``.null64 .null .nulls
  .null_bitmap`` (uint64 words, bit = 1 NULL), ``.null8`` (one byte per row,
  non-zero NULL) -- nullBitmapCandidateFiles :144-174;
* decoded validity is uint64 words, bit r = 1 when row r is valid, unused bits
  of the last word cleared (decodeValidityWordBitmap / ByteBitmap :114-140);
* a word file must hold exactly ceil(rows/64) words and a byte file exactly
  rows bytes, otherwise loading fails (:208-237).
"""
from __future__ import annotations

from pathlib import Path

import numpy as np

WORD_VALID = (".valid64", ".valid", ".validity", ".valid_bitmap")
WORD_NULL = (".null64", ".null", ".nulls", ".null_bitmap")


def word_count(rows: int) -> int:
    return (rows + 63) // 64


def last_word_mask(rows: int) -> int:
    rem = rows & 63
    return (1 << 64) - 1 if rem == 0 else (1 << rem) - 1


def decode_words(words: np.ndarray, rows: int, bits_are_valid: bool) -> np.ndarray:
    w = np.zeros(word_count(rows), dtype=np.uint64)
    n = min(len(words), len(w))
    w[:n] = np.asarray(words, dtype=np.uint64)[:n]
    if not bits_are_valid:
        w = ~w
    if len(w):
        w[-1] &= np.uint64(last_word_mask(rows))
    return w


def decode_bytes(data: np.ndarray, rows: int, bytes_are_valid: bool) -> np.ndarray:
    data = np.asarray(data, dtype=np.uint8)
    if len(data) != rows:
        raise ValueError("validity byte count does not match row count")
    valid = (data != 0) if bytes_are_valid else (data == 0)
    bits = np.zeros(word_count(rows) * 64, dtype=np.uint8)
    bits[:rows] = valid
    return np.packbits(bits, bitorder="little").view("<u8").astype(np.uint64)


def load_validity(base: Path, rows: int) -> np.ndarray | None:
    """Validity words of the column stored at `base` (no suffix), or None."""
    base = Path(base)
    candidates = [(s, "word", True) for s in WORD_VALID] + [(".valid8", "byte", True)] + \
                 [(s, "word", False) for s in WORD_NULL] + [(".null8", "byte", False)]
    for suffix, kind, is_valid in candidates:
        p = base.with_name(base.name + suffix)
        if not p.exists():
            continue
        raw = p.read_bytes()
        if kind == "word":
            if len(raw) != word_count(rows) * 8:
                raise ValueError(f"invalid null bitmap size for {base.name} at {p}: expected "
                                 f"{word_count(rows) * 8} bytes, got {len(raw)}")
            return decode_words(np.frombuffer(raw, dtype="<u8"), rows, is_valid)
        if len(raw) != rows:
            raise ValueError(f"invalid null bitmap size for {base.name} at {p}: expected {rows} bytes, got {len(raw)}")
        return decode_bytes(np.frombuffer(raw, dtype=np.uint8), rows, is_valid)
    return None


def load_column(path: Path, rows: int) -> np.ndarray:
    data = np.fromfile(path, dtype="<i4", count=rows)
    if len(data) != rows:
        raise ValueError(f"{path}: expected {rows} int32 values, found {len(data)}")
    return data.astype(np.int32)


def write_column(path: Path, values: np.ndarray, validity: np.ndarray | None = None) -> None:
    np.asarray(values, dtype="<i4").tofile(path)
    if validity is not None:
        np.asarray(validity, dtype="<u8").tofile(Path(str(path) + ".valid64"))
