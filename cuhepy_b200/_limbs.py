"""Python integers <-> little-endian 32-bit limb arrays (the C ABI layout)."""

from __future__ import annotations

from collections.abc import Iterable, Sequence

import numpy as np


def to_limbs(values: Sequence[int], words: int) -> np.ndarray:
    """Pack nonnegative integers into a C-contiguous uint32 array [len, words]."""
    width = 4 * words
    try:
        blob = b"".join(int(v).to_bytes(width, "little") for v in values)
    except OverflowError as exc:
        raise ValueError(f"integer does not fit in {width * 8} bits (or is negative)") from exc
    if not values:
        return np.zeros((0, words), dtype=np.uint32)
    return np.frombuffer(blob, dtype=np.uint32).reshape(len(values), words).copy()


def one_to_limbs(value: int, words: int) -> np.ndarray:
    return to_limbs([value], words)[0]


def from_limbs(array: np.ndarray) -> list[int]:
    """Unpack a uint32 array [count, words] into Python integers."""
    array = np.ascontiguousarray(array, dtype=np.uint32)
    if array.ndim == 1:
        array = array.reshape(1, -1)
    width = 4 * array.shape[1]
    raw = array.tobytes()
    return [int.from_bytes(raw[i:i + width], "little") for i in range(0, len(raw), width)]


def words_for(value: int) -> int:
    return max(1, (int(value).bit_length() + 31) // 32)


def as_u32(values: Iterable[int]) -> np.ndarray:
    return np.asarray(list(values), dtype=np.uint32)
