"""Test-only stand-in for gmpy2 2.3.0 (the version the reference pins).

``mpz`` is CPython's ``int``; every function below follows gmpy2's documented
semantics for the subset of the API the reference package calls.  Large modular
exponentiations go to the GMP 6.3.0 runtime through ``oracle.gmp``.
"""

from __future__ import annotations

import math
import random as _random
import sys
from pathlib import Path

sys.path.insert(0, str(Path(__file__).resolve().parents[3]))
from oracle import gmp as _gmp  # noqa: E402

mpz = int
xmpz = int


def version() -> str:
    return "2.3.0"


def mp_version() -> str:
    return "GMP " + _gmp.version()


def powmod(x: int, y: int, m: int) -> int:
    x, y, m = int(x), int(y), int(m)
    if y < 0:
        return pow(pow(x, -1, m), -y, m)
    return _gmp.powmod(x, y, m)


def invert(x: int, m: int) -> int:
    try:
        return pow(int(x), -1, int(m))
    except ValueError as exc:  # gmpy2 raises ZeroDivisionError
        raise ZeroDivisionError("invert() no inverse exists") from exc


def gcd(*values: int) -> int:
    return math.gcd(*[int(v) for v in values])


def lcm(*values: int) -> int:
    return math.lcm(*[int(v) for v in values])


def num_digits(x: int, base: int = 10) -> int:
    x = abs(int(x))
    if base == 2:
        return max(1, x.bit_length())
    return len(format(x, {8: "o", 10: "d", 16: "x"}[base])) if x else 1


_SMALL = [p for p in range(3, 1000, 2) if all(p % d for d in range(3, int(p**0.5) + 1, 2))]


def is_prime(x: int, n: int = 25) -> bool:
    """Miller-Rabin with n fixed pseudo-random bases (deterministic per input)."""
    x = int(x)
    if x < 2:
        return False
    if x in (2, 3):
        return True
    if x % 2 == 0:
        return False
    for p in _SMALL:
        if x == p:
            return True
        if x % p == 0:
            return False
    d, s = x - 1, 0
    while d % 2 == 0:
        d //= 2
        s += 1
    rng = _random.Random(x)
    for _ in range(max(n, 1)):
        a = rng.randrange(2, x - 1)
        y = _gmp.powmod(a, d, x)
        if y in (1, x - 1):
            continue
        for _ in range(s - 1):
            y = y * y % x
            if y == x - 1:
                break
        else:
            return False
    return True


def _pack(values: list[int], width: int) -> int:
    if len(values) == 1:
        return int(values[0])
    half = len(values) // 2
    return _pack(values[:half], width) | (_pack(values[half:], width) << (half * width))


def pack(values: list[int], width: int) -> int:
    """Concatenate nonnegative width-bit integers, first element least significant."""
    if not values:
        return 0
    if any(int(v) < 0 or int(v).bit_length() > width for v in values):
        raise ValueError("pack() requires nonnegative values that fit in the given width")
    return _pack(list(values), width)


def _unpack(x: int, width: int, count: int, out: list[int]) -> None:
    if count == 1:
        out.append(x)
        return
    half = count // 2
    _unpack(x & ((1 << (half * width)) - 1), width, half, out)
    _unpack(x >> (half * width), width, count - half, out)


def unpack(x: int, width: int) -> list[int]:
    """Split x into width-bit chunks, least significant first (at least one)."""
    x = int(x)
    if x < 0:
        raise ValueError("unpack() requires a nonnegative integer")
    count = max(1, -(-x.bit_length() // width))
    out: list[int] = []
    _unpack(x, width, count, out)
    return out
