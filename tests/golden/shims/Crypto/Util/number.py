"""Test-only stand-in for pycryptodome 3.23.0 ``Crypto.Util.number``.

``getPrime``/``getRandomRange`` draw from a module-level generator that
``seed()`` resets, so that "keys generated from seed 0" are reproducible.
"""

from __future__ import annotations

import random as _random

import gmpy2

_rng = _random.Random(0)


def seed(value: int) -> None:
    global _rng
    _rng = _random.Random(value)


def getRandomRange(a: int, b: int, randfunc=None) -> int:
    """Uniform integer in [a, b)."""
    return a + _rng.randrange(int(b) - int(a))


def getRandomNBitInteger(bits: int, randfunc=None) -> int:
    return _rng.getrandbits(bits) | (1 << (bits - 1))


def getPrime(bits: int, randfunc=None) -> int:
    """Random prime with exactly ``bits`` bits."""
    if bits < 2:
        raise ValueError("prime size must be at least two bits")
    while True:
        candidate = getRandomNBitInteger(bits) | 1
        if gmpy2.is_prime(candidate, 40):
            return candidate
