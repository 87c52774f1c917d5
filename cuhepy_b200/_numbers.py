"""Host-side number theory for key generation (not on the hot path).

Prime generation follows the reference's use of ``Crypto.Util.number``
(``getPrime(bits)`` = random prime with exactly ``bits`` bits) and
``gmpy2.is_prime`` (Miller-Rabin).  Randomness comes from the module-level
``secrets`` object so callers and tests may substitute a seeded source, the
same way the reference modules read ``secrets`` at call time.
"""

from __future__ import annotations

import math
import secrets

_SMALL_PRIMES = [p for p in range(3, 2000, 2) if all(p % d for d in range(3, int(p ** 0.5) + 1, 2))]


def is_probable_prime(x: int, rounds: int = 40) -> bool:
    x = int(x)
    if x < 2:
        return False
    if x in (2, 3):
        return True
    if x % 2 == 0:
        return False
    for p in _SMALL_PRIMES:
        if x == p:
            return True
        if x % p == 0:
            return False
    d, s = x - 1, 0
    while d % 2 == 0:
        d //= 2
        s += 1
    for _ in range(rounds):
        a = 2 + secrets.randbelow(x - 3)
        y = pow(a, d, x)
        if y in (1, x - 1):
            continue
        for _ in range(s - 1):
            y = y * y % x
            if y == x - 1:
                break
        else:
            return False
    return True


def get_prime(bits: int) -> int:
    """Random prime with exactly ``bits`` bits (Crypto.Util.number.getPrime)."""
    if bits < 2:
        raise ValueError("prime size must be at least two bits")
    while True:
        candidate = secrets.randbits(bits) | (1 << (bits - 1)) | 1
        if is_probable_prime(candidate):
            return candidate


def get_random_range(a: int, b: int) -> int:
    """Uniform integer in [a, b) (Crypto.Util.number.getRandomRange)."""
    return a + secrets.randbelow(b - a)


def lcm(a: int, b: int) -> int:
    return math.lcm(int(a), int(b))


def factors_from_phi(n: int, phi: int) -> tuple[int, int] | None:
    """The primes p <= q of n = p q from phi = (p - 1)(q - 1): p + q = n - phi + 1
    and p, q are the roots of x^2 - (p + q) x + n.  None when (n, phi) is not
    such a pair."""
    n, phi = int(n), int(phi)
    s = n - phi + 1
    disc = s * s - 4 * n
    if s <= 0 or disc < 0:
        return None
    root = math.isqrt(disc)
    if root * root != disc or (s - root) % 2:
        return None
    p, q = (s - root) // 2, (s + root) // 2
    if p <= 1 or p * q != n:
        return None
    return p, q
