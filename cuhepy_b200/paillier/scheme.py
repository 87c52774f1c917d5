"""Textbook Paillier with the reference's static API, computed on the B200.

Drop-in for ``cuhepy.paillier.scheme.Paillier`` (src/cuhepy/paillier/scheme.py):
the same key dictionaries, the same ``ValueError`` range checks and the same
randomness rule for r (``secrets.randbelow(n-1)+1`` until gcd(r, n) = 1,
scheme.py:47-60).  ``encrypt``/``decrypt``/``add`` each run one kernel launch
(the per-operation form); the ``*_batch`` methods run a whole batch in one
launch.  For g = n + 1, the generator ``key_gen`` produces, encryption uses
g^m = 1 + m*n mod n^2 inside the r^n kernel; keys with any other g (loaded
from elsewhere) take g^m by a per-item exponentiation and one product, so
every g the reference accepts gives the reference's powmod(g, m, n^2) * r^n.
"""

from __future__ import annotations

import math
import secrets
from collections.abc import Sequence

from cuhepy_b200 import _numbers
from cuhepy_b200.paillier.gpu import device_for


class Paillier:
    """Static Paillier operations (mirror of ``cuhepy.paillier.scheme.Paillier``)."""

    def __init__(self, keys: dict) -> None:
        self.keys = keys

    @staticmethod
    def key_gen(key_len: int) -> dict:
        """scheme.py:24-44: p, q random key_len-bit primes, g = n + 1."""
        p = _numbers.get_prime(key_len)
        q = _numbers.get_prime(key_len)
        n = p * q
        phi = (p - 1) * (q - 1)
        return {"sk": {"phi": phi, "inv": pow(phi, -1, n)}, "pk": {"g": 1 + n, "n": n, "n_squared": n * n}}

    @staticmethod
    def generate_random_r(pk: dict) -> int:
        """scheme.py:47-60."""
        n = int(pk["n"])
        while True:
            r = secrets.randbelow(n - 1) + 1
            if math.gcd(r, n) == 1:
                return r

    @staticmethod
    def encrypt(plaintext: int, pk: dict) -> int:
        """c = g^m r^n mod n^2 (scheme.py:63-83), one launch."""
        return Paillier.encrypt_batch([plaintext], pk)[0]

    @staticmethod
    def encrypt_batch(plaintexts: Sequence[int], pk: dict, rs: Sequence[int] | None = None) -> list[int]:
        """Batched encryption; r values are drawn like the reference unless given."""
        n = int(pk["n"])
        for m in plaintexts:
            if not 0 <= int(m) < n:
                raise ValueError("plaintext must be in range [0, n)")
        if rs is None:
            rs = [Paillier.generate_random_r(pk) for _ in plaintexts]
        for r in rs:
            if math.gcd(int(r), n) != 1:
                raise ValueError("random r is not coprime with n")
        ctx = device_for(n)
        ms, rs = [int(m) for m in plaintexts], [int(r) for r in rs]
        g = int(pk["g"]) % (n * n)
        if g == n + 1:
            return ctx.encrypt(ms, rs)
        # scheme.py:81-83 for a general g: powmod(g, m, n^2) * powmod(r, n, n^2)
        r_n = ctx.encrypt([0] * len(ms), rs)
        return ctx.mulmod(ctx.modexp_each([g] * len(ms), ms), r_n)

    @staticmethod
    def decrypt(ciphertext: int, keys: dict) -> int:
        """m = ((c^phi mod n^2 - 1) // n) * inv mod n (scheme.py:86-104)."""
        return Paillier.decrypt_batch([ciphertext], keys)[0]

    @staticmethod
    def decrypt_batch(ciphertexts: Sequence[int], keys: dict) -> list[int]:
        n2 = int(keys["pk"]["n_squared"])
        for c in ciphertexts:
            if not 0 <= int(c) < n2:
                raise ValueError("ciphertext must be in range [0, n^2)")
        ctx = device_for(int(keys["pk"]["n"]), (int(keys["sk"]["phi"]), int(keys["sk"]["inv"])),
                         phi=keys["sk"]["phi"])
        return ctx.decrypt([int(c) for c in ciphertexts])

    @staticmethod
    def add(ciphertext1: int, ciphertext2: int, pk: dict) -> int:
        """c1 * c2 mod n^2 (scheme.py:107-119)."""
        return Paillier.add_batch([ciphertext1], [ciphertext2], pk)[0]

    @staticmethod
    def add_batch(ciphertexts1: Sequence[int], ciphertexts2: Sequence[int], pk: dict) -> list[int]:
        n = int(pk["n"])
        return device_for(n).mulmod([int(c) for c in ciphertexts1], [int(c) for c in ciphertexts2])

    @staticmethod
    def multiply(ciphertext1: int, ciphertext2: int, pk: dict) -> int:
        raise NotImplementedError("Paillier is not homomorphic under multiplication")

    @staticmethod
    def xor(ciphertext1: int, ciphertext2: int, pk: dict) -> int:
        raise NotImplementedError("Paillier is not homomorphic under xor")
