"""Paillier-Lookup (alpha-subgroup Paillier with fixed-base tables) on the B200.

Drop-in for ``cuhepy.paillier.lookup.PaillierLookup``
(src/cuhepy/paillier/lookup.py).  Key generation follows lookup.py:44-100 on
the host; the g_table (lookup.py:104-110) and the noise table
(lookup.py:113-117) are computed on the device, encryption is the table
product of lookup.py:213-252 and decryption is L(c^a) * g_a_inv mod n
(lookup.py:257-278).  Noise indices are drawn with
``secrets.randbelow(len(noise_table))`` exactly as the reference does.
"""

from __future__ import annotations

import math
import secrets
from collections.abc import Sequence

import numpy as np

from cuhepy_b200 import _numbers
from cuhepy_b200.paillier.gpu import NOISE_MULTIPLES, PaillierDevice, device_for

MSG_BITS = 8
NOISE_TABLE_SIZE = 2 ** 8
MIN_ALPHA_LEN = 256
DEFAULT_ALPHA_LEN = 280


def message_chunks_for(key_len: int) -> int:
    return (key_len * 2 + MSG_BITS - 1) // MSG_BITS


class PaillierLookup:
    """Static Paillier-Lookup operations (mirror of the reference class)."""

    def __init__(self, keys: dict) -> None:
        self.keys = keys

    # -- key generation (host) ------------------------------------------------
    @staticmethod
    def gen_dsa_params_custom(p_bits: int, q_bits: int) -> tuple[int, int, int]:
        """lookup.py:120-165: p = k*q + 1 with exactly p_bits bits, g of order q."""
        if q_bits >= p_bits:
            raise ValueError("alpha_len too large: q_bits must be < p_bits")
        q = _numbers.get_prime(q_bits)
        k_lo = (1 << (p_bits - 1)) // q
        k_hi = ((1 << p_bits) - 1) // q
        if k_lo % 2 == 1:
            k_lo += 1
        while True:
            span = (k_hi - k_lo) // 2 + 1
            k = k_lo + 2 * _numbers.get_random_range(0, span)
            p = k * q + 1
            if p.bit_length() != p_bits:
                continue
            if _numbers.is_probable_prime(p):
                break
        e = (p - 1) // q
        while True:
            h = _numbers.get_random_range(2, p - 1)
            g = pow(h, e, p)
            if g != 1:
                return p, q, g

    @staticmethod
    def L(x: int, n: int) -> int:
        return (x - 1) // n

    @staticmethod
    def crt_pair(a1: int, m1: int, a2: int, m2: int) -> tuple[int, int]:
        M = m1 * m2
        t = ((a2 - a1) % m2) * pow(m1 % m2, -1, m2) % m2
        return (a1 + m1 * t) % M, M

    @staticmethod
    def key_gen(key_len: int, alpha_len: int) -> dict:
        """lookup.py:44-100 (host), with both tables computed on the device."""
        q_bits_bound = min(key_len, alpha_len)
        q_bits_1 = q_bits_bound // 2
        q_bits_2 = q_bits_bound - q_bits_1
        p1, q1, g1 = PaillierLookup.gen_dsa_params_custom(key_len, q_bits_1)
        p2, q2, g2 = PaillierLookup.gen_dsa_params_custom(key_len, q_bits_2)
        p, q = p1, p2
        n = p * q
        n_sq = n * n
        g1_p2 = (g1 % p) * (1 + p) % (p * p)
        g2_q2 = (g2 % q) * (1 + q) % (q * q)
        g, _ = PaillierLookup.crt_pair(g1_p2, p * p, g2_q2, q * q)
        a = math.lcm(q1, q2)
        ctx = device_for(n)
        check_na, check_n = ctx.modexp_each([g, g], [n * a, n])
        if check_na != 1 or check_n == 1:
            return PaillierLookup.key_gen(key_len, alpha_len)
        phi = (p - 1) * (q - 1)
        g_n = check_n
        g_a = ctx.modexp([g], a)[0]
        g_a_inv = pow(PaillierLookup.L(g_a, n), -1, n)
        chunks = message_chunks_for(key_len)
        g_table = PaillierLookup.precompute_g_table(g, n, key_len)
        noise_table = PaillierLookup.precompute_noise_table(g, n)
        return {
            "sk": {"phi": phi, "a": a, "g_a_inv": g_a_inv},
            "pk": {"g": g, "n": n, "n_squared": n_sq, "g_n": g_n},
            "g_table": g_table,
            "noise_table": noise_table,
            "key_len": key_len,
            "message_chunks": chunks,
        }

    @staticmethod
    def precompute_g_table(g: int, n: int, key_len: int, msg_bits: int = MSG_BITS) -> dict[int, list[int]]:
        """g_table[i][j] = (g^(2^(8i)))^j mod n^2, built on the device."""
        if msg_bits != MSG_BITS:
            raise ValueError("only 8-bit message digits are supported")
        ctx = device_for(n)
        ctx.build_tables(g, message_chunks_for(key_len), None)
        rows = ctx.g_table()
        return {i: row for i, row in enumerate(rows)}

    @staticmethod
    def generate_random_r(n: int) -> int:
        """lookup.py:168-180."""
        while True:
            r = secrets.randbelow(int(n)) + 1
            if math.gcd(r, int(n)) == 1:
                return r

    @staticmethod
    def precompute_noise_table(g: int, n: int, size: int = NOISE_TABLE_SIZE) -> list[int]:
        """noise[k] = g_n^{r_k} with g_n = g^n and random r_k (lookup.py:113-117)."""
        ctx = device_for(n)
        g_n = ctx.modexp([g], n)[0]
        exponents = [PaillierLookup.generate_random_r(n) for _ in range(size)]
        return ctx.modexp_each([g_n] * size, exponents)

    @staticmethod
    def dump_tables(keys: dict) -> dict:
        g_table = keys.get("g_table", {})
        return {"g_table": {k: [int(x) for x in v] for k, v in g_table.items()},
                "noise_table": [int(x) for x in keys.get("noise_table", [])]}

    @staticmethod
    def load_tables(data: dict) -> tuple[dict[int, list[int]], list[int]]:
        g_table = {int(k): [int(x) for x in v] for k, v in data.get("g_table", {}).items()}
        return g_table, [int(x) for x in data.get("noise_table", [])]

    # -- table residency --------------------------------------------------------
    @staticmethod
    def _install(pk: dict, g_table, noise_table, message_chunks: int) -> PaillierDevice:
        ctx = device_for(int(pk["n"]))
        rows = [g_table[i] for i in range(message_chunks)] if message_chunks else []
        fingerprint = (message_chunks, len(noise_table),
                       tuple(int(r[1]) for r in rows[:2]), tuple(int(v) for v in noise_table[:2]),
                       int(rows[-1][255]) if rows else 0, int(noise_table[-1]) if noise_table else 0)
        if getattr(ctx, "_lookup_fingerprint", None) != fingerprint:
            if not rows or not noise_table:
                raise ValueError("lookup encryption needs a g_table and a noise table")
            ctx.set_tables(rows, noise_table)
            ctx._lookup_fingerprint = fingerprint
        return ctx

    # -- encryption / decryption ------------------------------------------------
    @staticmethod
    def encrypt(plaintext: int, pk: dict, g_table=None, noise_table=None, message_chunks: int = 0) -> int:
        """lookup.py:213-252 (one launch)."""
        return PaillierLookup.encrypt_batch([plaintext], pk, g_table, noise_table, message_chunks)[0]

    @staticmethod
    def encrypt_batch(plaintexts: Sequence[int], pk: dict, g_table=None, noise_table=None,
                      message_chunks: int = 0, noise_index: np.ndarray | None = None) -> list[int]:
        if g_table is None:
            g_table = {}
        if noise_table is None:
            noise_table = [1]
        n = int(pk["n"])
        for m in plaintexts:
            if not 0 <= int(m) < n:
                raise ValueError("plaintext must be in range [0, n)")
        if noise_index is None:
            draws = []
            for _ in plaintexts:
                PaillierLookup.generate_random_r(n)  # consumed like the reference (lookup.py:226)
                draws.append([secrets.randbelow(len(noise_table)) for _ in range(NOISE_MULTIPLES)])
            noise_index = np.asarray(draws, dtype=np.uint8).reshape(len(plaintexts), NOISE_MULTIPLES)
        ctx = PaillierLookup._install(pk, g_table, noise_table, message_chunks)
        return ctx.lookup_encrypt_ints([int(m) for m in plaintexts], noise_index)

    @staticmethod
    def decrypt(ciphertext: int, keys: dict) -> int:
        return PaillierLookup.decrypt_batch([ciphertext], keys)[0]

    @staticmethod
    def decrypt_batch(ciphertexts: Sequence[int], keys: dict) -> list[int]:
        n2 = int(keys["pk"]["n_squared"])
        for c in ciphertexts:
            if not 0 <= int(c) < n2:
                raise ValueError("ciphertext must be in range [0, n^2)")
        ctx = device_for(int(keys["pk"]["n"]), (int(keys["sk"]["a"]), int(keys["sk"]["g_a_inv"])),
                         phi=keys["sk"].get("phi"))
        return ctx.decrypt([int(c) for c in ciphertexts])

    @staticmethod
    def add(ciphertext1: int, ciphertext2: int, pk: dict) -> int:
        return device_for(int(pk["n"])).mulmod([int(ciphertext1)], [int(ciphertext2)])[0]

    @staticmethod
    def multiply(ciphertext1: int, ciphertext2: int, pk: dict) -> int:
        raise NotImplementedError("Paillier is not homomorphic under multiplication")

    @staticmethod
    def xor(ciphertext1: int, ciphertext2: int, pk: dict) -> int:
        raise NotImplementedError("Paillier is not homomorphic under xor")

    @staticmethod
    def bitlen(x: int) -> int:
        return int(x).bit_length() if x > 0 else 0

    @staticmethod
    def lift_to_p2_with_p_component(g_mod_p: int, p: int) -> int:
        return (g_mod_p * (1 + p)) % (p * p)
