"""CPU oracle for the Paillier and Paillier-Lookup hot path.

TEST INFRASTRUCTURE ONLY: imported by ``tests/``, ``__graft_entry__.smoke()``
and the CPU-baseline leg of ``bench.py`` as the checker; never by the product.

A restatement of the reference algorithms over CPython integers, with the
encryption randomness passed in explicitly instead of drawn from ``secrets``
(the reference draws r and noise indices from the OS and has no seed hook).
Modular exponentiation goes to GMP 6.3.0 through ``oracle.gmp`` -- the same
library the reference's gmpy2 2.3.0 wraps.

Reference files (paths inside the cuhepy project):
  src/cuhepy/paillier/scheme.py   textbook Paillier
  src/cuhepy/paillier/lookup.py   alpha-subgroup variant with fixed-base tables
  src/cuhepy/hamming/paillier_lookup.py, hamming/paillier.py  Hamming codec
"""

from __future__ import annotations

import hashlib

from oracle.gmp import powmod

MSG_BITS = 8  # lookup.py:11
NOISE_TABLE_SIZE = 256  # lookup.py:12
NOISE_MULTIPLES = 14  # lookup.py:13


# --------------------------------------------------------------------------
# textbook Paillier: src/cuhepy/paillier/scheme.py
# --------------------------------------------------------------------------

def keys_from_primes(p: int, q: int) -> dict:
    """scheme.py:33-44: n=pq, phi=(p-1)(q-1), g=n+1, inv=phi^-1 mod n."""
    n = p * q
    phi = (p - 1) * (q - 1)
    return {"sk": {"phi": phi, "inv": pow(phi, -1, n)}, "pk": {"g": n + 1, "n": n, "n_squared": n * n}}


def encrypt(m: int, r: int, pk: dict) -> int:
    """scheme.py:63-83: c = g^m * r^n mod n^2 with the caller's r (scheme.py:78)."""
    n, n2 = pk["n"], pk["n_squared"]
    if not 0 <= m < n:
        raise ValueError("plaintext must be in range [0, n)")
    a = powmod(pk["g"], m, n2)
    b = powmod(r, n, n2)
    return a * b % n2


def decrypt(c: int, keys: dict) -> int:
    """scheme.py:86-104: m = ((c^phi mod n^2 - 1) // n) * inv mod n."""
    n, n2 = keys["pk"]["n"], keys["pk"]["n_squared"]
    if not 0 <= c < n2:
        raise ValueError("ciphertext must be in range [0, n^2)")
    x = powmod(c, keys["sk"]["phi"], n2) - 1
    return (x // n) * keys["sk"]["inv"] % n


def add(c1: int, c2: int, n_squared: int) -> int:
    """scheme.py:107-119 and lookup.py:282-294."""
    return c1 * c2 % n_squared


# --------------------------------------------------------------------------
# Paillier-Lookup: src/cuhepy/paillier/lookup.py
# --------------------------------------------------------------------------

def message_chunks(key_len: int) -> int:
    """lookup.py:99: number of 8-bit digits of a 2*key_len-bit plaintext."""
    return (key_len * 2 + MSG_BITS - 1) // MSG_BITS


def g_table(g: int, n: int, key_len: int) -> list[list[int]]:
    """lookup.py:104-110: g_table[i][j] = (g^(2^(8i)))^j mod n^2."""
    n2 = n * n
    table = []
    for i in range(message_chunks(key_len)):
        base = powmod(g, 1 << (MSG_BITS * i), n2)
        row = [1]
        for _ in range(1, 1 << MSG_BITS):
            row.append(row[-1] * base % n2)
        table.append(row)
    return table


def noise_table(g: int, n: int, exponents: list[int]) -> list[int]:
    """lookup.py:113-117: noise[k] = g_n^{r_k} mod n^2 with g_n = g^n mod n^2."""
    n2 = n * n
    g_n = powmod(g, n, n2)
    return [powmod(g_n, r, n2) for r in exponents]


def table_digest(rows: list[list[int]] | list[int], width_bytes: int) -> str:
    """SHA-256 over fixed-width little-endian entries, row-major."""
    digest = hashlib.sha256()
    flat = rows if rows and isinstance(rows[0], int) else [v for row in rows for v in row]
    for value in flat:
        digest.update(int(value).to_bytes(width_bytes, "little"))
    return digest.hexdigest()


def lookup_digits(m: int, chunks: int) -> list[int]:
    """lookup.py:239: base-256 digits of m, least significant first."""
    return [(m >> (MSG_BITS * i)) & 0xFF for i in range(chunks)]


def lookup_encrypt(m: int, pk: dict, table: list[list[int]], noise: list[int],
                   indices: list[int], chunks: int) -> int:
    """lookup.py:213-252: g_m = prod_i table[i][digit_i]; noise = prod of 14 noise entries.

    ``indices`` are the 14 noise-table indices the reference draws with
    ``secrets.randbelow(len(noise_table))`` (lookup.py:250).
    """
    n, n2 = pk["n"], pk["n_squared"]
    if not 0 <= m < n:
        raise ValueError("plaintext must be in range [0, n)")
    g_m = 1
    for i, d in enumerate(lookup_digits(m, chunks)):
        g_m = g_m * table[i][d] % n2
    acc = 1
    for k in indices:
        acc = acc * noise[k] % n2
    return g_m * acc % n2


def lookup_decrypt(c: int, keys: dict) -> int:
    """lookup.py:257-278: m = L(c^a mod n^2) * g_a_inv mod n, L(x) = (x-1)//n."""
    n, n2 = keys["pk"]["n"], keys["pk"]["n_squared"]
    if not 0 <= c < n2:
        raise ValueError("ciphertext must be in range [0, n^2)")
    c_a = (powmod(c, keys["sk"]["a"], n2) - 1) // n
    return c_a * keys["sk"]["g_a_inv"] % n


# --------------------------------------------------------------------------
# Hamming codec: src/cuhepy/hamming/paillier_lookup.py:61-77, 199-242
# --------------------------------------------------------------------------

def chunk_layout(embed_len: int, key_len: int) -> tuple[int, int]:
    """(chunk_len, chunk_num), paillier_lookup.py:73-77."""
    chunk_len = key_len * 2
    if embed_len > key_len:
        chunk_num = 2 * embed_len // chunk_len + int((2 * embed_len) % chunk_len != 0)
    else:
        chunk_num = 1
    return chunk_len, chunk_num


def encode_bits(bits: list[int], key_len: int) -> list[int]:
    """paillier_lookup.py:211-218: pad bit j to "0b_j", read chunk_len-bit MSB-first chunks."""
    chunk_len, chunk_num = chunk_layout(len(bits), key_len)
    padded = []
    for b in bits:
        if b not in (0, 1):
            raise ValueError("embedding must be binary")
        padded += ["0", str(b)]
    return [int("".join(padded[i * chunk_len:(i + 1) * chunk_len]), 2) for i in range(chunk_num)]


def decode_distance(plaintexts: list[int], key_len: int) -> int:
    """paillier_lookup.py:233-242: sum of the odd MSB-first positions of each chunk."""
    chunk_len = key_len * 2
    text = ""
    for d in plaintexts:
        s = f"{d:b}"
        if len(s) != chunk_len and len(s) != 0:
            s = "0" * (chunk_len - len(s)) + s
        text += s
    return sum(int(text[i]) for i in range(1, len(text), 2))
