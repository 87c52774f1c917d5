"""Host-side BFV parameters, packed layout and wire format.

* ``rns_primes`` / ``coefficient_modulus``: the reference's modulus choices
  (src/cuhepy/bfv/scheme.py:186-216): 60-bit primes p = 1 mod 2N searched
  downward from 2^60 - 2N + 1, and the largest prime below 2^bits.
* ``Layout``: the packed Hamming layout of one embedding length
  (src/cuhepy/hamming/bfv.py:108-138, 249-307): ``padded`` = next power of
  two, ``lanes = N / (2 padded)`` vectors per slot row, ``capacity = 2 lanes``
  vectors per ciphertext, rotation steps +-lanes * 2^i.
* ``pack_poly`` / ``unpack_poly``: the packed wire (bits(modulus) bits per
  coefficient, little-endian; src/cuhepy/bfv/_cpu_ext/packed_wire.h:21-60),
  vectorised with numpy bit operations.
"""

from __future__ import annotations

import numpy as np

_SMALL = (2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37)
_MORE = _SMALL + (41, 43, 47, 53, 59, 61, 67, 71, 73, 79, 83, 89, 97)


def is_prime(x: int) -> bool:
    """Miller-Rabin with the first twelve prime bases, deterministic below
    3.3e24 (every NTT prime); above that the first 25 prime bases, a
    probable-prime test like the reference's gmpy2.is_prime (error below
    4^-25 for any composite)."""
    if x < 2:
        return False
    for p in _SMALL:
        if x % p == 0:
            return x == p
    d, r = x - 1, 0
    while not d & 1:
        d >>= 1
        r += 1
    for a in (_SMALL if x < 3_317_044_064_679_887_385_961_981 else _MORE):
        y = pow(a, d, x)
        if y in (1, x - 1):
            continue
        for _ in range(r - 1):
            y = y * y % x
            if y == x - 1:
                break
        else:
            return False
    return True


def rns_primes(n: int, bits: int) -> tuple[int, ...]:
    """bits/60 NTT primes for degree n, largest first."""
    if bits < 60 or bits > 480 or bits % 60:
        raise ValueError("rns modulus bits must be a multiple of 60 in [60, 480]")
    primes, c = [], (1 << 60) - 2 * n + 1
    while len(primes) < bits // 60:
        if is_prime(c):
            primes.append(c)
        c -= 2 * n
    return tuple(primes)


def rns_modulus(n: int, bits: int) -> int:
    q = 1
    for p in rns_primes(n, bits):
        q *= p
    return q


def coefficient_modulus(bits: int) -> int:
    """Largest prime below 2^bits (scheme.py:186-193): the response modulus
    of a compacted search, and the ciphertext modulus of a native ring."""
    if not 2 <= bits <= 512:
        raise ValueError("coefficient modulus bits must be 2..512")
    c = (1 << bits) - 1
    while not is_prime(c):
        c -= 2
    return c


class Layout:
    """Packed layout of ``embed_len``-bit vectors in degree-``n`` slots."""

    def __init__(self, n: int, embed_len: int) -> None:
        if embed_len < 1 or n < 4:
            raise ValueError("invalid layout")
        self.n = int(n)
        self.embed_len = int(embed_len)
        self.padded = 1 << (self.embed_len - 1).bit_length()
        if 2 * self.padded > self.n:
            raise ValueError("embedding too long for the ring degree")
        self.lanes = self.n // (2 * self.padded)
        self.capacity = 2 * self.lanes

    def _levels(self) -> range:
        return range(self.padded.bit_length() - 1)

    def rotation_steps(self) -> list[int]:
        return [sign * (self.lanes << i) for i in self._levels() for sign in (1, -1)]

    def left(self) -> list[int]:
        """Galois exponents of the tile sums (rotation by +lanes * 2^i)."""
        return [pow(3, (self.lanes << i) % (self.n // 2), 2 * self.n) for i in self._levels()]

    def right(self) -> list[int]:
        """Galois exponents of the merge tree (rotation by -lanes * 2^i)."""
        return [pow(3, (self.n // 2 - (self.lanes << i)) % (self.n // 2), 2 * self.n) for i in self._levels()]

    def query_slots(self, bits) -> np.ndarray:
        """Each query bit repeated over the lanes, both slot rows."""
        row = np.zeros(self.n // 2, dtype=np.uint32)
        b = np.asarray(bits, dtype=np.uint32).reshape(-1)
        row[: b.size * self.lanes] = np.repeat(b, self.lanes)
        return np.concatenate([row, row])

    def index_slots(self, vectors) -> np.ndarray:
        """[tiles, n] slot rows: vector k of a tile at row k // lanes, lane
        k % lanes, bit d at position d * lanes + lane."""
        v = np.asarray(vectors, dtype=np.uint32)
        if v.ndim != 2 or v.shape[1] > self.padded:
            raise ValueError("vectors must be [count, <= padded] bits")
        tiles = (v.shape[0] + self.capacity - 1) // self.capacity
        out = np.zeros((tiles, 2, self.padded, self.lanes), dtype=np.uint32)
        for start in range(0, v.shape[0], self.capacity):
            chunk = v[start:start + self.capacity]
            for lane in range(chunk.shape[0]):
                row, col = divmod(lane, self.lanes)
                out[start // self.capacity, row, : chunk.shape[1], col] = chunk[lane]
        return out.reshape(tiles, self.n)

    def mask_slots(self, count: int) -> np.ndarray:
        """1 in the first slot of each of the first `count` vector lanes."""
        mask = np.zeros(self.n, dtype=np.uint32)
        for lane in range(count):
            row, col = divmod(lane, self.lanes)
            mask[row * (self.n // 2) + col] = 1
        return mask


def _coefficient_bytes(coeffs, width: int) -> np.ndarray:
    raw = b"".join(int(c).to_bytes(width, "little") for c in coeffs)
    return np.frombuffer(raw, dtype=np.uint8).reshape(len(coeffs), width)


def pack_poly(coeffs, bits: int) -> bytes:
    """Little-endian bit packing, `bits` bits per coefficient."""
    width = (bits + 7) // 8
    as_bits = np.unpackbits(_coefficient_bytes(coeffs, width), axis=1, bitorder="little")[:, :bits]
    return np.packbits(as_bits.reshape(-1), bitorder="little").tobytes()


def unpack_poly(data: bytes, bits: int, n: int) -> list[int]:
    width = (bits + 7) // 8
    flat = np.unpackbits(np.frombuffer(data, dtype=np.uint8), bitorder="little")[: n * bits].reshape(n, bits)
    padded = np.zeros((n, 8 * width), dtype=np.uint8)
    padded[:, :bits] = flat
    raw = np.packbits(padded, axis=1, bitorder="little").tobytes()
    return [int.from_bytes(raw[i * width:(i + 1) * width], "little") for i in range(n)]


def fixed_poly(coeffs, modulus: int) -> bytes:
    """Fixed-width bytes (ceil(bits(modulus) / 8) per coefficient), the
    _bfv_rns poly format."""
    width = (modulus.bit_length() + 7) // 8
    return b"".join(int(c).to_bytes(width, "little") for c in coeffs)
