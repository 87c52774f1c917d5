"""Client-side BFV encryption on the device (batched).

The reference's client encrypts one plaintext at a time in Python
(``BFV.encrypt``, src/cuhepy/bfv/scheme.py:426-444, with the batch encoding
of scheme.py:371-394): u ternary, e0 and e1 centred binomial with ``eta``
bits per side, c0 = b u + e0 + floor(Q/t) m and c1 = a u + e1.  Here the
noise is drawn on the GPU from a ChaCha20 keystream keyed from the operating
system's CSPRNG (``cuhe_bfv_encrypt_keyed``), or, with a seeded ``rng``, on
the host one draw at a time in the reference's order
(``cuhe_bfv_encrypt``); every ring product, the batch encoding and the wire
packing run on the GPU for the whole batch.  Given the same draws, the
ciphertexts are the reference's.
"""

from __future__ import annotations

import secrets
from typing import Any

import numpy as np

from cuhepy_b200.bfv import _bfv_rns


def _keystream(nbytes: int) -> bytes:
    """`nbytes` of ChaCha20 keystream under a fresh key and nonce from the
    operating system's CSPRNG (os.urandom itself when the `cryptography`
    package is absent)."""
    try:
        from cryptography.hazmat.primitives.ciphers import Cipher, algorithms
    except ImportError:  # pragma: no cover - the image ships cryptography
        return secrets.token_bytes(nbytes)
    enc = Cipher(algorithms.ChaCha20(secrets.token_bytes(32), secrets.token_bytes(16)), mode=None).encryptor()
    return enc.update(bytes(nbytes))


def draw_noise(count: int, n: int, eta: int = 21, rng: Any = None) -> tuple[np.ndarray, np.ndarray]:
    """(u [count, n] ternary, e [count, 2, n]) as int8.

    With ``rng`` (an object with ``randbelow``/``randbits``, like
    ``secrets``) the draws are made one value at a time in the reference's
    order per ciphertext (u, then e0, then e1; scheme.py:236-246, 438-439),
    so a seeded ``rng`` reproduces the reference's ciphertexts.  Without it,
    the same distributions are drawn in bulk from a cryptographic keystream
    (ChaCha20 keyed from the operating system's CSPRNG): u uniform on
    {-1, 0, 1} by rejection on bytes (0..254 are uniform mod 3), each e the
    difference of the popcounts of two independent eta-bit words."""
    if not 1 <= eta <= 63:
        raise ValueError("eta must be 1..63")
    if rng is not None:
        u = np.empty((count, n), dtype=np.int8)
        e = np.empty((count, 2, n), dtype=np.int8)
        for c in range(count):
            u[c] = [rng.randbelow(3) - 1 for _ in range(n)]
            for k in range(2):
                e[c, k] = [rng.randbits(eta).bit_count() - rng.randbits(eta).bit_count() for _ in range(n)]
        return u, e
    halves = count * 2 * n * 2
    wide = np.uint64 if eta > 31 else np.uint32
    size = np.dtype(wide).itemsize
    words = np.frombuffer(_keystream(size * halves), dtype=wide) & wide((1 << eta) - 1)
    pops = np.bitwise_count(words).astype(np.int8).reshape(count, 2, n, 2)
    e = pops[..., 0] - pops[..., 1]
    u = np.empty(count * n, dtype=np.int8)
    filled = 0
    while filled < u.size:
        want = u.size - filled
        raw = np.frombuffer(_keystream(want + want // 64 + 64), dtype=np.uint8)
        raw = raw[raw < 255][:want]
        u[filled:filled + raw.size] = (raw % 3).astype(np.int8) - 1
        filled += raw.size
    return u.reshape(count, n), e


def encrypt_batch(ring, public_key: tuple, t: int, slots, eta: int = 21, rng: Any = None) -> list[tuple[bytes, bytes]]:
    """Encrypt every row of ``slots`` ([count, N] slot values below t) under
    ``public_key`` = (b, a) fixed-width polys; returns packed (c0, c1)
    ciphertexts (the packed_search input wire)."""
    slots = np.ascontiguousarray(slots, dtype=np.uint32)
    if slots.ndim != 2:
        raise ValueError("slots must be [count, N]")
    if rng is not None:
        u, e = draw_noise(slots.shape[0], slots.shape[1], eta, rng)
        return _bfv_rns.encrypt_packed(ring, public_key, t, slots, u, e)
    if not 1 <= eta <= 63:
        raise ValueError("eta must be 1..63")
    n = slots.shape[1]
    blocks = (n // 4 if eta <= 31 else n // 2) + n // 8  # keystream blocks per ciphertext
    per_key = max(1, (1 << 32) // max(1, blocks))
    out: list[tuple[bytes, bytes]] = []
    for first in range(0, slots.shape[0], per_key):
        part = slots[first:first + per_key]
        for attempt in range(4):
            try:
                out += _bfv_rns.encrypt_packed_keyed(ring, public_key, t, part, secrets.token_bytes(32),
                                                     secrets.token_bytes(12), eta)
                break
            except _bfv_rns.KeystreamRejected:
                if attempt == 3:
                    raise
    return out
