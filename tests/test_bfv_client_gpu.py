"""Client-side BFV encryption on the device: with the reference's own random
draws replayed, the GPU batch reproduces the golden query and index
ciphertexts of the reference's BFVClient bit for bit."""

import random

import numpy as np
import pytest

from bfv_helpers import Seeded, fixed, packed, regenerate_fixture
from conftest import load_golden
from oracle import bfv as ob

pytestmark = pytest.mark.gpu


class Recorder:
    """Seeded draws, recorded in order so they can be replayed."""

    def __init__(self, seed):
        self.inner = Seeded(seed)

    def randbelow(self, n):
        return self.inner.randbelow(n)

    def randbits(self, k):
        return self.inner.randbits(k)


@pytest.mark.parametrize("name", ["bfv_n16_q60_g4.json", "bfv_n256_q180_g30.json", "bfv_n16_q480_g127.json"])
def test_gpu_encryption_reproduces_the_golden_ciphertexts(name):
    from cuhepy_b200.bfv import _bfv_rns as m
    from cuhepy_b200.bfv.client import draw_noise, encrypt_batch

    data = load_golden(name)
    params, layout, keys, query, index, vectors = regenerate_fixture(data)
    q, n, t = params.q, params.n, params.t
    ring = m.create_ring(n, format(q, "x"), params.gadget_bits, True, True, 2)
    # replay the fixture's draws: key generation, then u, e0, e1 per ciphertext
    rng = Seeded(data["seed"])
    ob.key_gen(params, layout.rotation_steps(), rng)
    qbits = [int(b) for b in data["query"]]
    slots = [layout.query_slots(qbits)] + list(layout.index_slots(vectors))
    slots = np.array([[int(v) for v in s] for s in slots], dtype=np.uint32)
    pk = (fixed(keys["b"], q), fixed(keys["a"], q))
    got = encrypt_batch(ring, pk, t, slots, params.eta, rng)
    bits = q.bit_length()
    want = [query] + list(index)
    assert len(got) == len(want)
    for (c0, c1), ct in zip(got, want):
        assert c0 == packed(ct[0], bits) and c1 == packed(ct[1], bits)
    # the fast host noise has the right shapes and ranges
    u, e = draw_noise(3, n, params.eta)
    assert set(np.unique(u)) <= {-1, 0, 1} and np.abs(e).max() <= params.eta


def test_gpu_encryption_decrypts_and_rejects_bad_slots():
    from cuhepy_b200.bfv import _bfv_rns as m
    from cuhepy_b200.bfv.client import encrypt_batch

    params = ob.Params(256, 65537, 180, 30, 21)
    q, n, t = params.q, params.n, params.t
    rng = Seeded(123)
    layout = ob.Layout(n, 16)
    keys = ob.key_gen(params, layout.rotation_steps(), rng)
    ring = m.create_ring(n, format(q, "x"), params.gadget_bits, True, True, 2)
    pk = (fixed(keys["b"], q), fixed(keys["a"], q))
    r = random.Random(4)
    slots = np.array([[r.randrange(t) for _ in range(n)] for _ in range(5)], dtype=np.uint32)
    cts = encrypt_batch(ring, pk, t, slots, params.eta)  # bulk CSPRNG noise
    bits = q.bit_length()
    for row, (c0, c1) in zip(slots, cts):
        ct = (ob.unpack_poly(c0, bits, n), ob.unpack_poly(c1, bits, n))
        assert ob.batch_decode(ob.decrypt(ct, keys), n, t) == [int(v) for v in row]
    bad = slots.copy()
    bad[0, 0] = t
    with pytest.raises(ValueError):
        encrypt_batch(ring, pk, t, bad, params.eta)


@pytest.mark.parametrize("n", [16, 256, 8192])
def test_gpu_batch_encode_matches_the_oracle(n):
    from cuhepy_b200.bfv import _bfv_rns as m

    q = 1
    for p in ob.rns_primes(n, 180):
        q *= p
    ring = m.create_ring(n, format(q, "x"), 30, True, True, 2)
    r = random.Random(n)
    t = 65537
    rows = [[r.randrange(t) for _ in range(n)] for _ in range(3)] + [[t - 1] * n, [0] * n]
    got = m.batch_encode(ring, t, np.array(rows, dtype=np.uint32))
    for row, coeffs in zip(rows, got):
        assert [int(c) for c in coeffs] == ob.batch_encode(row, n, t)
    with pytest.raises(ValueError):
        m.batch_encode(ring, 65539, np.array(rows[:1], dtype=np.uint32))  # 65539 != 1 mod 2N


def _keystream_noise(key, nonce, count, n, eta):
    """The keyed draws of cuhe_bfv_encrypt_keyed rebuilt on the host from the
    `cryptography` package's ChaCha20 (16-byte nonce = 32-bit little-endian
    block counter, then the 12-byte nonce)."""
    from cryptography.hazmat.primitives.ciphers import Cipher, algorithms

    e_blocks = n // 4 if eta <= 31 else n // 2
    blocks = e_blocks + n // 8
    wide = np.uint32 if eta <= 31 else np.uint64
    mask = wide((1 << eta) - 1)
    u = np.empty((count, n), dtype=np.int8)
    e = np.empty((count, 2, n), dtype=np.int8)
    for c in range(count):
        counter = (c * blocks).to_bytes(4, "little")
        stream = Cipher(algorithms.ChaCha20(key, counter + nonce), mode=None).encryptor().update(bytes(64 * blocks))
        words = np.frombuffer(stream[:64 * e_blocks], dtype=wide) & mask
        pops = np.bitwise_count(words).astype(np.int16).reshape(2 * n, 2)
        e[c] = (pops[:, 0] - pops[:, 1]).astype(np.int8).reshape(2, n)
        raw = np.frombuffer(stream[64 * e_blocks:], dtype=np.uint8).reshape(n, 8)
        first = np.argmax(raw < 255, axis=1)
        assert (raw < 255).any(axis=1).all()
        u[c] = (raw[np.arange(n), first] % 3).astype(np.int8) - 1
    return u, e


@pytest.mark.parametrize("n,eta", [(256, 21), (256, 40), (8192, 21)])
def test_keyed_device_noise_is_the_documented_chacha20_draw(n, eta):
    """cuhe_bfv_encrypt_keyed equals cuhe_bfv_encrypt given the noise rebuilt
    on the host from the same key and nonce: the device keystream and the
    noise derivation are exact."""
    from cuhepy_b200.bfv import _bfv_rns as m

    params = ob.Params(n, 65537, 180, 30, eta)
    q, t = params.q, params.t
    ring = m.create_ring(n, format(q, "x"), params.gadget_bits, True, True, 2)
    r = random.Random(n + eta)
    pk = tuple(fixed([r.randrange(q) for _ in range(n)], q) for _ in range(2))  # any (b, a) below q
    count = 3
    slots = np.array([[r.randrange(t) for _ in range(n)] for _ in range(count)], dtype=np.uint32)
    key, nonce = bytes(range(32)), bytes(range(100, 112))
    u, e = _keystream_noise(key, nonce, count, n, eta)
    assert set(np.unique(u)) <= {-1, 0, 1} and np.abs(e).max() <= eta
    assert m.encrypt_packed_keyed(ring, pk, t, slots, key, nonce, eta) == m.encrypt_packed(ring, pk, t, slots, u, e)
