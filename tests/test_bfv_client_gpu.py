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
