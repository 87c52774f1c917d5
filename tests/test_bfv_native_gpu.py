"""Bit-exact parity of the B200 BFV evaluator on native rings (residue=False).

A native ring keeps ciphertexts as integers mod q for any odd modulus q (a
prime from coefficient_modulus, or a product of NTT primes): the reference
computes its products with GMP (rns_ntt.h native path, bindings.cpp
create_ring residue=False); the B200 evaluator computes them exactly through
Garner reconstruction over auxiliary NTT primes.  Compared with
  * the reference's golden responses of its "native" backend, and
  * the reference's own compiled _bfv_rns (oracle/_ref) on seeded inputs,
    up to the full-size ring N=8192 with a 180-bit prime q.
Integer work: equality is exact.
"""

import math
import random

import pytest

from bfv_helpers import fixed, key_bytes, packed, random_keys, reference_native, regenerate_fixture
from conftest import GOLDEN, load_golden
from oracle import bfv as ob

pytestmark = pytest.mark.gpu
FIXTURES = sorted(p.name for p in GOLDEN.glob("bfv_n*.json"))


def native():
    from cuhepy_b200.bfv import _bfv_rns

    return _bfv_rns


@pytest.mark.parametrize("name", FIXTURES)
def test_native_ring_search_matches_reference_golden(name):
    data = load_golden(name)
    params, layout, keys, query, index, vectors = regenerate_fixture(data)
    q, n = params.q, params.n
    m = native()
    ring = m.create_ring(n, format(q, "x"), params.gadget_bits, True, False)
    assert m.ring_info(ring)["residue_prime_count"] == 0
    relin = m.compile_key(ring, key_bytes(keys["relin"], q))
    exps = sorted(set(layout.left()) | set(layout.right()))
    galois = tuple((g, m.compile_key(ring, key_bytes(keys["galois"][g], q))) for g in exps)
    target = min(ob.coefficient_modulus(data["response_modulus_bits"]), q)
    server = m.create_server(relin, galois, layout.padded, params.t, format(target, "x"))
    bits = q.bit_length()
    qp = (packed(query[0], bits), packed(query[1], bits))
    ip = tuple((packed(c[0], bits), packed(c[1], bits)) for c in index)
    for compact, key in ((False, "native_full"), (True, "native_compact")):
        width = (n * (target.bit_length() if compact else bits) + 7) // 8
        want = [(int(w[6], 16).to_bytes(width, "little"), int(w[7], 16).to_bytes(width, "little"))
                for w in data["results"][key]]
        assert m.packed_search(server, qp, ip, len(vectors), compact) == want, (name, compact)


def _native_pair(n, q, gadget):
    ref = reference_native()
    if ref is None:
        pytest.skip("reference checker oracle/_ref not built")
    m = native()
    rring = ref.create_ring(n, format(q, "x"), gadget, True, False)
    ring = m.create_ring(n, format(q, "x"), gadget, True, False)
    rinfo, info = ref.ring_info(rring), m.ring_info(ring)
    assert info["primes"] == rinfo["primes"]
    assert info["switch_prime_count"] == rinfo["switch_prime_count"]
    assert info["residue_prime_count"] == rinfo["residue_prime_count"] == 0
    return ref, m, rring, ring


NATIVE_RINGS = [
    (16, ob.coefficient_modulus(100), 15),
    (16, ob.coefficient_modulus(180), 30),
    (64, ob.coefficient_modulus(60), 4),
    (32, ob.coefficient_modulus(200), 61),
    (256, ob.coefficient_modulus(180), 1),
    (1024, ob.coefficient_modulus(180), 30),
    (8192, ob.coefficient_modulus(180), 30),
    (64, math.prod(ob.rns_primes(64, 120)), 40),
    (16, ob.coefficient_modulus(300), 30),
    (16, ob.coefficient_modulus(480), 127),
    (32, (1 << 512) - 1, 61),
    (8, ob.coefficient_modulus(100), 15),
    (16384, ob.coefficient_modulus(180), 30),
]


@pytest.mark.parametrize("n,q,gadget", NATIVE_RINGS)
def test_native_primitives_match_reference_checker(n, q, gadget):
    ref, m, rring, ring = _native_pair(n, q, gadget)
    rng = random.Random(n + q.bit_length() + gadget)
    digits = (q.bit_length() + gadget - 1) // gadget
    (key,) = random_keys(n, q, digits, 1, seed=n + 1)
    kb = key_bytes(key, q)
    rkey, gkey = ref.compile_key(rring, kb), m.compile_key(ring, kb)
    polys = [[rng.randrange(q) for _ in range(n)] for _ in range(4)]
    polys.append([q - 1] * n)
    polys.append([0] * (n - 1) + [q - 1])
    for poly in polys:
        b = fixed(poly, q)
        assert m.apply_key(gkey, b) == ref.apply_key(rkey, b)
        assert m.ring_product(ring, b, fixed(polys[0], q)) == ref.ring_product(rring, b, fixed(polys[0], q))
    for t in (65537, 97, 2):
        for lhs, rhs in ((polys[0], polys[1]), (polys[4], polys[4])):
            a = (fixed(lhs, q), fixed(rhs, q))
            assert m.multiply(ring, a, None, t) == ref.multiply(rring, a, None, t), t
            bb = (fixed(polys[5], q), fixed(polys[2], q))
            assert m.multiply(ring, a, bb, t) == ref.multiply(rring, a, bb, t), t
    for g in (3, 2 * n - 1, 5, 1):
        ct = (fixed(polys[0], q), fixed(polys[1], q))
        assert m.rotate_rows(gkey, ct, g) == ref.rotate_rows(rkey, ct, g)


@pytest.mark.parametrize("n,q,gadget,embed", [(16, ob.coefficient_modulus(180), 30, 3),
                                              (256, ob.coefficient_modulus(120), 40, 20)])
def test_native_hamming_tile_matches_reference_checker(n, q, gadget, embed):
    ref, m, rring, ring = _native_pair(n, q, gadget)
    layout = ob.Layout(n, embed)
    digits = (q.bit_length() + gadget - 1) // gadget
    exps = layout.left()
    keys = random_keys(n, q, digits, 1 + len(exps), seed=n)
    kb = [key_bytes(k, q) for k in keys]
    rrelin, grelin = ref.compile_key(rring, kb[0]), m.compile_key(ring, kb[0])
    rrot = tuple((g, ref.compile_key(rring, kb[1 + i])) for i, g in enumerate(exps))
    grot = tuple((g, m.compile_key(ring, kb[1 + i])) for i, g in enumerate(exps))
    rng = random.Random(q)
    query = tuple(fixed([rng.randrange(q) for _ in range(n)], q) for _ in range(2))
    tile = tuple(fixed([rng.randrange(q) for _ in range(n)], q) for _ in range(2))
    mask = fixed([rng.randrange(2) for _ in range(n)], q)
    t = 97 if n == 16 else 65537
    assert m.hamming_tile(grelin, query, tile, grot, mask, t) == ref.hamming_tile(rrelin, query, tile, rrot, mask, t)


@pytest.mark.parametrize("n,q_bits,gadget,t,padded,tiles,extra", [
    (16, 180, 30, 97, 4, 9, 3),
    (256, 100, 25, 65537, 16, 20, 7),
    (8192, 180, 30, 65537, 512, 3, 5),
])
def test_native_packed_search_matches_reference_checker(n, q_bits, gadget, t, padded, tiles, extra):
    """Several response groups, a ragged last group and a partial last tile,
    compact and full, through packed and resident-index searches."""
    q = ob.coefficient_modulus(q_bits)
    ref, m, rring, ring = _native_pair(n, q, gadget)
    layout = ob.Layout(n, padded)
    exps = sorted(set(layout.left()) | set(layout.right()))
    digits = (q_bits + gadget - 1) // gadget
    keys = random_keys(n, q, digits, 1 + len(exps), seed=n + tiles)
    kb = [key_bytes(k, q) for k in keys]
    rrelin, grelin = ref.compile_key(rring, kb[0]), m.compile_key(ring, kb[0])
    rg = tuple((g, ref.compile_key(rring, kb[1 + i])) for i, g in enumerate(exps))
    gg = tuple((g, m.compile_key(ring, kb[1 + i])) for i, g in enumerate(exps))
    target = ob.coefficient_modulus(min(50, q_bits - 1))
    rserver = ref.create_server(rrelin, rg, padded, t, format(target, "x"))
    gserver = m.create_server(grelin, gg, padded, t, format(target, "x"))
    rng = random.Random(n * tiles)
    bits = q.bit_length()

    def ct():
        return tuple(packed([rng.randrange(q) for _ in range(n)], bits) for _ in range(2))

    query = ct()
    index = tuple(ct() for _ in range(tiles))
    count = (tiles - 1) * layout.capacity + extra
    resident = m.upload_index(gserver, index)
    for compact in (True, False):
        want = ref.packed_search(rserver, query, index, count, compact)
        assert m.packed_search(gserver, query, index, count, compact) == want, compact
        assert m.search_index(gserver, resident, query, count, compact) == want, compact
    assert m.packed_search(gserver, query, (), 0, True) == []


@pytest.mark.parametrize("q_hex,gadget,n,level", [
    ("100", 15, 16, 0), ("3", 15, 16, 0), ("1", 1, 16, 0), ("ff" * 64, 30, 16, 0), ("ff" * 64 + "1", 30, 16, 0),
    ("65", 15, 24, 0), ("10001", 0, 16, 0), ("10001", 600, 16, 0), ("10001", 15, 16, 2), ("10001", 15, 16, 3),
    ("0f", 4, 16, 0),
])
def test_native_ring_parameters_match_reference_checker(q_hex, gadget, n, level):
    """Accepted or refused (ValueError) exactly as the reference's create_ring."""
    ref = reference_native()
    if ref is None:
        pytest.skip("reference checker oracle/_ref not built")
    m = native()
    try:
        rinfo = ref.ring_info(ref.create_ring(n, q_hex, gadget, True, False, level))
    except ValueError:
        with pytest.raises(ValueError):
            m.create_ring(n, q_hex, gadget, True, False, level)
        return
    info = m.ring_info(m.create_ring(n, q_hex, gadget, True, False, level))
    assert info["primes"] == rinfo["primes"]
    assert info["switch_prime_count"] == rinfo["switch_prime_count"]


def test_native_ring_errors():
    m = native()
    q = ob.coefficient_modulus(100)
    with pytest.raises(ValueError, match="(?i)residue"):
        m.create_ring(16, format(q, "x"), 15, True, False, 2)
    ring = m.create_ring(16, format(q, "x"), 15, True, False)
    (key,) = random_keys(16, q, 7, 1, seed=3)
    k = m.compile_key(ring, key_bytes(key, q))
    with pytest.raises(ValueError, match="Noncanonical"):
        m.apply_key(k, fixed([q] + [0] * 15, q))
    with pytest.raises(ValueError):
        m.rotate_rows(k, (fixed([0] * 16, q), fixed([0] * 16, q)), 4)


class _PrimeParams(ob.Params):
    """The reference's default BFVClient() ring: q is the largest prime below
    2^q_bits (scheme.py:186-193) instead of a product of NTT primes."""

    @property
    def q(self):
        return ob.coefficient_modulus(self.q_bits)


def test_default_parameters_search_decrypts_to_hamming_distances():
    """The reference's test_default_parameters_match_gmp (test_bfv_rns.py:178-194)
    on the device: N=8192, 180-bit prime q, 30-bit gadget, t=65537, embed 512,
    33 vectors with the query and its complement among them.  Real keys and
    encryptions (the oracle's client, seeded); the uncompacted responses equal
    the reference checker's, and the compacted ones decrypt to the plaintext
    Hamming distances."""
    from bfv_helpers import Seeded

    params = _PrimeParams(8192, 65537, 180, 30, 21)
    n, t, q = params.n, params.t, params.q
    layout = ob.Layout(n, 512)
    rng = Seeded(1337)
    keys = ob.key_gen(params, layout.rotation_steps(), rng)
    bits_rng = random.Random(1337)
    query = [bits_rng.getrandbits(1) for _ in range(512)]
    vectors = [[bits_rng.getrandbits(1) for _ in range(512)] for _ in range(33)]
    vectors[0] = query[:]
    vectors[1] = [1 - b for b in query]
    qct = ob.encrypt(ob.batch_encode(layout.query_slots(query), n, t), keys, rng)
    index = [ob.encrypt(ob.batch_encode(s, n, t), keys, rng) for s in layout.index_slots(vectors)]
    m = native()
    ring = m.create_ring(n, format(q, "x"), params.gadget_bits, True, False)
    relin = m.compile_key(ring, key_bytes(keys["relin"], q))
    exps = sorted(set(layout.left()) | set(layout.right()))
    galois = tuple((g, m.compile_key(ring, key_bytes(keys["galois"][g], q))) for g in exps)
    target = ob.coefficient_modulus(50)
    server = m.create_server(relin, galois, layout.padded, t, format(target, "x"))
    bits = q.bit_length()
    qp = (packed(qct[0], bits), packed(qct[1], bits))
    ip = tuple((packed(c[0], bits), packed(c[1], bits)) for c in index)
    full = m.packed_search(server, qp, ip, len(vectors), False)
    ref = reference_native()
    if ref is not None:
        rring = ref.create_ring(n, format(q, "x"), params.gadget_bits, True, False)
        rrelin = ref.compile_key(rring, key_bytes(keys["relin"], q))
        rg = tuple((g, ref.compile_key(rring, key_bytes(keys["galois"][g], q))) for g in exps)
        rserver = ref.create_server(rrelin, rg, layout.padded, t, format(target, "x"))
        assert full == ref.packed_search(rserver, qp, ip, len(vectors), False)
    (response,) = m.packed_search(server, qp, ip, len(vectors), True)
    ct = tuple(ob.unpack_poly(c, target.bit_length(), n) for c in response)
    slots = ob.batch_decode(ob.decrypt(ct, keys, target), n, t)
    got = []
    for pos in range(len(vectors)):
        tile, lane = divmod(pos, layout.capacity)
        row, col = divmod(lane, layout.lanes)
        got.append(slots[row * (n // 2) + tile * layout.lanes + col])
    assert got == [sum(x != y for x, y in zip(v, query)) for v in vectors]
    assert got[0] == 0 and got[1] == 512
