"""Bit-exact parity of the B200 BFV residue evaluator.

Compared, through the drop-in _bfv_rns module (C ABI), against
  * golden responses made by the reference's BFVClient (every backend), and
  * the reference's own compiled _bfv_rns (oracle/_ref) on seeded inputs,
    including the full-size ring N=8192, Q=3x60-bit, 30-bit gadget.
Integer work: equality is exact.
"""

import random

import pytest

from bfv_helpers import (
    fixed,
    key_bytes,
    packed,
    random_keys,
    reference_native,
    regenerate_fixture,
    unfixed,
)
from conftest import GOLDEN, load_golden
from oracle import bfv as ob

pytestmark = pytest.mark.gpu
FIXTURES = sorted(p.name for p in GOLDEN.glob("bfv_n*.json"))


def native():
    from cuhepy_b200.bfv import _bfv_rns

    return _bfv_rns


@pytest.mark.parametrize("name", FIXTURES)
def test_packed_search_matches_reference_golden(name):
    data = load_golden(name)
    params, layout, keys, query, index, vectors = regenerate_fixture(data)
    q, n = params.q, params.n
    m = native()
    ring = m.create_ring(n, format(q, "x"), params.gadget_bits, True, True, 2)
    info = m.ring_info(ring)
    assert info["residue_prime_count"] == info["switch_prime_count"] == params.q_bits // 60
    assert info["primes"][:len(params.primes)] == params.primes
    relin = m.compile_key(ring, key_bytes(keys["relin"], q))
    exps = sorted(set(layout.left()) | set(layout.right()))
    galois = tuple((g, m.compile_key(ring, key_bytes(keys["galois"][g], q))) for g in exps)
    target = min(ob.coefficient_modulus(data["response_modulus_bits"]), q)
    server = m.create_server(relin, galois, layout.padded, params.t, format(target, "x"))
    bits = q.bit_length()
    qp = (packed(query[0], bits), packed(query[1], bits))
    ip = tuple((packed(c[0], bits), packed(c[1], bits)) for c in index)
    for compact, key in ((False, "full"), (True, "compact")):
        ref = next(v for k, v in data["results"].items() if k.endswith(key))
        out_bits = target.bit_length() if compact else bits
        width = (n * out_bits + 7) // 8
        want = [(int(w[6], 16).to_bytes(width, "little"), int(w[7], 16).to_bytes(width, "little")) for w in ref]
        got = m.packed_search(server, qp, ip, len(vectors), compact)
        assert got == want, (name, compact)
    assert m.packed_search(server, qp, (), 0, True) == []


def _ring_pair(n, q_bits, gadget, t=None):
    ref = reference_native()
    if ref is None:
        pytest.skip("reference checker oracle/_ref not built")
    q = 1
    for p in ob.rns_primes(n, q_bits):
        q *= p
    m = native()
    return ref, m, q, ref.create_ring(n, format(q, "x"), gadget, True, True, 2), \
        m.create_ring(n, format(q, "x"), gadget, True, True, 2)


@pytest.mark.parametrize("n,q_bits,gadget", [(16, 60, 4), (16, 180, 30), (64, 480, 127), (1024, 180, 30),
                                             (8192, 180, 30), (64, 120, 61), (32, 180, 1), (8, 120, 30),
                                             (16384, 180, 30)])
def test_primitives_match_reference_checker(n, q_bits, gadget):
    ref, m, q, rring, ring = _ring_pair(n, q_bits, gadget)
    assert m.ring_info(ring)["primes"] == ref.ring_info(rring)["primes"]
    rng = random.Random(n + q_bits + gadget)
    digits = (q_bits + gadget - 1) // gadget
    (key,) = random_keys(n, q, digits, 1, seed=n)
    kb = key_bytes(key, q)
    rkey, gkey = ref.compile_key(rring, kb), m.compile_key(ring, kb)
    polys = [[rng.randrange(q) for _ in range(n)] for _ in range(4)]
    polys.append([q - 1] * n)
    polys.append([0] * (n - 1) + [q - 1])
    for poly in polys:
        b = fixed(poly, q)
        assert m.apply_key(gkey, b) == ref.apply_key(rkey, b)
        assert m.ring_product(ring, b, fixed(polys[0], q)) == ref.ring_product(rring, b, fixed(polys[0], q))
    t = 65537 if n <= 16384 and 65537 % (2 * n) == 1 else 97
    for lhs, rhs in ((polys[0], polys[1]), (polys[2], polys[3]), (polys[4], polys[4])):
        a = (fixed(lhs, q), fixed(rhs, q))
        assert m.multiply(ring, a, None, t) == ref.multiply(rring, a, None, t)
        bb = (fixed(polys[5], q), fixed(polys[1], q))
        assert m.multiply(ring, a, bb, t) == ref.multiply(rring, a, bb, t)
    for g in (3, 2 * n - 1, 5):
        ct = (fixed(polys[0], q), fixed(polys[1], q))
        assert m.rotate_rows(gkey, ct, g) == ref.rotate_rows(rkey, ct, g)


def test_full_size_packed_search_matches_reference_checker():
    """N=8192, Q = 3 x 60-bit primes, 30-bit gadget, t=65537, embed 512:
    three tiles (two full, one partial) in one response, compact and full."""
    n, q_bits, gadget, t, padded = 8192, 180, 30, 65537, 512
    ref, m, q, rring, ring = _ring_pair(n, q_bits, gadget)
    layout = ob.Layout(n, padded)
    exps = sorted(set(layout.left()) | set(layout.right()))
    digits = 6
    keys = random_keys(n, q, digits, 1 + len(exps), seed=8192)
    kb = [key_bytes(k, q) for k in keys]
    rrelin, grelin = ref.compile_key(rring, kb[0]), m.compile_key(ring, kb[0])
    rg = tuple((g, ref.compile_key(rring, kb[1 + i])) for i, g in enumerate(exps))
    gg = tuple((g, m.compile_key(ring, kb[1 + i])) for i, g in enumerate(exps))
    target = ob.coefficient_modulus(50)
    rserver = ref.create_server(rrelin, rg, padded, t, format(target, "x"))
    gserver = m.create_server(grelin, gg, padded, t, format(target, "x"))
    rng = random.Random(7)
    bits = q.bit_length()

    def ct():
        return tuple(packed([rng.randrange(q) for _ in range(n)], bits) for _ in range(2))

    query = ct()
    index = (ct(), ct(), ct())
    count = 2 * layout.capacity + 5
    for compact in (True, False):
        want = ref.packed_search(rserver, query, index, count, compact)
        got = m.packed_search(gserver, query, index, count, compact)
        assert got == want, compact


def test_boundary_errors():
    ref, m, q, rring, ring = _ring_pair(16, 180, 30)
    (key,) = random_keys(16, q, 6, 1, seed=1)
    k = m.compile_key(ring, key_bytes(key, q))
    with pytest.raises(ValueError):
        m.compile_key(ring, key_bytes(key, q)[:-1])
    bad = fixed([q] + [0] * 15, q)
    with pytest.raises(ValueError, match="Noncanonical"):
        m.apply_key(k, bad)
    with pytest.raises(TypeError):
        m.apply_key(k, "not bytes")
    with pytest.raises(ValueError):
        m.rotate_rows(k, (fixed([0] * 16, q), fixed([0] * 16, q)), 4)
    with pytest.raises(ValueError, match="(?i)residue"):
        m.create_ring(16, format(ob.coefficient_modulus(100), "x"), 15, True, False, 2)
    layout = ob.Layout(16, 3)
    with pytest.raises(ValueError, match="rotation key"):
        m.create_server(k, (), layout.padded, 97, format(ob.coefficient_modulus(40), "x"))


def test_resident_index_search_matches_packed_search():
    data = load_golden("bfv_n256_q180_g30.json")
    params, layout, keys, query, index, vectors = regenerate_fixture(data)
    q, n = params.q, params.n
    m = native()
    ring = m.create_ring(n, format(q, "x"), params.gadget_bits, True, True, 2)
    relin = m.compile_key(ring, key_bytes(keys["relin"], q))
    exps = sorted(set(layout.left()) | set(layout.right()))
    galois = tuple((g, m.compile_key(ring, key_bytes(keys["galois"][g], q))) for g in exps)
    target = min(ob.coefficient_modulus(40), q)
    server = m.create_server(relin, galois, layout.padded, params.t, format(target, "x"))
    bits = q.bit_length()
    qp = (packed(query[0], bits), packed(query[1], bits))
    ip = tuple((packed(c[0], bits), packed(c[1], bits)) for c in index)
    resident = m.upload_index(server, ip)
    for compact in (True, False):
        assert m.search_index(server, resident, qp, len(vectors), compact) == \
            m.packed_search(server, qp, ip, len(vectors), compact)
    bad = (packed([q] * n, bits), ip[0][1])
    with pytest.raises(ValueError, match="Noncanonical"):
        m.upload_index(server, (bad,) + ip[1:])


@pytest.mark.parametrize("residue", [True, False])
def test_pipelined_host_index_search_matches_reference_checker(residue):
    """A host-memory index of 589 tiles is uploaded in sub-batches of 256
    tiles overlapped with the tile circuits (three sub-batches, the last one
    ragged, a partial last tile); the responses equal the reference
    checker's and the resident-index search's, on residue and native rings."""
    ref = reference_native()
    if ref is None:
        pytest.skip("reference checker oracle/_ref not built")
    n, gadget, t, tiles = 16, 30, 97, 589
    q = 1
    for p in ob.rns_primes(n, 180):
        q *= p
    if not residue:
        q = ob.coefficient_modulus(180)
    m = native()
    rring = ref.create_ring(n, format(q, "x"), gadget, True, residue, 2 if residue else 0)
    ring = m.create_ring(n, format(q, "x"), gadget, True, residue, 2 if residue else 0)
    layout = ob.Layout(n, 3)
    exps = sorted(set(layout.left()) | set(layout.right()))
    keys = random_keys(n, q, 6, 1 + len(exps), seed=589)
    kb = [key_bytes(k, q) for k in keys]
    rrelin, grelin = ref.compile_key(rring, kb[0]), m.compile_key(ring, kb[0])
    rg = tuple((g, ref.compile_key(rring, kb[1 + i])) for i, g in enumerate(exps))
    gg = tuple((g, m.compile_key(ring, kb[1 + i])) for i, g in enumerate(exps))
    target = ob.coefficient_modulus(40)
    rserver = ref.create_server(rrelin, rg, layout.padded, t, format(target, "x"))
    gserver = m.create_server(grelin, gg, layout.padded, t, format(target, "x"))
    rng = random.Random(589)
    bits = q.bit_length()

    def ct():
        return tuple(packed([rng.randrange(q) for _ in range(n)], bits) for _ in range(2))

    query = ct()
    index = tuple(ct() for _ in range(tiles))
    count = (tiles - 1) * layout.capacity + 3
    resident = m.upload_index(gserver, index)
    for compact in (True, False):
        want = ref.packed_search(rserver, query, index, count, compact)
        assert m.packed_search(gserver, query, index, count, compact) == want, compact
        assert m.search_index(gserver, resident, query, count, compact) == want, compact
    bad = index[:300] + ((packed([q] * n, bits), index[300][1]),) + index[301:]
    with pytest.raises(ValueError, match="Noncanonical"):
        m.packed_search(gserver, query, bad, count, True)
