"""Rings of degree N = 32768, the reference's largest (bfv/scheme.py:279-280).

A plane of 32768 words exceeds one CTA's shared memory, so these rings use
the split transform (the stage that pairs the two halves of a plane on global
memory, each half in shared memory) and the unfused key switch.  Compared
with the oracle's exact products and the reference's own compiled _bfv_rns
(oracle/_ref).  Integer work: equality is exact."""

import math
import random

import numpy as np
import pytest

from bfv_helpers import fixed, key_bytes, packed, random_keys, reference_native
from oracle import bfv as ob

pytestmark = pytest.mark.gpu
N = 32768


def native():
    from cuhepy_b200.bfv import _bfv_rns

    return _bfv_rns


def test_split_ntt_is_the_negacyclic_ring_map_and_inverts():
    import torch

    m = native()
    primes = ob.rns_primes(N, 120)
    ring = m.create_ring(N, format(math.prod(primes), "x"), 30, True, True, 2)
    r = random.Random(5)
    rows = []
    for p in primes:
        a = [r.randrange(p) for _ in range(N)]
        b = [r.randrange(p) for _ in range(N)]
        rows.append((a, b, ob.ring_product(a, b, p)))
    # plane k * 2 + j uses prime j
    planes = np.zeros((6, N), dtype=np.uint64)
    for j, (a, b, c) in enumerate(rows):
        for k, row in enumerate((a, b, c)):
            planes[k * 2 + j] = row
    x = torch.from_numpy(planes.view(np.int64)).cuda()
    original = x.clone()
    m.ntt(ring, x, 2)
    torch.cuda.synchronize()
    got = x.cpu().numpy().view(np.uint64)
    for j, p in enumerate(primes):
        fa, fb, fc = (got[k * 2 + j].astype(object) for k in range(3))
        assert all(int(u) * int(v) % p == int(w) for u, v, w in zip(fa, fb, fc))
    m.ntt(ring, x, 2, inverse=True)
    torch.cuda.synchronize()
    assert torch.equal(x, original)


def test_batch_encode_matches_the_oracle():
    m = native()
    ring = m.create_ring(N, format(math.prod(ob.rns_primes(N, 180)), "x"), 30, True, True, 2)
    r = random.Random(32768)
    t = 65537
    rows = [[r.randrange(t) for _ in range(N)], [t - 1] * N]
    got = m.batch_encode(ring, t, np.array(rows, dtype=np.uint32))
    for row, coeffs in zip(rows, got):
        assert [int(c) for c in coeffs] == ob.batch_encode(row, N, t)


def _pair(q, gadget, residue):
    ref = reference_native()
    if ref is None:
        pytest.skip("reference checker oracle/_ref not built")
    m = native()
    level = 2 if residue else 0
    rring = ref.create_ring(N, format(q, "x"), gadget, True, residue, level)
    ring = m.create_ring(N, format(q, "x"), gadget, True, residue, level)
    assert m.ring_info(ring)["primes"] == ref.ring_info(rring)["primes"]
    return ref, m, rring, ring


@pytest.mark.parametrize("residue", [True, False])
def test_primitives_match_reference_checker(residue):
    q = math.prod(ob.rns_primes(N, 180)) if residue else ob.coefficient_modulus(180)
    ref, m, rring, ring = _pair(q, 30, residue)
    rng = random.Random(7 + residue)
    (key,) = random_keys(N, q, 6, 1, seed=3)
    kb = key_bytes(key, q)
    rkey, gkey = ref.compile_key(rring, kb), m.compile_key(ring, kb)
    a, b = ([rng.randrange(q) for _ in range(N)] for _ in range(2))
    fa, fb = fixed(a, q), fixed(b, q)
    assert m.apply_key(gkey, fa) == ref.apply_key(rkey, fa)
    assert m.ring_product(ring, fa, fb) == ref.ring_product(rring, fa, fb)
    assert m.multiply(ring, (fa, fb), None, 65537) == ref.multiply(rring, (fa, fb), None, 65537)
    for g in (3, 2 * N - 1):
        assert m.rotate_rows(gkey, (fa, fb), g) == ref.rotate_rows(rkey, (fa, fb), g)


def test_packed_search_matches_reference_checker():
    """Two tiles of 64 vectors (embed 512), a partial second tile, compact
    and full responses."""
    q = math.prod(ob.rns_primes(N, 180))
    ref, m, rring, ring = _pair(q, 30, True)
    layout = ob.Layout(N, 512)
    exps = sorted(set(layout.left()) | set(layout.right()))
    keys = random_keys(N, q, 6, 1 + len(exps), seed=11)
    kb = [key_bytes(k, q) for k in keys]
    rrelin, grelin = ref.compile_key(rring, kb[0]), m.compile_key(ring, kb[0])
    rg = tuple((g, ref.compile_key(rring, kb[1 + i])) for i, g in enumerate(exps))
    gg = tuple((g, m.compile_key(ring, kb[1 + i])) for i, g in enumerate(exps))
    target = ob.coefficient_modulus(50)
    rserver = ref.create_server(rrelin, rg, layout.padded, 65537, format(target, "x"))
    gserver = m.create_server(grelin, gg, layout.padded, 65537, format(target, "x"))
    rng = random.Random(13)
    bits = q.bit_length()

    def ct():
        return tuple(packed([rng.randrange(q) for _ in range(N)], bits) for _ in range(2))

    query = ct()
    index = (ct(), ct())
    count = layout.capacity + 5
    for compact in (True, False):
        assert m.packed_search(gserver, query, index, count, compact) == \
            ref.packed_search(rserver, query, index, count, compact), compact
