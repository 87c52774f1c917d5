"""The package's host-side BFV layout and wire helpers equal the oracle's
restatement of the reference (no GPU)."""

import random

import pytest

from cuhepy_b200.bfv import layout as lay
from oracle import bfv as ob


@pytest.mark.parametrize("n,bits", [(16, 60), (256, 180), (8192, 180), (16384, 480), (4096, 120)])
def test_primes_match(n, bits):
    assert lay.rns_primes(n, bits) == ob.rns_primes(n, bits)


def test_coefficient_modulus_matches():
    for bits in (20, 40, 50, 61, 64, 100, 180, 300, 512):
        assert lay.coefficient_modulus(bits) == ob.coefficient_modulus(bits)


@pytest.mark.parametrize("n,embed", [(16, 3), (256, 16), (8192, 512), (8192, 256), (8192, 1024), (64, 5)])
def test_layout_matches(n, embed):
    a, b = lay.Layout(n, embed), ob.Layout(n, embed)
    assert (a.padded, a.lanes, a.capacity) == (b.padded, b.lanes, b.capacity)
    assert a.rotation_steps() == b.rotation_steps() and a.left() == b.left() and a.right() == b.right()
    rng = random.Random(n + embed)
    bits = [rng.getrandbits(1) for _ in range(embed)]
    assert [int(v) for v in a.query_slots(bits)] == b.query_slots(bits)
    vectors = [[rng.getrandbits(1) for _ in range(embed)] for _ in range(2 * a.capacity + 3)]
    assert [[int(v) for v in row] for row in a.index_slots(vectors)] == b.index_slots(vectors)
    for count in (1, a.capacity, a.capacity - 1):
        assert [int(v) for v in a.mask_slots(count)] == b.mask_slots(count)


@pytest.mark.parametrize("bits", [1, 17, 60, 180, 181, 479])
def test_wire_round_trip_matches(bits):
    rng = random.Random(bits)
    poly = [rng.getrandbits(bits) for _ in range(64)] + [0, (1 << bits) - 1]
    packed = lay.pack_poly(poly, bits)
    assert packed == ob.pack_poly(poly, bits)
    assert lay.unpack_poly(packed, bits, len(poly)) == poly == ob.unpack_poly(packed, bits, len(poly))
