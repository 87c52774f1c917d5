"""Pin the BFV oracle to the golden vectors produced by the reference code:
the same seeded draws must reproduce the reference's keys and ciphertexts, and
the oracle's search must return the reference's responses bit for bit."""

import random

import pytest

from conftest import GOLDEN, load_golden
from oracle import bfv as ob

FIXTURES = sorted(p.name for p in GOLDEN.glob("bfv_n*.json"))


class Seeded:
    def __init__(self, seed):
        self._rng = random.Random(seed)

    def randbelow(self, n):
        return self._rng.randrange(n)

    def randbits(self, k):
        return self._rng.getrandbits(k)


def regenerate(data):
    params = ob.Params(data["n"], data["t"], data["q_bits"], data["gadget_bits"], data["eta"])
    layout = ob.Layout(params.n, data["embed_len"])
    rng = Seeded(data["seed"])
    keys = ob.key_gen(params, layout.rotation_steps(), rng)
    query_bits = [int(b) for b in data["query"]]
    vectors = [[int(b) for b in v] for v in data["vectors"]]
    query = ob.encrypt(ob.batch_encode(layout.query_slots(query_bits), params.n, params.t), keys, rng)
    index = [ob.encrypt(ob.batch_encode(s, params.n, params.t), keys, rng) for s in layout.index_slots(vectors)]
    return params, layout, keys, query, index, vectors


def wire_components(wire, bits, n):
    return tuple(ob.unpack_poly(int(w, 16).to_bytes((n * bits + 7) // 8, "little"), bits, n) for w in wire[6:8])


@pytest.mark.parametrize("name", FIXTURES)
def test_bfv_oracle_reproduces_reference(name):
    data = load_golden(name)
    if data["n"] > 64:
        pytest.skip("large ring covered by the slow marker")
    _check(data)


@pytest.mark.slow
@pytest.mark.parametrize("name", [f for f in FIXTURES if "n256" in f])
def test_bfv_oracle_reproduces_reference_n256(name):
    _check(load_golden(name))


def _check(data):
    params, layout, keys, query, index, vectors = regenerate(data)
    q, n = params.q, params.n
    assert ob.key_id(params, keys["b"], keys["a"]) == data["key_id"]
    bits = q.bit_length()
    assert wire_components(data["query_wire"], bits, n) == tuple(query)
    for wire, ct in zip(data["index_wire"], index):
        assert wire_components(wire, bits, n) == tuple(ct)
    target = min(ob.coefficient_modulus(data["response_modulus_bits"]), q)
    full = ob.search(query, index, len(vectors), keys, layout, None)
    comp = ob.search(query, index, len(vectors), keys, layout, target)
    ref_full = next(v for k, v in data["results"].items() if k.endswith("full"))
    ref_comp = next(v for k, v in data["results"].items() if k.endswith("compact"))
    for ours, ref in zip(full, ref_full):
        assert tuple(ours) == wire_components(ref, bits, n)
    for ours, ref in zip(comp, ref_comp):
        assert tuple(ours) == wire_components(ref, target.bit_length(), n)
    # decrypt the compacted responses and check the distances
    got = []
    for g, ct in enumerate(comp):
        slots = ob.batch_decode(ob.decrypt(ct, keys, target), n, params.t)
        for pos in range(min(n, len(vectors) - g * n)):
            tile, lane = divmod(pos, layout.capacity)
            row, col = divmod(lane, layout.lanes)
            got.append(slots[row * (n // 2) + tile * layout.lanes + col])
    assert got == data["distances"]
    qv = [int(b) for b in data["query"]]
    assert got == [sum(a != b for a, b in zip(qv, v)) for v in vectors]
