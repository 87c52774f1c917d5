"""Concurrent calls give the results of sequential ones (the reference's
threading contract: its module releases the GIL and shares immutable plans,
test_bfv_native.py:81-105 and test_bfv_rns.py:160-168).  Here searches from
several host threads run on the ring's lanes (CUDA streams with their own
workspaces) and the other primitives share lane 0."""

import random
from concurrent.futures import ThreadPoolExecutor

import pytest

from bfv_helpers import fixed, key_bytes, packed, random_keys
from oracle import bfv as ob

pytestmark = pytest.mark.gpu


def native():
    from cuhepy_b200.bfv import _bfv_rns

    return _bfv_rns


@pytest.mark.parametrize("residue,tiles", [(True, 20), (False, 20), (True, 530)])
def test_concurrent_searches_and_primitives_match_sequential(residue, tiles):
    """Six searches over three lanes at once (host-memory and resident
    indexes; 530 tiles takes the pipelined upload), interleaved with key
    applications on the same ring."""
    m = native()
    n, gadget, t = (256, 30, 65537) if tiles == 20 else (16, 30, 97)
    if residue:
        q = 1
        for p in ob.rns_primes(n, 180):
            q *= p
    else:
        q = ob.coefficient_modulus(180)
    ring = m.create_ring(n, format(q, "x"), gadget, True, residue, 2 if residue else 0)
    layout = ob.Layout(n, 16 if n == 256 else 3)
    exps = sorted(set(layout.left()) | set(layout.right()))
    keys = random_keys(n, q, 6, 1 + len(exps), seed=tiles + residue)
    kb = [key_bytes(k, q) for k in keys]
    relin = m.compile_key(ring, kb[0])
    galois = tuple((g, m.compile_key(ring, kb[1 + i])) for i, g in enumerate(exps))
    server = m.create_server(relin, galois, layout.padded, t, format(ob.coefficient_modulus(40), "x"))
    rng = random.Random(tiles)
    bits = q.bit_length()

    def ct():
        return tuple(packed([rng.randrange(q) for _ in range(n)], bits) for _ in range(2))

    queries = [ct() for _ in range(3)]
    index = tuple(ct() for _ in range(tiles))
    count = tiles * layout.capacity - 1
    polys = [fixed([rng.randrange(q) for _ in range(n)], q) for _ in range(3)]
    want_search = [m.packed_search(server, qy, index, count, True) for qy in queries]
    want_key = [m.apply_key(relin, p) for p in polys]
    resident = m.upload_index(server, index)
    m.set_lanes(ring, 3)
    jobs = []
    for k in range(6):
        jobs.append(("packed" if k % 2 else "resident", k % 3))
        jobs.append(("key", k % 3))

    def run(job):
        kind, k = job
        if kind == "packed":
            return m.packed_search(server, queries[k], index, count, True)
        if kind == "resident":
            return m.search_index(server, resident, queries[k], count, True)
        return m.apply_key(relin, polys[k])

    with ThreadPoolExecutor(max_workers=4) as pool:
        got = list(pool.map(run, jobs))
    for (kind, k), result in zip(jobs, got):
        assert result == (want_key[k] if kind == "key" else want_search[k]), (kind, k)
