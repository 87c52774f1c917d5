"""Parity of the benchmarked BFV search configuration against the reference.

The timed BFV search (N = 8192, 30-bit gadget, t = 65537, embed 512, a
16,384-vector index = 1,024 tiles, two response groups, compacted to a
50-bit prime) takes code paths that small rings never reach: 3,072-CTA key
switch launches, the two-stream split of a tile batch with per-half merge
trees, merge waves of at most 148 (op, prime) pairs on the unfused switch,
and the host index uploaded in 256-tile pieces beside the tile circuits.
Here that exact configuration runs through the drop-in ``_bfv_rns`` and is
compared, byte for byte, with the reference's own compiled ``_bfv_rns``
(oracle/_ref, ``ResidueServer::search`` of bfv_residue.h:225-241 and the
merge tree of bfv_server.h:15-45), on

  * the residue ring Q = 3 x 60-bit primes, 1,024 tiles with a partial last
    tile (16,379 vectors), and
  * the native ring q = the largest prime below 2^180 (the reference's
    default client ring), 600 tiles (two uneven response groups),

for the host-index search (``packed_search``) and the resident-index search
(``search_index``), compacted and full.  Keys and ciphertexts are uniform
residues from a seeded generator, every tile distinct; the server circuit is
deterministic arithmetic on them, so equality is exact.  The reference
searches run on host threads beside the GPU work (the module releases the
GIL), the reference's own concurrency contract (test_bfv_rns.py:153-175).
"""

from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

from bfv_helpers import random_fixed_poly, random_packed_poly, reference_native, with_head
from oracle import bfv as ob

pytestmark = pytest.mark.gpu

N, GADGET, T, PADDED = 8192, 30, 65537, 512


def _case(residue: bool):
    if residue:
        q = 1
        for p in ob.rns_primes(N, 180):
            q *= p
        tiles, count = 1024, 1024 * 16 - 5
    else:
        q = ob.coefficient_modulus(180)
        tiles, count = 600, 599 * 16 + 7
    return q, tiles, count


def _inputs(q, tiles, seed):
    rng = np.random.default_rng(seed)
    layout = ob.Layout(N, PADDED)
    exps = sorted(set(layout.left()) | set(layout.right()))
    keys = [tuple((random_fixed_poly(rng, N, q), random_fixed_poly(rng, N, q)) for _ in range(6))
            for _ in range(1 + len(exps))]
    base = [tuple(random_packed_poly(rng, N, q) for _ in range(2)) for _ in range(32)]
    heads = rng.integers(0, 1 << 62, size=(tiles, 4), dtype=np.int64)
    index = []
    for i in range(tiles):
        b, a = base[i % len(base)]
        h = [int(v) % q for v in heads[i]]
        index.append((with_head(b, q, h[:2]), with_head(a, q, h[2:])))
    query = tuple(random_packed_poly(rng, N, q) for _ in range(2))
    assert len(set(index)) == tiles
    return layout, exps, keys, query, tuple(index)


def _server(mod, q, residue, layout, exps, keys):
    ring = mod.create_ring(N, format(q, "x"), GADGET, True, residue, 2 if residue else 0)
    relin = mod.compile_key(ring, keys[0])
    galois = tuple((g, mod.compile_key(ring, keys[1 + i])) for i, g in enumerate(exps))
    return mod.create_server(relin, galois, layout.padded, T, format(ob.coefficient_modulus(50), "x"))


@pytest.mark.parametrize("residue", [True, False], ids=["residue_1024_tiles", "native_600_tiles"])
def test_benchmarked_search_matches_reference_checker(residue):
    ref = reference_native()
    if ref is None:
        pytest.skip("reference checker oracle/_ref not built")
    from cuhepy_b200.bfv import _bfv_rns as m

    q, tiles, count = _case(residue)
    layout, exps, keys, query, index = _inputs(q, tiles, seed=16384 + residue)
    assert (tiles + layout.padded - 1) // layout.padded == 2
    rserver = _server(ref, q, residue, layout, exps, keys)
    with ThreadPoolExecutor(2) as pool:
        want = {compact: pool.submit(ref.packed_search, rserver, query, index, count, compact)
                for compact in (True, False)}
        gserver = _server(m, q, residue, layout, exps, keys)
        got = {compact: m.packed_search(gserver, query, index, count, compact) for compact in (True, False)}
        resident = m.upload_index(gserver, index)
        assert resident.tiles == tiles
        got_resident = {compact: m.search_index(gserver, resident, query, count, compact)
                        for compact in (True, False)}
        want = {compact: f.result() for compact, f in want.items()}
    for compact in (True, False):
        assert len(want[compact]) == 2
        assert got[compact] == want[compact], ("packed_search", compact)
        assert got_resident[compact] == want[compact], ("search_index", compact)
    # the bench's timed call: the resident search again, now that every
    # workspace and key is warm, and a second packed search (re-imported index)
    assert m.search_index(gserver, resident, query, count, True) == want[True]
    assert m.packed_search(gserver, query, index, count, True) == want[True]
