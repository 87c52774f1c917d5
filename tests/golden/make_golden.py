"""Generate the golden fixtures in tests/golden/ by running the REFERENCE code.

Run in a container where the reference project is present (read-only):

    python tests/golden/make_golden.py [--reference <reference tree>]   (default: $CUHEPY_REFERENCE)

The reference's own Python package is imported unmodified.  Its missing
third-party wheels are replaced by the test-only shims in tests/golden/shims
(gmpy2 over CPython int + GMP 6.3.0, a seeded Crypto.Util.number), and the
module-level ``secrets`` objects of the reference modules are replaced by a
seeded recorder so that every random draw (Paillier r, lookup noise
exponents and noise indices, BFV secrets/errors) is reproducible and written
into the fixture next to the outputs it produced.

Fixtures are plain JSON with integers as hex strings.
"""

from __future__ import annotations

import argparse
import json
import math
import os
import random
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]


class RecordingSecrets:
    """Seeded replacement for the ``secrets`` module; records every draw."""

    def __init__(self, seed: int) -> None:
        self._rng = random.Random(seed)
        self.log: list[tuple[str, int, int]] = []

    def randbelow(self, n: int) -> int:
        value = self._rng.randrange(int(n))
        self.log.append(("below", int(n), value))
        return value

    def randbits(self, k: int) -> int:
        value = self._rng.getrandbits(int(k))
        self.log.append(("bits", int(k), value))
        return value

    def take(self) -> list[tuple[str, int, int]]:
        out, self.log = self.log, []
        return out


def h(x: int) -> str:
    return format(int(x), "x")


def setup(reference: Path):
    sys.path.insert(0, str(HERE / "shims"))
    sys.path.insert(0, str(reference / "src"))
    sys.path.insert(0, str(REPO))
    import cuhepy.paillier.scheme as scheme
    import cuhepy.paillier.lookup as lookup
    import cuhepy.bfv.scheme as bfv_scheme
    from Crypto.Util import number
    return scheme, lookup, bfv_scheme, number


def paillier_fixture(scheme, number, key_len: int) -> dict:
    """Paillier.key_gen / encrypt / add / decrypt (src/cuhepy/paillier/scheme.py:24-119)."""
    number.seed(0)
    rec = RecordingSecrets(2)
    scheme.secrets = rec
    keys = scheme.Paillier.key_gen(key_len)
    pk, n = keys["pk"], keys["pk"]["n"]
    rng = random.Random(1)
    plaintexts = [0, 1, 2, (1 << 32) - 1, n - 1, n - 2]
    plaintexts += [rng.randrange(1 << 32) for _ in range(10)]
    cases = []
    for m in plaintexts:
        rec.take()
        c = scheme.Paillier.encrypt(m, pk)
        draws = rec.take()
        # generate_random_r: r = randbelow(n-1)+1 until gcd(r, n) == 1 (scheme.py:56-59)
        r = draws[-1][2] + 1
        cases.append({"m": h(m), "r": h(r), "c": h(c)})
    sums = []
    for i in range(0, len(cases) - 1, 2):
        c1, c2 = int(cases[i]["c"], 16), int(cases[i + 1]["c"], 16)
        s = scheme.Paillier.add(c1, c2, pk)
        sums.append({"i": i, "j": i + 1, "c": h(s), "m": h(scheme.Paillier.decrypt(s, keys))})
    for case in cases:
        case["d"] = h(scheme.Paillier.decrypt(int(case["c"], 16), keys))
    return {
        "key_len": key_len,
        "pk": {k: h(v) for k, v in pk.items()},
        "sk": {k: h(v) for k, v in keys["sk"].items()},
        "encrypt": cases,
        "add": sums,
    }


def lookup_fixture(lookup, number, key_len: int, alpha_len: int, hamming_vectors: int) -> dict:
    """PaillierLookup key_gen / encrypt / add / decrypt (src/cuhepy/paillier/lookup.py)."""
    from oracle import paillier as oracle
    number.seed(0)
    rec = RecordingSecrets(3)
    lookup.secrets = rec
    keys = lookup.PaillierLookup.key_gen(key_len, alpha_len)
    draws = rec.take()
    pk, n = keys["pk"], keys["pk"]["n"]
    # precompute_noise_table: 256 x generate_random_r(n), each randbelow(n)+1 with a gcd retry
    exps = []
    pending = None
    for kind, bound, value in draws:
        r = value + 1
        if math.gcd(r, n) == 1:
            exps.append(r)
    assert len(exps) == 256, len(exps)
    width = (pk["n_squared"].bit_length() + 7) // 8
    chunks = keys["message_chunks"]
    noise = keys["noise_table"]
    assert noise == oracle.noise_table(pk["g"], n, exps)
    g_digest = oracle.table_digest([keys["g_table"][i] for i in range(chunks)], width)
    rng = random.Random(1)
    plaintexts = [0, 1, 255, 256, n - 1, (1 << (2 * key_len - 8)) - 1]
    plaintexts = [m for m in plaintexts if m < n]
    plaintexts += [rng.randrange(n) for _ in range(8)]
    cases = []
    for m in plaintexts:
        rec.take()
        c = lookup.PaillierLookup.encrypt(m, pk, keys["g_table"], noise, chunks)
        d = rec.take()
        indices = [v for kind, bound, v in d if bound == 256][-14:]
        cases.append({"m": h(m), "indices": indices, "c": h(c),
                      "d": h(lookup.PaillierLookup.decrypt(c, keys))})
    sums = []
    for i in range(0, len(cases) - 1, 2):
        s = lookup.PaillierLookup.add(int(cases[i]["c"], 16), int(cases[i + 1]["c"], 16), pk)
        sums.append({"i": i, "j": i + 1, "c": h(s), "m": h(lookup.PaillierLookup.decrypt(s, keys))})
    # Hamming flow through the reference CPU client (hamming/paillier_lookup.py:56-242)
    import cuhepy.hamming.paillier_lookup as hpl
    hamming = []
    if hamming_vectors:
        client = hpl.PaillierLookupCPU(embed_len=512, key_len=key_len, alpha_len=alpha_len, skip_key_gen=True)
        client.keys = keys
        vrng = random.Random(1337)
        vectors = [[vrng.getrandbits(1) for _ in range(512)] for _ in range(hamming_vectors)]
        vectors[1] = [1 - b for b in vectors[0]]
        enc = []
        for v in vectors:
            rec.take()
            ct = client.encrypt(v)
            d = rec.take()
            enc.append({"bits": "".join(map(str, v)), "indices": [x for kind, bound, x in d if bound == 256][-14:],
                        "c": [h(x) for x in ct]})
        for i in range(1, len(vectors)):
            server = [int(PaillierLookupAdd) for PaillierLookupAdd in
                      [lookup.PaillierLookup.add(int(enc[0]["c"][0], 16), int(enc[i]["c"][0], 16), pk)]]
            dist = client.decode_hamming_client(server)
            hamming.append({"i": 0, "j": i, "c": h(server[0]), "distance": dist})
        hamming = {"vectors": enc, "pairs": hamming}
    return {
        "key_len": key_len,
        "alpha_len": alpha_len,
        "message_chunks": chunks,
        "pk": {k: h(v) for k, v in pk.items()},
        "sk": {k: h(v) for k, v in keys["sk"].items()},
        "noise_exponents": [h(r) for r in exps],
        "noise_table_sha256": oracle.table_digest(noise, width),
        "g_table_sha256": g_digest,
        "encrypt": cases,
        "add": sums,
        "hamming": hamming,
    }


class SeededSecrets(RecordingSecrets):
    """Seeded source whose randbelow/randbits match random.Random(seed)."""


def load_reference_native() -> None:
    """Make the compiled reference _bfv_rns (oracle/_ref) importable as the
    reference package's own extension module."""
    import importlib.util

    sys.path.insert(0, str(REPO / "oracle" / "_ref"))
    import _bfv_rns  # noqa: F401  (built by oracle/Makefile)

    sys.modules["cuhepy.bfv._cpu_ext._bfv_rns"] = _bfv_rns
    assert importlib.util.find_spec("cuhepy.bfv._cpu_ext") is not None


def bfv_fixture(bfv_scheme, n: int, t: int, bits: int, gadget: int, embed_len: int,
                vectors: list[list[int]], query: list[int], seed: int, backends: tuple[str, ...]) -> dict:
    """BFVClient (hamming/bfv.py) with rns_modulus=True: keys, a packed index, one
    query and encode_hamming_server_packed on several server backends."""
    import json as _json

    load_reference_native()
    import cuhepy.hamming.bfv as hb

    rec = SeededSecrets(seed)
    bfv_scheme.secrets = rec
    client = hb.BFVClient(embed_len, n, t, bits, gadget, response_modulus_bits=40, rns_modulus=True)
    q_wire = client.encrypt_vec_one(query)
    index = client.encrypt_vec_packed(vectors)
    results = {}
    for backend in backends:
        server = hb.BFVClient(skip_key_gen=True, server_backend=backend)
        server.load_config(_json.loads(client.stringify_config()))
        server.load_stringified_keys(client.stringify_pk())
        for compact in (False, True):
            res = server.encode_hamming_server_packed(q_wire, index, len(vectors), compact=compact)
            results[f"{backend}_{'compact' if compact else 'full'}"] = [[h(v) for v in ct] for ct in res]
    first = next(iter(results))
    for name, value in results.items():
        other = first if name.endswith("full") == first.endswith("full") else None
        if other and value != results[other]:
            raise AssertionError(f"backend {name} differs from {other}")
    compacted = [[int(v, 16) for v in ct] for ct in results[f"{backends[0]}_compact"]]
    distances = client.decode_hamming_client_packed(compacted, len(vectors))
    return {
        "seed": seed, "n": n, "t": t, "q_bits": bits, "gadget_bits": gadget, "embed_len": embed_len,
        "response_modulus_bits": 40, "eta": 21,
        "vectors": ["".join(map(str, v)) for v in vectors], "query": "".join(map(str, query)),
        "key_id": client._pk()["key_id"],
        "query_wire": [h(v) for v in q_wire], "index_wire": [[h(v) for v in ct] for ct in index],
        "results": results, "distances": distances,
    }


def main() -> None:
    parser = argparse.ArgumentParser()
    parser.add_argument("--reference", default=os.environ.get("CUHEPY_REFERENCE") or "/root/reference", type=Path)
    parser.add_argument("--only", default="")
    args = parser.parse_args()
    scheme, lookup, bfv_scheme, number = setup(args.reference)
    small_vectors = [[0, 1, 0], [1, 0, 1], [0, 0, 0]] * 13
    rng = random.Random(1337)
    mid_vectors = [[rng.getrandbits(1) for _ in range(20)] for _ in range(77)]
    mid_query = [rng.getrandbits(1) for _ in range(20)]
    all_backends = ("residue", "native", "rns", "optimized", "reference")
    jobs = {
        "paillier_512": lambda: paillier_fixture(scheme, number, 512),
        "paillier_1024": lambda: paillier_fixture(scheme, number, 1024),
        "lookup_512": lambda: lookup_fixture(lookup, number, 512, 280, 0),
        "lookup_1024": lambda: lookup_fixture(lookup, number, 1024, 280, 6),
    }
    for bits, gadget in ((60, 4), (120, 15), (180, 30), (180, 61), (480, 127)):
        jobs[f"bfv_n16_q{bits}_g{gadget}"] = (
            lambda b=bits, g=gadget: bfv_fixture(bfv_scheme, 16, 97, b, g, 3, small_vectors, [0, 1, 0],
                                                 100 + b + g, all_backends))
    jobs["bfv_n256_q180_g30"] = lambda: bfv_fixture(
        bfv_scheme, 256, 7681, 180, 30, 20, mid_vectors, mid_query, 4242, ("residue", "native", "reference"))
    for name, job in jobs.items():
        if args.only and args.only not in name:
            continue
        data = job()
        path = HERE / f"{name}.json"
        path.write_text(json.dumps(data, indent=0, sort_keys=True))
        print(f"wrote {path} ({path.stat().st_size} bytes)")


if __name__ == "__main__":
    main()
