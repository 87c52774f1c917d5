"""Record the reference's own Python BFV layer driving its native module.

Run where the reference project is present (read-only):

    python tests/golden/make_bfv_transcript.py --reference <path of the reference tree>

The reference package is imported unmodified (through the test-only shims of
tests/golden/shims, exactly as make_golden.py does).  Its compiled native
module ``cuhepy.bfv._cpu_ext._bfv_rns`` is the reference's own C++ backend
built by oracle/Makefile (oracle/_ref), wrapped in a recorder that writes down
every call the Python layer makes -- function, arguments, result -- with the
module's opaque handles (rings, keys, servers) replaced by numbered handles.

Flows recorded, each with the reference's seeded client:
  * ``BFVClient(server_backend="residue")`` (rns_modulus=True):
    ``encode_hamming_server_packed`` compact and full, ``encode_hamming_server``,
    a profiled native search, ``cache_info`` -- hamming/bfv.py:309-374 over
    ``BFVNativeServer`` (bfv/native.py:16-118);
  * the default prime-q ring (rns_modulus=False) with
    ``server_backend="native"``, the same calls;
  * ``server_backend="rns"`` (``BFVEvaluator`` over ``BFVRNSArithmetic``,
    bfv/evaluator.py:94-120, bfv/rns.py:27-133): the tile circuits run through
    ``hamming_tile`` and the merge tree's rotations through ``rotate_rows``.

tests/test_bfv_transcript_gpu.py replays every call against the drop-in
``cuhepy_b200.bfv._bfv_rns`` on the device and requires identical results, so
the reference's Python layer, given the drop-in, receives exactly what it
received from its own backend.  Written to tests/golden/bfv_transcript.json.
"""

from __future__ import annotations

import argparse
import base64
import json
import os
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]
sys.path.insert(0, str(HERE))

import make_golden  # noqa: E402


class Recorder:
    """Stands in for the native module and logs every call."""

    FUNCTIONS = ("create_ring", "ring_info", "compile_key", "key_bytes", "apply_key", "ring_product", "multiply",
                 "rotate_rows", "hamming_tile", "create_server", "server_bytes", "packed_search",
                 "profile_hamming_tile", "profile_packed_search")

    def __init__(self, native) -> None:
        self._native = native
        self.ABI_VERSION = native.ABI_VERSION
        self.calls: list[dict] = []
        self._handles: dict[int, int] = {}
        for name in self.FUNCTIONS:
            setattr(self, name, self._wrap(name))

    def _encode(self, value):
        if isinstance(value, bytes):
            return {"b64": base64.b64encode(value).decode()}
        if isinstance(value, (tuple, list)):
            return {"tuple" if isinstance(value, tuple) else "list": [self._encode(v) for v in value]}
        if isinstance(value, dict):
            return {"dict": {str(k): self._encode(v) for k, v in value.items()}}
        if value is None or isinstance(value, (bool, int, float, str)):
            return value
        handle = self._handles.get(id(value))
        if handle is None:
            handle = len(self._handles)
            self._handles[id(value)] = handle
            self._keep = getattr(self, "_keep", []) + [value]  # ids stay unique while recording
        return {"handle": handle}

    def _wrap(self, name):
        fn = getattr(self._native, name)

        def call(*args):
            out = fn(*args)
            self.calls.append({"fn": name, "args": [self._encode(a) for a in args], "out": self._encode(out)})
            return out

        return call

    def profile_call(self, callback):
        return self._native.profile_call(callback)


def run_case(hb, bfv_scheme, rec: Recorder, *, backend: str, rns_modulus: bool, n: int, t: int, bits: int,
             gadget: int, embed: int, vectors, query, seed: int) -> dict:
    rec.calls = []
    bfv_scheme.secrets = make_golden.SeededSecrets(seed)
    client = hb.BFVClient(embed, n, t, bits, gadget, response_modulus_bits=40, rns_modulus=rns_modulus)
    q_wire = client.encrypt_vec_one(query)
    index = client.encrypt_vec_packed(vectors)
    server = hb.BFVClient(skip_key_gen=True, server_backend=backend)
    server.load_config(json.loads(client.stringify_config()))
    server.load_stringified_keys(client.stringify_pk())
    full = server.encode_hamming_server_packed(q_wire, index, len(vectors), compact=False)
    compact = server.encode_hamming_server_packed(q_wire, index, len(vectors), compact=True)
    single = server.encode_hamming_server(q_wire, index[0])
    profile = {}
    if backend in ("native", "residue"):
        again = server._native().search(q_wire, index, len(vectors), compact=True, profile=profile)
        assert again == compact
    extra = {}
    if backend == "rns":
        # the evaluator's own operations over BFVRNSArithmetic: exact tensor
        # with scale-and-round (multiply) + relinearization (apply_key),
        # plaintext products (ring_product), xor, subtraction and a rotation
        ev, pk = server._evaluator(), server._pk()
        q_ct = bfv_scheme.BFV.ciphertext_from_ints(q_wire, pk)
        t_ct = bfv_scheme.BFV.ciphertext_from_ints(index[0], pk)
        ones = bfv_scheme.BFV.batch_encode([1] * n, client.params)
        slots = lambda ct: bfv_scheme.BFV.batch_decode(bfv_scheme.BFV.decrypt(ct, client.keys), client.params)
        extra = {"square": slots(ev.multiply(q_ct, q_ct)), "xor": slots(ev.xor(q_ct, t_ct)),
                 "times_ones": slots(ev.multiply_plain(q_ct, ones)),
                 "rotated": slots(ev.rotate_rows(ev.subtract(q_ct, t_ct), client.lanes_per_row))}
    info = server._evaluator().cache_info()
    distances = client.decode_hamming_client_packed(compact, len(vectors))
    first = client.decode_hamming_client_one(single)
    return {
        "backend": backend, "rns_modulus": rns_modulus, "n": n, "t": t, "q_bits": bits, "gadget_bits": gadget,
        "embed_len": embed, "seed": seed, "vector_count": len(vectors),
        "calls": rec.calls,
        "responses": {"full": [[format(v, "x") for v in ct] for ct in full],
                      "compact": [[format(v, "x") for v in ct] for ct in compact],
                      "single": [format(v, "x") for v in single]},
        "distances": distances, "single_distance": first,
        "profiled_phases": sorted(profile), "cache_info_keys": sorted(info),
        "evaluator_slots": extra,
    }


def main() -> None:
    parser = argparse.ArgumentParser()
    parser.add_argument("--reference", default=os.environ.get("CUHEPY_REFERENCE"), type=Path,
                        help="root of the reference tree (default: $CUHEPY_REFERENCE)")
    args = parser.parse_args()
    if args.reference is None:
        parser.error("give --reference or set CUHEPY_REFERENCE")
    scheme, lookup, bfv_scheme, number = make_golden.setup(args.reference)
    make_golden.load_reference_native()
    native = sys.modules["cuhepy.bfv._cpu_ext._bfv_rns"]
    rec = Recorder(native)
    sys.modules["cuhepy.bfv._cpu_ext._bfv_rns"] = rec
    import cuhepy.bfv._cpu_ext as ext
    ext._bfv_rns = rec
    import cuhepy.hamming.bfv as hb

    small = [[0, 1, 0], [1, 0, 1], [0, 0, 0], [1, 1, 1]] * 9 + [[1, 0, 0], [0, 1, 1], [1, 1, 0]]
    cases = [
        dict(backend="residue", rns_modulus=True, n=16, t=97, bits=180, gadget=30, embed=3, vectors=small,
             query=[0, 1, 1], seed=501),
        dict(backend="native", rns_modulus=False, n=16, t=97, bits=180, gadget=30, embed=3, vectors=small,
             query=[1, 1, 0], seed=502),
        dict(backend="rns", rns_modulus=True, n=16, t=97, bits=120, gadget=15, embed=3, vectors=small[:13],
             query=[1, 0, 1], seed=503),
    ]
    out = {"reference_abi": native.ABI_VERSION, "cases": [run_case(hb, bfv_scheme, rec, **c) for c in cases]}
    for case in out["cases"]:
        vectors = [c for c in cases if c["seed"] == case["seed"]][0]
        want = [sum(a != b for a, b in zip(v, vectors["query"])) for v in vectors["vectors"]]
        assert case["distances"] == want, case["backend"]
    path = HERE / "bfv_transcript.json"
    path.write_text(json.dumps(out, indent=0, sort_keys=True))
    print(f"wrote {path} ({path.stat().st_size} bytes, "
          f"{sum(len(c['calls']) for c in out['cases'])} calls)")


if __name__ == "__main__":
    main()
