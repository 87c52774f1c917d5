"""The reference's own Python BFV layer, replayed on the drop-in module.

tests/golden/bfv_transcript.json records every call that the reference's
unmodified Python layer -- ``BFVClient`` with the ``residue``, ``native`` and
``rns`` server backends, ``BFVNativeServer`` (bfv/native.py:16-118) and
``BFVEvaluator`` over ``BFVRNSArithmetic`` (bfv/evaluator.py:94-318,
bfv/rns.py:27-133) -- made into its native module ``_bfv_rns``, with the
results the reference's C++ backend returned (generator:
tests/golden/make_bfv_transcript.py).  Replaying each call in order against
``cuhepy_b200.bfv._bfv_rns`` must give the same result, so that layer,
imported with the drop-in in place of its backend, receives exactly what its
own backend gave it: the same rings, keys, tile circuits, rotations,
products, packed searches and responses.  Integer work: equality is exact,
except the informational fields (``ring_info``'s compiler/GMP strings and
table sizes, ``key_bytes``/``server_bytes`` payload sizes, profile timings),
whose layouts differ by design.
"""

import base64
import json

import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu

RING_FIELDS = ("primes", "switch_prime_count", "residue_prime_count", "kernel_level", "fast_arithmetic")


def _decode(value, handles):
    if isinstance(value, dict):
        if "b64" in value:
            return base64.b64decode(value["b64"])
        if "tuple" in value:
            return tuple(_decode(v, handles) for v in value["tuple"])
        if "list" in value:
            return [_decode(v, handles) for v in value["list"]]
        if "dict" in value:
            return {k: _decode(v, handles) for k, v in value["dict"].items()}
        if "handle" in value:
            return handles[value["handle"]]
    return value


def _cases():
    data = json.loads((GOLDEN / "bfv_transcript.json").read_text())
    return data["cases"]


@pytest.mark.parametrize("case", _cases(), ids=lambda c: f"{c['backend']}_n{c['n']}_q{c['q_bits']}")
def test_reference_python_layer_calls_replay_identically(case):
    from cuhepy_b200.bfv import _bfv_rns as m

    assert m.ABI_VERSION == 4
    handles = {}
    for i, call in enumerate(case["calls"]):
        fn, recorded = call["fn"], call["out"]
        args = [_decode(a, handles) for a in call["args"]]
        got = getattr(m, fn)(*args)
        where = f"call {i}: {fn}"
        if isinstance(recorded, dict) and "handle" in recorded:
            handles[recorded["handle"]] = got
        elif fn == "ring_info":
            want = _decode(recorded, handles)
            assert {k: got[k] for k in RING_FIELDS} == {k: (tuple(want[k]) if k == "primes" else want[k])
                                                       for k in RING_FIELDS}, where
        elif fn in ("key_bytes", "server_bytes"):
            assert isinstance(got, int) and got > 0, where
        elif fn.startswith("profile_"):
            assert got[0] == _decode(recorded, handles)[0], where
            assert isinstance(got[1], dict), where
        else:
            assert got == _decode(recorded, handles), where
    assert case["distances"] and all(0 <= d <= case["embed_len"] for d in case["distances"])
