"""Shared helpers for the BFV parity tests (inputs, packing, reference checker)."""

from __future__ import annotations

import importlib.util
import random
import sys
from pathlib import Path

import numpy as np

from oracle import bfv as ob

REPO = Path(__file__).resolve().parents[1]


class Seeded:
    def __init__(self, seed):
        self._rng = random.Random(seed)

    def randbelow(self, n):
        return self._rng.randrange(n)

    def randbits(self, k):
        return self._rng.getrandbits(k)


def fixed(poly, q):
    """Fixed-width little-endian coefficient bytes (bindings.cpp:43-82)."""
    width = (q.bit_length() + 7) // 8
    return b"".join(int(c).to_bytes(width, "little") for c in poly)


def unfixed(data, q, n):
    width = (q.bit_length() + 7) // 8
    return [int.from_bytes(data[i * width:(i + 1) * width], "little") for i in range(n)]


def packed(poly, bits):
    return ob.pack_poly(poly, bits)


def reference_native():
    """The reference's compiled _bfv_rns (oracle/_ref), or None when absent."""
    ref_dir = REPO / "oracle" / "_ref"
    if not any(ref_dir.glob("_bfv_rns*.so")):
        return None
    if "cuhe_ref_bfv_rns" in sys.modules:
        return sys.modules["cuhe_ref_bfv_rns"]
    path = next(ref_dir.glob("_bfv_rns*.so"))
    spec = importlib.util.spec_from_file_location("_bfv_rns", path)
    module = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(module)
    sys.modules["cuhe_ref_bfv_rns"] = module
    return module


def random_keys(n, q, digits, count, seed):
    """Uniform (not RLWE-distributed) gadget keys: exercises every arithmetic
    path with the full range of coefficients."""
    rng = random.Random(seed)
    return [tuple((tuple(rng.randrange(q) for _ in range(n)), tuple(rng.randrange(q) for _ in range(n)))
                  for _ in range(digits)) for _ in range(count)]


def key_bytes(key, q):
    return tuple((fixed(b, q), fixed(a, q)) for b, a in key)


def _below_q_bits(rng, rows, q):
    """rows x bits(q) little-endian bit matrix of uniform draws, those at or
    above q mapped below 2^(bits-1) by clearing their top bit."""
    bits = q.bit_length()
    x = rng.integers(0, 2, size=(rows, bits), dtype=np.uint8)
    qb = np.array([(q >> i) & 1 for i in range(bits)], dtype=np.uint8)
    rev = (x != qb)[:, ::-1]
    first = rev.argmax(axis=1)
    ge = ~rev.any(axis=1) | (x[:, ::-1][np.arange(rows), first] == 1)
    x[ge, bits - 1] = 0
    return x


def random_fixed_poly(rng, n, q):
    """One canonical polynomial (coefficients < q) as fixed-width bytes."""
    bits = q.bit_length()
    width = (bits + 7) // 8
    x = _below_q_bits(rng, n, q)
    padded = np.zeros((n, 8 * width), dtype=np.uint8)
    padded[:, :bits] = x
    return np.packbits(padded, axis=1, bitorder="little").tobytes()


def random_packed_poly(rng, n, q):
    """One canonical polynomial as the bit-packed wire (bits(q) per coefficient)."""
    x = _below_q_bits(rng, n, q).reshape(-1)
    return np.packbits(x, bitorder="little").tobytes()


def with_head(poly, q, values):
    """A packed polynomial with its first len(values) coefficients replaced."""
    bits = q.bit_length()
    count = len(values)
    span = (count * bits + 7) // 8
    head = int.from_bytes(poly[:span], "little")
    keep = head >> (count * bits)
    new = 0
    for i, v in enumerate(values):
        new |= int(v) << (i * bits)
    return (new | (keep << (count * bits))).to_bytes(span, "little") + poly[span:]


def regenerate_fixture(data):
    params = ob.Params(data["n"], data["t"], data["q_bits"], data["gadget_bits"], data["eta"])
    layout = ob.Layout(params.n, data["embed_len"])
    rng = Seeded(data["seed"])
    keys = ob.key_gen(params, layout.rotation_steps(), rng)
    query_bits = [int(b) for b in data["query"]]
    vectors = [[int(b) for b in v] for v in data["vectors"]]
    query = ob.encrypt(ob.batch_encode(layout.query_slots(query_bits), params.n, params.t), keys, rng)
    index = [ob.encrypt(ob.batch_encode(s, params.n, params.t), keys, rng) for s in layout.index_slots(vectors)]
    return params, layout, keys, query, index, vectors
