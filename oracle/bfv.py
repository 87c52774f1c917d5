"""CPU oracle for the BFV packed Hamming evaluator (residue / RNS-modulus form).

TEST INFRASTRUCTURE ONLY: imported by ``tests/``, ``__graft_entry__.smoke()``
and the CPU-baseline leg of ``bench.py`` as the checker; never by the product.

A restatement over CPython integers of the reference's BFV scheme and of the
public-key Hamming search it evaluates.  Randomness is read from a
``secrets``-like object passed in by the caller, with the same calls in the
same order as the reference, so that a recorded / seeded source reproduces the
reference's keys and ciphertexts exactly.

Reference files (paths inside the cuhepy project):
  src/cuhepy/bfv/scheme.py           parameters, key_gen, encrypt/decrypt,
                                     multiply, relinearize, rotate, wire v1
  src/cuhepy/bfv/evaluator.py        the "reference" backend's tile circuit
  src/cuhepy/hamming/bfv.py          packed layout, masks, merge tree
  src/cuhepy/bfv/_cpu_ext/bfv_server.h   merge order and compaction (the
                                     residue server returns identical results)
"""

from __future__ import annotations

import hashlib
import json
from dataclasses import dataclass, field

from oracle.gmp import mul as _mul


# --------------------------------------------------------------------------
# parameters: scheme.py:186-216
# --------------------------------------------------------------------------

def is_prime(x: int) -> bool:
    """Deterministic Miller-Rabin for x < 3.3e24; probabilistic above."""
    if x < 2:
        return False
    small = (2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37)
    for p in small:
        if x % p == 0:
            return x == p
    d, s = x - 1, 0
    while d % 2 == 0:
        d //= 2
        s += 1
    bases = small if x < 3317044064679887385961981 else small + (41, 43, 47, 53, 59, 61, 67, 71, 73, 79, 83, 89)
    for a in bases:
        y = pow(a, d, x)
        if y in (1, x - 1):
            continue
        for _ in range(s - 1):
            y = y * y % x
            if y == x - 1:
                break
        else:
            return False
    return True


def rns_primes(n: int, bits: int) -> tuple[int, ...]:
    """scheme.py:196-216: 60-bit primes p = 1 mod 2N searched downward from 2^60-2N+1."""
    if bits < 60 or bits > 480 or bits % 60:
        raise ValueError("rns modulus bits must be a multiple of 60 in [60, 480]")
    out, candidate = [], (1 << 60) - 2 * n + 1
    for _ in range(bits // 60):
        while not is_prime(candidate):
            candidate -= 2 * n
        out.append(candidate)
        candidate -= 2 * n
    return tuple(out)


def coefficient_modulus(bits: int) -> int:
    """scheme.py:186-193: largest prime below 2^bits."""
    candidate = (1 << bits) - 1
    while not is_prime(candidate):
        candidate -= 2
    return candidate


@dataclass(frozen=True)
class Params:
    n: int = 8192
    t: int = 65537
    q_bits: int = 180
    gadget_bits: int = 30
    eta: int = 21

    @property
    def primes(self) -> tuple[int, ...]:
        return rns_primes(self.n, self.q_bits)

    @property
    def q(self) -> int:
        out = 1
        for p in self.primes:
            out *= p
        return out

    @property
    def digits(self) -> int:
        return (self.q_bits + self.gadget_bits - 1) // self.gadget_bits


# --------------------------------------------------------------------------
# polynomial arithmetic over Z[X]/(X^N+1): scheme.py:100-136
# --------------------------------------------------------------------------

def _pack(values, width):
    if len(values) == 1:
        return int(values[0])
    half = len(values) // 2
    return _pack(values[:half], width) | (_pack(values[half:], width) << (half * width))


def _unpack(x, width, count):
    if count == 1:
        return [x]
    half = count // 2
    return _unpack(x & ((1 << (half * width)) - 1), width, half) + _unpack(x >> (half * width), width, count - half)


def poly_product(lhs, rhs):
    """Exact negacyclic product of nonnegative coefficient vectors (Kronecker)."""
    n = len(lhs)
    width = max(max(int(c).bit_length() for c in lhs), 1) + max(max(int(c).bit_length() for c in rhs), 1)
    width += n.bit_length()
    a = _pack([int(c) for c in lhs], width)
    b = a if lhs is rhs else _pack([int(c) for c in rhs], width)
    coeffs = _unpack(_mul(a, b), width, 2 * n)
    return [coeffs[i] - coeffs[i + n] for i in range(n)]


def ring_product(lhs, rhs, q):
    return [c % q for c in poly_product(lhs, rhs)]


def automorphism(poly, g, q):
    """X -> X^g (scheme.py:129-136)."""
    n = len(poly)
    out = [0] * n
    for i, v in enumerate(poly):
        pos = (i * g) % (2 * n)
        out[pos % n] = (v if pos < n else -v) % q
    return out


def round_div(value, divisor):
    """scheme.py:100-102: nearest integer, ties toward +infinity."""
    return (2 * value + divisor) // (2 * divisor)


# --------------------------------------------------------------------------
# batching: scheme.py:139-183, 371-406
# --------------------------------------------------------------------------

def _ntt(values, root, modulus):
    result = list(values)
    n = len(result)
    j = 0
    for i in range(1, n):
        bit = n >> 1
        while j & bit:
            j ^= bit
            bit >>= 1
        j ^= bit
        if i < j:
            result[i], result[j] = result[j], result[i]
    length = 2
    while length <= n:
        stride = pow(root, n // length, modulus)
        for start in range(0, n, length):
            w = 1
            for off in range(length // 2):
                u = result[start + off]
                v = result[start + off + length // 2] * w % modulus
                result[start + off] = (u + v) % modulus
                result[start + off + length // 2] = (u - v) % modulus
                w = w * stride % modulus
        length *= 2
    return result


_PLAN: dict = {}


def batch_plan(n, t):
    key = (n, t)
    if key not in _PLAN:
        c = 2
        while True:
            psi = pow(c, (t - 1) // (2 * n), t)
            if pow(psi, n, t) == t - 1:
                break
            c += 1
        twists = [pow(psi, i, t) for i in range(n)]
        exps = [pow(3, i, 2 * n) for i in range(n // 2)]
        order = [(e - 1) // 2 for e in exps] + [((-e) % (2 * n) - 1) // 2 for e in exps]
        _PLAN[key] = (psi * psi % t, twists, order)
    return _PLAN[key]


def batch_encode(slots, n, t):
    root, twists, order = batch_plan(n, t)
    ev = [0] * n
    for pos, v in zip(order, slots):
        ev[pos] = int(v)
    coeffs = _ntt(ev, pow(root, -1, t), t)
    inv_n = pow(n, -1, t)
    return [c * inv_n * pow(tw, -1, t) % t for c, tw in zip(coeffs, twists)]


def batch_decode(poly, n, t):
    root, twists, order = batch_plan(n, t)
    ev = _ntt([int(c) * tw % t for c, tw in zip(poly, twists)], root, t)
    return [ev[i] for i in order]


# --------------------------------------------------------------------------
# keys and encryption: scheme.py:236-361, 426-473
# --------------------------------------------------------------------------

def small_poly(n, eta, q, rng):
    return [(rng.randbits(eta).bit_count() - rng.randbits(eta).bit_count()) % q for _ in range(n)]


def ternary_poly(n, q, rng):
    return [(rng.randbelow(3) - 1) % q for _ in range(n)]


def key_gen(params: Params, rotation_steps, rng) -> dict:
    """scheme.py:292-361 (same random draws in the same order)."""
    n, q = params.n, params.q
    s = ternary_poly(n, q, rng)
    a = [rng.randbelow(q) for _ in range(n)]
    error = small_poly(n, params.eta, q, rng)
    a_s = ring_product(a, s, q)
    b = [(e - v) % q for e, v in zip(error, a_s)]

    def switch_key(source):
        out = []
        for shift in range(0, params.q_bits, params.gadget_bits):
            a_i = [rng.randbelow(q) for _ in range(n)]
            e_i = small_poly(n, params.eta, q, rng)
            prod = ring_product(a_i, s, q)
            b_i = [((v << shift) - av + e) % q for v, av, e in zip(source, prod, e_i)]
            out.append((b_i, a_i))
        return out

    relin = switch_key(ring_product(s, s, q))
    galois = {}
    for steps in rotation_steps:
        g = pow(3, steps % (n // 2), 2 * n)
        if g != 1 and g not in galois:
            galois[g] = switch_key(automorphism(s, g, q))
    return {"params": params, "q": q, "b": b, "a": a, "s": s, "relin": relin, "galois": galois}


def encrypt(plain, keys, rng):
    """scheme.py:426-444."""
    params, q = keys["params"], keys["q"]
    n = params.n
    u = ternary_poly(n, q, rng)
    e0, e1 = small_poly(n, params.eta, q, rng), small_poly(n, params.eta, q, rng)
    bu, au = ring_product(keys["b"], u, q), ring_product(keys["a"], u, q)
    delta = q // params.t
    c0 = [(v + e + delta * m) % q for v, e, m in zip(bu, e0, plain)]
    c1 = [(v + e) % q for v, e in zip(au, e1)]
    return (c0, c1)


def decrypt(ct, keys, modulus=None):
    """scheme.py:447-473: round(t * (c0 + c1*s) / q) mod t."""
    q = modulus or keys["q"]
    t = keys["params"].t
    big = keys["q"]
    s = [(c if c <= big // 2 else c - big) % q for c in keys["s"]]  # centred secret (scheme.py:360)
    phase = ct[-1]
    for poly in reversed(ct[:-1]):
        phase = [(x + y) % q for x, y in zip(ring_product(phase, s, q), poly)]
    return [round_div(t * c, q) % t for c in phase]


# --------------------------------------------------------------------------
# evaluation: scheme.py:535-626 (the residue server computes the same values)
# --------------------------------------------------------------------------

def switch(poly, key, q, bits):
    """Gadget dot product sum_i digit_i(poly) * key_i (scheme.py:535-548)."""
    n = len(poly)
    mask = (1 << bits) - 1
    acc = [[0] * n, [0] * n]
    for i, pair in enumerate(key):
        digits = [(c >> (i * bits)) & mask for c in poly]
        for k in range(2):
            prod = poly_product(digits, pair[k])
            acc[k] = [x + y for x, y in zip(acc[k], prod)]
    return [c % q for c in acc[0]], [c % q for c in acc[1]]


def square_relin(ct, keys):
    """multiply(ct, ct) with exact signed scale-and-round, then relinearize (scheme.py:571-600)."""
    q, t = keys["q"], keys["params"].t
    a0, a1 = ct
    d0 = poly_product(a0, a0)
    d2 = poly_product(a1, a1)
    cross = poly_product(a0, a1)
    d1 = [2 * c for c in cross]
    c0, c1, c2 = ([round_div(t * c, q) % q for c in poly] for poly in (d0, d1, d2))
    k0, k1 = switch(c2, keys["relin"], q, keys["params"].gadget_bits)
    return ([(x + y) % q for x, y in zip(c0, k0)], [(x + y) % q for x, y in zip(c1, k1)])


def rotate(ct, g, keys):
    """rotate_rows by Galois exponent g (scheme.py:610-626)."""
    q = keys["q"]
    if g == 1:
        return ct
    c0, c1 = (automorphism(c, g, q) for c in ct)
    k0, k1 = switch(c1, keys["galois"][g], q, keys["params"].gadget_bits)
    return ([(x + y) % q for x, y in zip(c0, k0)], k1)


def add(x, y, q):
    return tuple([(a + b) % q for a, b in zip(p, r)] for p, r in zip(x, y))


def multiply_plain(ct, plain, q):
    return tuple(ring_product(c, plain, q) for c in ct)


def compact(ct, q, target):
    """bfv_server.h:142-151 == scheme.py:628-652: floor((2*target*c + q) / (2q)) mod target."""
    return tuple([(2 * target * c + q) // (2 * q) % target for c in poly] for poly in ct)


@dataclass
class Layout:
    """hamming/bfv.py:108-138: packed layout for one embedding length."""
    n: int
    embed_len: int
    padded: int = field(init=False)
    lanes: int = field(init=False)
    capacity: int = field(init=False)

    def __post_init__(self):
        self.padded = 1 << (self.embed_len - 1).bit_length()
        self.lanes = self.n // (2 * self.padded)
        self.capacity = 2 * self.lanes

    def rotation_steps(self):
        return [sign * self.lanes * (1 << i) for i in range(self.padded.bit_length() - 1) for sign in (1, -1)]

    def left(self):
        return [pow(3, (self.lanes << i) % (self.n // 2), 2 * self.n) for i in range(self.padded.bit_length() - 1)]

    def right(self):
        return [pow(3, (self.n // 2 - (self.lanes << i)) % (self.n // 2), 2 * self.n)
                for i in range(self.padded.bit_length() - 1)]

    def query_slots(self, bits):
        row = [int(b) for b in bits for _ in range(self.lanes)]
        row.extend([0] * ((self.padded - self.embed_len) * self.lanes))
        return row + row

    def index_slots(self, vectors):
        tiles = []
        for start in range(0, len(vectors), self.capacity):
            slots = [0] * self.n
            for lane, vec in enumerate(vectors[start:start + self.capacity]):
                row, col = divmod(lane, self.lanes)
                for d, bit in enumerate(vec):
                    slots[row * (self.n // 2) + d * self.lanes + col] = int(bit)
            tiles.append(slots)
        return tiles

    def mask_slots(self, count):
        mask = [0] * self.n
        for lane in range(count):
            row, col = divmod(lane, self.lanes)
            mask[row * (self.n // 2) + col] = 1
        return mask


def tile_circuit(query, tile, keys, layout: Layout, count):
    """ResidueServer::tile (bfv_residue.h:192-215) / BFVEvaluator.hamming_tile."""
    q, params = keys["q"], keys["params"]
    diff = tuple([(a - b) % q for a, b in zip(x, y)] for x, y in zip(query, tile))
    dist = square_relin(diff, keys)
    for g in layout.left():
        dist = add(dist, rotate(dist, g, keys), q)
    mask = batch_encode(layout.mask_slots(count), params.n, params.t)
    return multiply_plain(dist, mask, q)


def search(query, index, vector_count, keys, layout: Layout, compact_to: int | None):
    """merge_hamming_tiles (bfv_server.h:15-45) over tile_circuit, then compaction."""
    q = keys["q"]
    tiles = len(index)
    right = layout.right()
    out = []
    for start in range(0, tiles, layout.padded):
        stack = []
        for at in range(start, min(start + layout.padded, tiles)):
            count = min(layout.capacity, vector_count - at * layout.capacity)
            result = tile_circuit(query, index[at], keys, layout, count)
            size, level = 1, 0
            while stack and stack[-1][1] == size:
                rotated = rotate(result, right[level], keys)
                result = add(stack.pop()[0], rotated, q)
                size *= 2
                level += 1
            stack.append((result, size))
        result = stack.pop()[0]
        while stack:
            size = stack[-1][1]
            level = size.bit_length() - 1
            rotated = rotate(result, right[level], keys)
            result = add(stack.pop()[0], rotated, q)
        out.append(compact(result, q, compact_to) if compact_to else result)
    return out


# --------------------------------------------------------------------------
# wire: packed_wire.h / scheme.py:669-702
# --------------------------------------------------------------------------

def pack_poly(poly, bits):
    """Little-endian bit packing, `bits` bits per coefficient (packed_wire.h:41-60)."""
    value = _pack([int(c) for c in poly], bits)
    return value.to_bytes((len(poly) * bits + 7) // 8, "little")


def unpack_poly(data, bits, n):
    value = int.from_bytes(data, "little")
    return _unpack(value, bits, n)


def key_id(params: Params, b, a) -> str:
    """scheme.py:249-255 for an RNS-modulus parameter set."""
    d = {"poly_modulus_degree": params.n, "plain_modulus": params.t, "coeff_modulus_bits": params.q_bits,
         "decomposition_bits": params.gadget_bits, "error_eta": params.eta, "rns_modulus": True}
    digest = hashlib.sha256(json.dumps(d, sort_keys=True).encode())
    width = (params.q_bits + 7) // 8
    for poly in (b, a):
        for c in poly:
            digest.update(int(c).to_bytes(width, "little"))
    return digest.hexdigest()
