"""Drop-in for the reference's native module ``_bfv_rns`` (ABI_VERSION 4).

Same function names, argument meanings, buffer formats and error mapping as
src/cuhepy/bfv/_cpu_ext/bindings.cpp:405-433 (``ValueError`` for invalid
arguments, ``TypeError`` for non-bytes buffers, ``RuntimeError`` otherwise);
the arithmetic runs on the B200 through libcuhe_bfv_b200.so.  Rings are
residue rings (Q a product of the first 60-bit NTT primes) or native rings
(residue=False: any odd q up to 512 bits, exact products).  The C ABI
releases no Python state, so the GIL is dropped during every call (ctypes
releases it for foreign calls).
"""

from __future__ import annotations

import ctypes
import time
from typing import Any

from cuhepy_b200 import _native

ABI_VERSION = 4
PHASES = ("tensor", "relinearize", "rotate", "mask", "merge", "output")

_u8p = ctypes.POINTER(ctypes.c_uint8)
_u64p = ctypes.POINTER(ctypes.c_uint64)
_vp = ctypes.c_void_p

BFV_SIGNATURES: dict[str, tuple] = {
    "cuhe_bfv_last_error": (ctypes.c_char_p, []),
    "cuhe_bfv_create_ring": (ctypes.c_int, [ctypes.c_uint64, ctypes.c_char_p, ctypes.c_uint64, ctypes.c_int,
                                            ctypes.c_int, ctypes.c_uint64, ctypes.c_int, ctypes.POINTER(_vp)]),
    "cuhe_bfv_ring_release": (None, [_vp]),
    "cuhe_bfv_ring_info": (ctypes.c_int, [_vp, _u64p, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                          ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int), _u64p, _u64p,
                                          ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]),
    "cuhe_bfv_compile_key": (ctypes.c_int, [_vp, ctypes.c_char_p, ctypes.c_uint64, ctypes.POINTER(_vp)]),
    "cuhe_bfv_key_release": (None, [_vp]),
    "cuhe_bfv_key_bytes": (ctypes.c_uint64, [_vp]),
    "cuhe_bfv_apply_key": (ctypes.c_int, [_vp, ctypes.c_char_p, _vp]),
    "cuhe_bfv_ring_product": (ctypes.c_int, [_vp, ctypes.c_char_p, ctypes.c_char_p, _vp]),
    "cuhe_bfv_multiply": (ctypes.c_int, [_vp, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_uint64, _vp]),
    "cuhe_bfv_rotate_rows": (ctypes.c_int, [_vp, ctypes.c_char_p, ctypes.c_uint64, _vp]),
    "cuhe_bfv_hamming_tile": (ctypes.c_int, [_vp, ctypes.c_char_p, ctypes.c_char_p, _u64p, ctypes.POINTER(_vp),
                                             ctypes.c_uint64, ctypes.c_char_p, ctypes.c_uint64, _vp]),
    "cuhe_bfv_create_server": (ctypes.c_int, [_vp, _u64p, ctypes.POINTER(_vp), ctypes.c_uint64, ctypes.c_uint64,
                                              ctypes.c_uint64, ctypes.c_char_p, ctypes.POINTER(_vp)]),
    "cuhe_bfv_server_release": (None, [_vp]),
    "cuhe_bfv_server_bytes": (ctypes.c_uint64, [_vp]),
    "cuhe_bfv_server_layout": (ctypes.c_int, [_vp, _u64p, _u64p, _u64p, _u64p, _u64p]),
    "cuhe_bfv_packed_search": (ctypes.c_int, [_vp, ctypes.c_char_p, _vp, ctypes.c_uint64, ctypes.c_uint64,
                                              ctypes.c_int, _vp, ctypes.c_uint64, _u64p]),
    "cuhe_bfv_last_profile": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_double), ctypes.c_int]),
    "cuhe_bfv_upload_index": (ctypes.c_int, [_vp, _vp, ctypes.c_uint64, ctypes.POINTER(_vp)]),
    "cuhe_bfv_index_release": (None, [_vp]),
    "cuhe_bfv_search_index": (ctypes.c_int, [_vp, _vp, ctypes.c_char_p, ctypes.c_uint64, ctypes.c_int, _vp,
                                             ctypes.c_uint64, _u64p]),
    "cuhe_bfv_set_lanes": (ctypes.c_int, [_vp, ctypes.c_int]),
    "cuhe_bfv_batch_encode": (ctypes.c_int, [_vp, ctypes.c_uint64, _vp, ctypes.c_uint64, _vp]),
    "cuhe_bfv_encrypt": (ctypes.c_int, [_vp, ctypes.c_char_p, ctypes.c_uint64, _vp, _vp, _vp, ctypes.c_uint64,
                                        _vp]),
    "cuhe_bfv_encrypt_keyed": (ctypes.c_int, [_vp, ctypes.c_char_p, ctypes.c_uint64, _vp, ctypes.c_char_p,
                                              ctypes.c_char_p, ctypes.c_uint, ctypes.c_uint64, _vp]),
    "cuhe_bfv_packed_search_parts": (ctypes.c_int, [_vp, ctypes.c_char_p, ctypes.POINTER(ctypes.c_char_p),
                                                    ctypes.c_uint64, ctypes.c_uint64, ctypes.c_int, _vp,
                                                    ctypes.c_uint64, _u64p]),
    "cuhe_bfv_upload_index_parts": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_char_p), ctypes.c_uint64,
                                                   ctypes.POINTER(_vp)]),
    "cuhe_bfv_ntt": (ctypes.c_int, [_vp, _vp, ctypes.c_uint64, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                    ctypes.c_int, _vp]),
    "cuhe_bfv_get_lanes": (ctypes.c_int, [_vp]),
    "cuhe_bfv_search_workspace": (ctypes.c_uint64, [_vp, ctypes.c_uint64, ctypes.c_int]),
    "cuhe_bfv_reserve_workspace": (ctypes.c_int, [_vp, ctypes.c_uint64, ctypes.c_int]),
}

BFV_LIB = "libcuhe_bfv_b200.so"


def lib() -> ctypes.CDLL:
    return _native._load(BFV_LIB, BFV_SIGNATURES)


def _check(rc: int) -> None:
    if rc == 0:
        return
    message = lib().cuhe_bfv_last_error()
    text = message.decode() if message else f"status {rc}"
    if rc in (-1, -5):
        raise ValueError(text)
    if rc == -2:
        raise MemoryError(text)
    raise RuntimeError(text)


CUHE_RANGE = -5


class KeystreamRejected(ValueError):
    """A keyed noise draw met eight bytes of 255 for one coefficient
    (probability 2^-64): encrypt again under a new key."""


class _Handle:
    """Capsule equivalent: owns one reference of a native object."""

    _release = ""

    def __init__(self, ptr: int, parents: tuple = ()) -> None:
        self._ptr = ptr
        self._parents = parents

    @property
    def ptr(self) -> int:
        return self._ptr

    def __del__(self) -> None:
        ptr, self._ptr = getattr(self, "_ptr", None), None
        if ptr:
            try:
                getattr(lib(), self._release)(ptr)
            except Exception:  # pragma: no cover - interpreter shutdown
                pass


class Ring(_Handle):
    _release = "cuhe_bfv_ring_release"

    def __init__(self, ptr: int, n: int, coefficient_bytes: int, q_bits: int = 0) -> None:
        super().__init__(ptr)
        self.n = n
        self.coefficient_bytes = coefficient_bytes
        self.q_bits = q_bits


class Key(_Handle):
    _release = "cuhe_bfv_key_release"

    def __init__(self, ptr: int, ring: Ring) -> None:
        super().__init__(ptr, (ring,))
        self.ring = ring


class Server(_Handle):
    _release = "cuhe_bfv_server_release"

    def __init__(self, ptr: int, ring: Ring, keys: tuple) -> None:
        super().__init__(ptr, keys)
        self.ring = ring
        cap, padded, inb, outb, compb = (ctypes.c_uint64() for _ in range(5))
        _check(lib().cuhe_bfv_server_layout(ptr, ctypes.byref(cap), ctypes.byref(padded), ctypes.byref(inb),
                                            ctypes.byref(outb), ctypes.byref(compb)))
        self.capacity = cap.value
        self.padded = padded.value
        self.input_bytes = inb.value
        self.output_bytes = outb.value
        self.compact_bytes = compb.value


def _get(obj: Any, cls: type) -> Any:
    if not isinstance(obj, cls):
        raise TypeError(f"expected a {cls.__name__} handle")
    if not obj.ptr:
        raise ValueError("released handle")
    return obj


def _poly(value: Any, ring: Ring) -> bytes:
    if not isinstance(value, bytes):
        raise TypeError("Polynomial must be fixed-width bytes")
    if len(value) != ring.n * ring.coefficient_bytes:
        raise ValueError("Incorrect polynomial byte length")
    return value


def _pair(value: Any, ring: Ring) -> bytes:
    if not isinstance(value, tuple) or len(value) != 2:
        raise ValueError("Expected two ciphertext components")
    return _poly(value[0], ring) + _poly(value[1], ring)


def _u64(value: Any, what: str) -> int:
    if isinstance(value, bool) or not isinstance(value, int):
        raise TypeError(f"{what} must be an integer")
    if value < 0 or value >= 1 << 64:
        raise OverflowError(f"{what} out of range")
    return value


def _split(raw: bytes, count: int, size: int) -> tuple[bytes, ...]:
    return tuple(raw[i * size:(i + 1) * size] for i in range(count))


def create_ring(n: int, q_hex: str, digit_bits: int, fast: bool = False, residue: bool = False,
                kernel_level: int = 0) -> Ring:
    n, digit_bits, kernel_level = _u64(n, "n"), _u64(digit_bits, "digit_bits"), _u64(kernel_level, "kernel_level")
    if not isinstance(q_hex, str):
        raise TypeError("q_hex must be a string")
    handle = _vp()
    _check(lib().cuhe_bfv_create_ring(n, q_hex.encode(), digit_bits, int(bool(fast)), int(bool(residue)),
                                      kernel_level, 0, ctypes.byref(handle)))
    q_bits = int(q_hex, 16).bit_length()
    return Ring(handle.value, n, (q_bits + 7) // 8, q_bits)


def ring_info(ring: Ring) -> dict[str, Any]:
    ring = _get(ring, Ring)
    primes = (ctypes.c_uint64 * 32)()
    count, switch, residue, level, fast = (ctypes.c_int() for _ in range(5))
    table, cb = ctypes.c_uint64(), ctypes.c_uint64()
    _check(lib().cuhe_bfv_ring_info(ring.ptr, primes, 32, ctypes.byref(count), ctypes.byref(switch),
                                    ctypes.byref(residue), ctypes.byref(table), ctypes.byref(cb), ctypes.byref(level),
                                    ctypes.byref(fast)))
    return {
        "primes": tuple(primes[i] for i in range(count.value)),
        "switch_prime_count": switch.value,
        "transform_table_bytes": table.value,
        "gmp": "none (B200 residue arithmetic)",
        "compiler": "nvcc sm_100a",
        "fast_arithmetic": bool(fast.value),
        "residue_prime_count": residue.value,
        "kernel_level": level.value,
    }


def compile_key(ring: Ring, key: Any) -> Key:
    ring = _get(ring, Ring)
    if not isinstance(key, tuple):
        raise ValueError("Incorrect gadget digit count")
    blob = b"".join(_pair(pair, ring) for pair in key)
    handle = _vp()
    _check(lib().cuhe_bfv_compile_key(ring.ptr, blob, len(key), ctypes.byref(handle)))
    return Key(handle.value, ring)


def key_bytes(key: Key) -> int:
    return int(lib().cuhe_bfv_key_bytes(_get(key, Key).ptr))


def apply_key(key: Key, poly: bytes) -> tuple[bytes, bytes]:
    key = _get(key, Key)
    data = _poly(poly, key.ring)
    out = ctypes.create_string_buffer(2 * len(data))
    _check(lib().cuhe_bfv_apply_key(key.ptr, data, out))
    return _split(out.raw, 2, len(data))


def ring_product(ring: Ring, lhs: bytes, rhs: bytes) -> bytes:
    ring = _get(ring, Ring)
    a, b = _poly(lhs, ring), _poly(rhs, ring)
    out = ctypes.create_string_buffer(len(a))
    _check(lib().cuhe_bfv_ring_product(ring.ptr, a, b, out))
    return out.raw


def multiply(ring: Ring, lhs: Any, rhs: Any, t: int) -> tuple[bytes, bytes, bytes]:
    ring = _get(ring, Ring)
    t = _u64(t, "t")
    a = _pair(lhs, ring)
    b = None if rhs is None else _pair(rhs, ring)
    size = ring.n * ring.coefficient_bytes
    out = ctypes.create_string_buffer(3 * size)
    _check(lib().cuhe_bfv_multiply(ring.ptr, a, b, t, out))
    return _split(out.raw, 3, size)


def rotate_rows(key: Key, ciphertext: Any, exponent: int) -> tuple[bytes, bytes]:
    key = _get(key, Key)
    data = _pair(ciphertext, key.ring)
    exponent = _u64(exponent, "exponent")
    out = ctypes.create_string_buffer(len(data))
    _check(lib().cuhe_bfv_rotate_rows(key.ptr, data, exponent, out))
    return _split(out.raw, 2, len(data) // 2)


def _rotation_list(rotations: Any, ring: Ring) -> tuple[list[int], list[Key]]:
    if not isinstance(rotations, tuple):
        raise ValueError("Rotations must be a tuple")
    exps, keys = [], []
    for entry in rotations:
        if not isinstance(entry, tuple) or len(entry) != 2:
            raise ValueError("Invalid rotation key entry")
        exps.append(_u64(entry[0], "exponent"))
        key = _get(entry[1], Key)
        if key.ring.ptr != ring.ptr:
            raise ValueError("Rotation key belongs to another native ring")
        keys.append(key)
    return exps, keys


def hamming_tile(relin: Key, query: Any, tile: Any, rotations: Any, mask: bytes, t: int) -> tuple[bytes, bytes]:
    relin = _get(relin, Key)
    ring = relin.ring
    t = _u64(t, "t")
    q, tl, m = _pair(query, ring), _pair(tile, ring), _poly(mask, ring)
    exps, keys = _rotation_list(rotations, ring)
    exp_arr = (ctypes.c_uint64 * max(1, len(exps)))(*exps)
    key_arr = (_vp * max(1, len(keys)))(*[k.ptr for k in keys])
    out = ctypes.create_string_buffer(len(q))
    _check(lib().cuhe_bfv_hamming_tile(relin.ptr, q, tl, exp_arr, key_arr, len(exps), m, t, out))
    return _split(out.raw, 2, len(q) // 2)


def create_server(relin: Key, keys: Any, padded: int, t: int, target_hex: str) -> Server:
    relin = _get(relin, Key)
    ring = relin.ring
    padded, t = _u64(padded, "padded"), _u64(t, "t")
    if not isinstance(target_hex, str):
        raise TypeError("target must be a hexadecimal string")
    if not isinstance(keys, tuple):
        raise ValueError("Rotation keys must be a tuple")
    exps, handles = _rotation_list(keys, ring)
    exp_arr = (ctypes.c_uint64 * max(1, len(exps)))(*exps)
    key_arr = (_vp * max(1, len(handles)))(*[k.ptr for k in handles])
    handle = _vp()
    _check(lib().cuhe_bfv_create_server(relin.ptr, exp_arr, key_arr, len(exps), padded, t, target_hex.encode(),
                                        ctypes.byref(handle)))
    return Server(handle.value, ring, (relin, *handles))


def server_bytes(server: Server) -> int:
    return int(lib().cuhe_bfv_server_bytes(_get(server, Server).ptr))


def _packed(value: Any, server: Server) -> bytes:
    if not isinstance(value, tuple) or len(value) != 2:
        raise ValueError("Expected two packed components")
    for part in value:
        if not isinstance(part, bytes) or len(part) != server.input_bytes:
            raise ValueError("Incorrect packed polynomial bytes")
    return value[0] + value[1]


def _poly_pointers(index: Any, server: Server):
    """One pointer per packed polynomial of the index tuple, into the bytes
    objects themselves (validated, not copied); None for an empty index."""
    if not isinstance(index, tuple):
        raise ValueError("index must be a tuple of packed ciphertexts")
    parts = []
    for value in index:
        if not isinstance(value, tuple) or len(value) != 2:
            raise ValueError("Expected two packed components")
        for part in value:
            if not isinstance(part, bytes) or len(part) != server.input_bytes:
                raise ValueError("Incorrect packed polynomial bytes")
            parts.append(part)
    if not parts:
        return None
    return (ctypes.c_char_p * len(parts))(*parts)


def packed_search(server: Server, query: Any, index: Any, count: int, compact: bool) -> list[tuple[bytes, bytes]]:
    server = _get(server, Server)
    count = _u64(count, "count")
    if not isinstance(index, tuple) or count > (1 << 64) - 1 - server.capacity or \
            (count + server.capacity - 1) // server.capacity != len(index):
        raise ValueError("vector_count does not match the packed ciphertext count")
    q = _packed(query, server)
    polys = _poly_pointers(index, server)
    groups = (len(index) + server.padded - 1) // server.padded
    size = server.compact_bytes if compact else server.output_bytes
    out = ctypes.create_string_buffer(max(1, groups * 2 * size))
    responses = ctypes.c_uint64()
    _check(lib().cuhe_bfv_packed_search_parts(server.ptr, q, polys, len(index), count, int(bool(compact)), out,
                                              len(out), ctypes.byref(responses)))
    raw = out.raw
    return [(raw[(2 * i) * size:(2 * i + 1) * size], raw[(2 * i + 1) * size:(2 * i + 2) * size])
            for i in range(responses.value)]


class ResidentIndex(_Handle):
    """An encrypted index validated, unpacked and kept in HBM for a server."""

    _release = "cuhe_bfv_index_release"

    def __init__(self, ptr: int, server: Server, tiles: int) -> None:
        super().__init__(ptr, (server,))
        self.server = server
        self.tiles = tiles


def upload_index(server: Server, index: Any) -> ResidentIndex:
    """Serving form: keep the packed index resident (not in the reference API)."""
    server = _get(server, Server)
    polys = _poly_pointers(index, server)
    handle = _vp()
    _check(lib().cuhe_bfv_upload_index_parts(server.ptr, polys, len(index), ctypes.byref(handle)))
    return ResidentIndex(handle.value, server, len(index))


def search_index(server: Server, index: ResidentIndex, query: Any, count: int,
                 compact: bool) -> list[tuple[bytes, bytes]]:
    """packed_search over a resident index; identical responses."""
    server = _get(server, Server)
    index = _get(index, ResidentIndex)
    count = _u64(count, "count")
    if (count + server.capacity - 1) // server.capacity != index.tiles:
        raise ValueError("vector_count does not match the packed ciphertext count")
    q = _packed(query, server)
    groups = (index.tiles + server.padded - 1) // server.padded
    size = server.compact_bytes if compact else server.output_bytes
    out = ctypes.create_string_buffer(max(1, groups * 2 * size))
    responses = ctypes.c_uint64()
    _check(lib().cuhe_bfv_search_index(server.ptr, index.ptr, q, count, int(bool(compact)), out, len(out),
                                       ctypes.byref(responses)))
    raw = out.raw
    return [(raw[(2 * i) * size:(2 * i + 1) * size], raw[(2 * i + 1) * size:(2 * i + 2) * size])
            for i in range(responses.value)]


def ntt(ring: Ring, planes, primes: int, inverse: bool = False, threads: int = 0, radix_log: int = 0,
        stream: int | None = None) -> None:
    """In-place batched NTT of device planes ([count, N] 64-bit residues, a
    torch CUDA tensor; plane b mod the ring's prime b % primes), enqueued on
    `stream` (a cudaStream_t as int; None: the current torch stream) without
    synchronising, so it can be captured in a CUDA graph (not in the
    reference API)."""
    import torch

    ring = _get(ring, Ring)
    if not (isinstance(planes, torch.Tensor) and planes.is_cuda and planes.dim() == 2
            and planes.shape[1] == ring.n and planes.element_size() == 8 and planes.is_contiguous()):
        raise ValueError("planes must be a contiguous CUDA tensor [count, N] of 64-bit words")
    if stream is None:
        stream = torch.cuda.current_stream(planes.device).cuda_stream
    _check(lib().cuhe_bfv_ntt(ring.ptr, planes.data_ptr(), planes.shape[0], int(primes), int(bool(inverse)),
                              int(threads), int(radix_log), _vp(stream)))


def batch_encode(ring: Ring, t: int, slots):
    """Batch encoding on the device (not in the reference ABI): slots
    [count, N] below t -> [count, N] plaintext coefficients (numpy uint64)."""
    import numpy as np

    ring = _get(ring, Ring)
    slots = np.ascontiguousarray(slots, dtype=np.uint32)
    if slots.ndim == 1:
        slots = slots.reshape(1, -1)
    if slots.ndim != 2 or slots.shape[1] != ring.n:
        raise ValueError("slots must be [count, N]")
    out = np.empty(slots.shape, dtype=np.uint64)
    _check(lib().cuhe_bfv_batch_encode(ring.ptr, int(t), slots.ctypes.data, slots.shape[0], out.ctypes.data))
    return out


def encrypt_packed(ring: Ring, public_key: Any, t: int, slots, u, e) -> list[tuple[bytes, bytes]]:
    """Batched client encryption on the device (not in the reference ABI):
    public_key = (b, a) fixed-width polys; slots [count, N] (< t), u
    [count, N] ternary, e [count, 2, N] signed small noise (numpy arrays).
    Returns packed (c0, c1) per plaintext, the packed_search wire."""
    import numpy as np

    ring = _get(ring, Ring)
    if not isinstance(public_key, tuple) or len(public_key) != 2:
        raise ValueError("public key must be (b, a)")
    pk = b"".join(_poly(p, ring) for p in public_key)
    slots = np.ascontiguousarray(slots, dtype=np.uint32)
    u = np.ascontiguousarray(u, dtype=np.int8)
    e = np.ascontiguousarray(e, dtype=np.int8)
    count = slots.shape[0] if slots.ndim == 2 else -1
    if slots.shape != (count, ring.n) or u.shape != (count, ring.n) or e.shape != (count, 2, ring.n):
        raise ValueError("slots, u and e must be [count, N], [count, N] and [count, 2, N]")
    size = (ring.n * ring.q_bits + 7) // 8
    out = np.empty(max(1, count * 2 * size), dtype=np.uint8)  # filled by the call: no zeroing
    _check(lib().cuhe_bfv_encrypt(ring.ptr, pk, int(t), slots.ctypes.data, u.ctypes.data, e.ctypes.data, count,
                                  out.ctypes.data))
    view = memoryview(out)
    return [(bytes(view[2 * i * size:(2 * i + 1) * size]), bytes(view[(2 * i + 1) * size:(2 * i + 2) * size]))
            for i in range(count)]


def encrypt_packed_keyed(ring: Ring, public_key: Any, t: int, slots, key: bytes, nonce: bytes,
                         eta: int = 21) -> list[tuple[bytes, bytes]]:
    """encrypt_packed with the noise drawn on the device from the ChaCha20
    keystream of (key, nonce) (layout: cuhe_bfv_encrypt_keyed).  Raises
    KeystreamRejected in the 2^-64-per-coefficient case that needs a new
    key."""
    import numpy as np

    ring = _get(ring, Ring)
    if not isinstance(public_key, tuple) or len(public_key) != 2:
        raise ValueError("public key must be (b, a)")
    if len(key) != 32 or len(nonce) != 12:
        raise ValueError("key must be 32 bytes and nonce 12 bytes")
    pk = b"".join(_poly(p, ring) for p in public_key)
    slots = np.ascontiguousarray(slots, dtype=np.uint32)
    count = slots.shape[0] if slots.ndim == 2 else -1
    if slots.shape != (count, ring.n):
        raise ValueError("slots must be [count, N]")
    size = (ring.n * ring.q_bits + 7) // 8
    out = np.empty(max(1, count * 2 * size), dtype=np.uint8)
    rc = lib().cuhe_bfv_encrypt_keyed(ring.ptr, pk, int(t), slots.ctypes.data, bytes(key), bytes(nonce), int(eta),
                                      count, out.ctypes.data)
    if rc == CUHE_RANGE:
        message = lib().cuhe_bfv_last_error()
        raise KeystreamRejected(message.decode() if message else "keystream draw rejected")
    _check(rc)
    view = memoryview(out)
    return [(bytes(view[2 * i * size:(2 * i + 1) * size]), bytes(view[(2 * i + 1) * size:(2 * i + 2) * size]))
            for i in range(count)]


def set_lanes(ring: Ring, lanes: int) -> None:
    """Execution lanes of a ring (1..8): concurrent searches from several host
    threads take free lanes and overlap on the GPU (not in the reference API)."""
    _check(lib().cuhe_bfv_set_lanes(_get(ring, Ring).ptr, int(lanes)))


def get_lanes(ring: Ring) -> int:
    return int(lib().cuhe_bfv_get_lanes(_get(ring, Ring).ptr))


def search_workspace(server: Server, tiles: int, compact: bool = True) -> int:
    """Device bytes one lane holds for a search over `tiles` tiles."""
    return int(lib().cuhe_bfv_search_workspace(_get(server, Server).ptr, int(tiles), int(bool(compact))))


def reserve_workspace(server: Server, tiles: int, compact: bool = True) -> None:
    """Allocate that workspace on every active lane of the server's ring now,
    so later searches of up to `tiles` tiles allocate no device memory."""
    _check(lib().cuhe_bfv_reserve_workspace(_get(server, Server).ptr, _u64(tiles, "tiles"), int(bool(compact))))


def _profile(fn, *args) -> tuple[Any, dict[str, Any]]:
    start = time.perf_counter()
    result = fn(*args)
    wall = time.perf_counter() - start
    timings: dict[str, Any] = {"other": {"seconds": wall, "calls": 1}}
    if fn is packed_search:
        ms = (ctypes.c_double * 6)()
        _check(lib().cuhe_bfv_last_profile(_get(args[0], Server).ptr, ms, 6))
        for name, value in zip(PHASES, ms):
            timings[name] = {"seconds": value / 1e3, "calls": 1}
    return result, timings


def profile_hamming_tile(*args: Any) -> tuple[Any, dict[str, Any]]:
    return _profile(hamming_tile, *args)


def profile_packed_search(*args: Any) -> tuple[Any, dict[str, Any]]:
    return _profile(packed_search, *args)


def profile_call(callback: Any) -> tuple[Any, dict[str, Any]]:
    return _profile(callback)
