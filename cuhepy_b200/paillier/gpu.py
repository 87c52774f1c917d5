"""Per-key device contexts for the Paillier kernels (wrapper over the C ABI).

A :class:`PaillierDevice` owns one ``cuhe_paillier`` context: the modulus n,
its Montgomery constants mod n^2 and mod n, an optional secret exponent /
multiplier, and the device-resident Paillier-Lookup tables.  Every batched
method accepts either Python integers (converted to the limb layout) or
numpy / torch arrays in that layout; torch CUDA tensors are passed through as
device pointers without a copy.
"""

from __future__ import annotations

import ctypes
import threading
from collections import OrderedDict
from collections.abc import Sequence
from typing import Any

import numpy as np

from cuhepy_b200 import _native
from cuhepy_b200._limbs import from_limbs, to_limbs, words_for
from cuhepy_b200._numbers import factors_from_phi

NOISE_MULTIPLES = 14


def _ptr(array: Any) -> int:
    """Address of a numpy array or a torch tensor (host or device)."""
    if isinstance(array, np.ndarray):
        if not array.flags["C_CONTIGUOUS"]:
            raise ValueError("arrays crossing the C ABI must be C-contiguous")
        return array.ctypes.data
    data_ptr = getattr(array, "data_ptr", None)
    if data_ptr is not None:
        if not array.is_contiguous():
            raise ValueError("tensors crossing the C ABI must be contiguous")
        return int(data_ptr())
    raise TypeError(f"unsupported buffer type {type(array)!r}")


class PaillierDevice:
    """Device context for modulus n (public) with an optional secret."""

    def __init__(self, n: int, device: int = 0) -> None:
        self._lib = _native.paillier_lib()
        n = int(n)
        if n <= 1 or n % 2 == 0:
            raise ValueError("n must be an odd integer > 1")
        nw = words_for(n)
        limbs = to_limbs([n], nw)[0]
        handle = ctypes.c_void_p()
        rc = self._lib.cuhe_paillier_create(
            limbs.ctypes.data_as(_native.c_u32_p), nw, int(device), ctypes.byref(handle)
        )
        if rc != 0:
            message = self._lib.cuhe_last_error(None)
            raise RuntimeError(f"cannot create a B200 Paillier context: {message.decode() if message else rc}")
        self._ctx = handle
        self.n = n
        self.n_squared = n * n
        self.words = int(self._lib.cuhe_paillier_words(self._ctx))
        self.device = int(device)
        self.secret: tuple[int, int] | None = None
        self.tables: tuple[int, int] | None = None  # (message_chunks, noise_entries)
        self._lock = threading.RLock()

    # -- lifetime ---------------------------------------------------------
    def close(self) -> None:
        ctx, self._ctx = getattr(self, "_ctx", None), None
        if ctx:
            self._lib.cuhe_paillier_destroy(ctx)

    def __del__(self) -> None:  # pragma: no cover - interpreter shutdown order
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc: int) -> None:
        _native.raise_for_status(rc, self._lib, self._ctx)

    # -- configuration ----------------------------------------------------
    def set_secret(self, exponent: int, multiplier: int) -> None:
        e = to_limbs([int(exponent)], words_for(exponent))[0]
        m = to_limbs([int(multiplier) % self.n], words_for(int(multiplier) % self.n))[0]
        self._check(self._lib.cuhe_paillier_set_secret(
            self._ctx, e.ctypes.data_as(_native.c_u32_p), e.size, m.ctypes.data_as(_native.c_u32_p), m.size))
        self.secret = (int(exponent), int(multiplier))

    def set_factors(self, p: int | None, q: int | None) -> None:
        """Install n = p q so that decrypt / decode run by the CRT (same
        results, half-width exponentiations); None, None removes them."""
        if p is None and q is None:
            self._check(self._lib.cuhe_paillier_set_factors(self._ctx, None, 0, None, 0))
            return
        pl = to_limbs([int(p)], words_for(int(p)))[0]
        ql = to_limbs([int(q)], words_for(int(q)))[0]
        self._check(self._lib.cuhe_paillier_set_factors(
            self._ctx, pl.ctypes.data_as(_native.c_u32_p), pl.size, ql.ctypes.data_as(_native.c_u32_p), ql.size))

    @property
    def has_factors(self) -> bool:
        return bool(self._lib.cuhe_paillier_has_factors(self._ctx))

    def set_fp64(self, enable: int) -> None:
        """CRT exponentiations as 52-bit-limb products on the FP64 pipe for n^2
        of 4096 bits or more (1, the default; 2: also for 2048 bits) or as
        32-bit word products on the integer pipe (0); identical results."""
        self._check(self._lib.cuhe_paillier_set_fp64(self._ctx, int(enable)))

    @property
    def fp64(self) -> int:
        return int(self._lib.cuhe_paillier_get_fp64(self._ctx))

    def set_stream(self, stream: int | None) -> None:
        self._check(self._lib.cuhe_paillier_set_stream(self._ctx, ctypes.c_void_p(stream or 0)))

    def synchronize(self) -> None:
        self._check(self._lib.cuhe_synchronize(self._ctx))

    def set_tuning(self, threads_per_instance: int = 0, window: int = 0) -> None:
        self._check(self._lib.cuhe_paillier_set_tuning(self._ctx, int(threads_per_instance), int(window)))

    VARIANTS = {64: [(8, 3), (8, 4), (16, 4)],
                128: [(8, 4), (16, 3), (16, 4), (16, 5), (32, 3), (32, 4)],
                256: [(16, 4), (32, 3), (32, 4), (32, 5)]}

    def autotune(self, exponent_bits: int = 0, count: int = 0, reps: int = 2) -> dict:
        """Time every compiled (threads per instance, window) variant on a
        fixed-exponent batch of this context's width and keep the fastest.

        The measurement uses a device-resident batch (one resident wave of
        groups per SM at least) and CUDA events on a private stream; returns
        the timings so callers can record the choice."""
        import torch

        rng = np.random.default_rng(5)
        count = count or 148 * (128 // 8) * 4
        bits = exponent_bits or max(2, self.n.bit_length())
        exponent = int(rng.integers(1, 1 << 62)) | (1 << 62)
        while exponent.bit_length() < bits:
            exponent = (exponent << 62) | int(rng.integers(0, 1 << 62))
        exponent >>= max(0, exponent.bit_length() - bits)
        raw = rng.integers(0, 1 << 32, size=(count, self.words), dtype=np.uint64).astype(np.uint32)
        raw[:, -1] = 0  # below n^2
        base = torch.from_numpy(raw.view(np.int32)).cuda(self.device)
        out = torch.empty_like(base)
        stream = torch.cuda.Stream(self.device)
        self.set_stream(stream.cuda_stream)
        timings = {}
        try:
            for tpi, window in self.VARIANTS[self.words]:
                self.set_tuning(tpi, window)
                with torch.cuda.stream(stream):
                    self.modexp_array(base, exponent, out, count)
                    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    start.record(stream)
                    for _ in range(reps):
                        self.modexp_array(base, exponent, out, count)
                    end.record(stream)
                end.synchronize()
                timings[(tpi, window)] = start.elapsed_time(end) / reps
        finally:
            self.set_stream(None)
        best = min(timings, key=timings.get)
        self.set_tuning(*best)
        return {"best": best, "ms": {f"{t}x{w}": v for (t, w), v in timings.items()}}

    def tuning(self) -> tuple[int, int]:
        tpi, w = ctypes.c_int(), ctypes.c_int()
        self._check(self._lib.cuhe_paillier_get_tuning(self._ctx, ctypes.byref(tpi), ctypes.byref(w)))
        return tpi.value, w.value

    # -- conversions --------------------------------------------------------
    def limbs(self, values: Sequence[int]) -> np.ndarray:
        return to_limbs(values, self.words)

    def empty(self, count: int) -> np.ndarray:
        return np.zeros((count, self.words), dtype=np.uint32)

    # -- array-level operations (limb layout, host or device buffers) -------
    def encrypt_array(self, m, r, out, count: int) -> None:
        self._check(self._lib.cuhe_paillier_encrypt(self._ctx, _ptr(m), _ptr(r), _ptr(out), int(count)))

    def decrypt_array(self, c, out, count: int) -> None:
        self._check(self._lib.cuhe_paillier_decrypt(self._ctx, _ptr(c), _ptr(out), int(count)))

    def mulmod_array(self, a, b, out, count: int) -> None:
        self._check(self._lib.cuhe_paillier_mulmod(self._ctx, _ptr(a), _ptr(b), _ptr(out), int(count)))

    def mulmod_outer_array(self, q, nq: int, x, nx: int, out) -> None:
        self._check(self._lib.cuhe_paillier_mulmod_outer(self._ctx, _ptr(q), int(nq), _ptr(x), int(nx), _ptr(out)))

    def decode_array(self, c, vectors: int, chunk_num: int, chunk_len: int, out) -> None:
        self._check(self._lib.cuhe_paillier_decode_hamming(
            self._ctx, _ptr(c), int(vectors), int(chunk_num), int(chunk_len), _ptr(out)))

    def modexp_array(self, base, exponent: int, out, count: int) -> None:
        e = to_limbs([int(exponent)], words_for(exponent))[0]
        self._check(self._lib.cuhe_paillier_modexp(
            self._ctx, _ptr(base), e.ctypes.data_as(_native.c_u32_p), e.size, _ptr(out), int(count)))

    def modexp_each_array(self, base, exponents, exponent_words: int, out, count: int) -> None:
        self._check(self._lib.cuhe_paillier_modexp_each(
            self._ctx, _ptr(base), _ptr(exponents), int(exponent_words), _ptr(out), int(count)))

    def set_wide_table(self, mode: int) -> None:
        """16-bit-digit encryption table (half the table products, same
        ciphertexts): 1 (default) built for calls of at least 65,536
        ciphertexts when it fits, 2 always, 0 never."""
        self._check(self._lib.cuhe_lookup_set_wide_table(self._ctx, int(mode)))

    def wide_table_ready(self) -> bool:
        return bool(self._lib.cuhe_lookup_wide_table_ready(self._ctx))

    def lookup_encrypt_bits_array(self, bits, vectors: int, embed_len: int, chunk_len: int, chunk_num: int,
                                  noise_index, out) -> None:
        self._check(self._lib.cuhe_lookup_encrypt_bits(
            self._ctx, _ptr(bits), int(vectors), int(embed_len), int(chunk_len), int(chunk_num),
            _ptr(noise_index), _ptr(out)))

    def lookup_encrypt_ints_array(self, m, count: int, noise_index, out) -> None:
        self._check(self._lib.cuhe_lookup_encrypt_ints(self._ctx, _ptr(m), int(count), _ptr(noise_index), _ptr(out)))

    # -- hexadecimal wire format (parsed and formatted on the device) --------
    def from_hex(self, strings: Sequence[str], reduce: bool = True) -> np.ndarray:
        """Limb array [count, K] of hexadecimal strings (optional 0x prefix),
        reduced mod n^2 unless reduce is False; digits beyond K words are
        dropped.  ValueError("Invalid hex digit") on any other character."""
        count = len(strings)
        if count == 0:
            return np.zeros((0, self.words), dtype=np.uint32)
        try:
            text = "".join(strings).encode("ascii")
        except (UnicodeEncodeError, TypeError) as exc:
            raise ValueError("Invalid hex digit") from exc
        offsets = np.zeros(count + 1, dtype=np.int64)
        np.cumsum(np.fromiter((len(x) for x in strings), dtype=np.int64, count=count), out=offsets[1:])
        out = self.empty(count)
        self._check(self._lib.cuhe_paillier_from_hex(self._ctx, text, offsets.ctypes.data, count, int(reduce),
                                                     out.ctypes.data))
        return out

    def to_hex(self, limbs) -> list[str]:
        """Lowercase hexadecimal strings (no prefix, no leading zeros, "0" for
        zero) of a limb array [count, K], formatted on the device."""
        count = int(limbs.shape[0])
        if count == 0:
            return []
        width = 8 * self.words
        buf = ctypes.create_string_buffer(count * width)
        self._check(self._lib.cuhe_paillier_to_hex(self._ctx, _ptr(limbs), count, buf))
        text = buf.raw.decode("ascii")
        return [text[i * width:(i + 1) * width].lstrip("0") or "0" for i in range(count)]

    # -- Python-integer conveniences ----------------------------------------
    def encrypt(self, plaintexts: Sequence[int], rs: Sequence[int]) -> list[int]:
        if len(plaintexts) != len(rs):
            raise ValueError("one r per plaintext is required")
        for m in plaintexts:
            if not 0 <= int(m) < self.n:
                raise ValueError("plaintext must be in range [0, n)")
        if not plaintexts:
            return []
        m, r = self.limbs(plaintexts), self.limbs(rs)
        out = self.empty(len(plaintexts))
        self.encrypt_array(m, r, out, len(plaintexts))
        return from_limbs(out)

    def decrypt(self, ciphertexts: Sequence[int]) -> list[int]:
        for c in ciphertexts:
            if not 0 <= int(c) < self.n_squared:
                raise ValueError("ciphertext must be in range [0, n^2)")
        if not ciphertexts:
            return []
        c = self.limbs(ciphertexts)
        out = self.empty(len(ciphertexts))
        self.decrypt_array(c, out, len(ciphertexts))
        return from_limbs(out)

    def mulmod(self, a: Sequence[int], b: Sequence[int]) -> list[int]:
        if len(a) != len(b):
            raise ValueError("ct1 and ct2 must have the same length")
        if not a:
            return []
        # the reference reduces arbitrary nonnegative products mod n^2
        aa = self.limbs([int(v) % self.n_squared for v in a])
        bb = self.limbs([int(v) % self.n_squared for v in b])
        out = self.empty(len(a))
        self.mulmod_array(aa, bb, out, len(a))
        return from_limbs(out)

    def mulmod_outer(self, queries: Sequence[int], index: Sequence[int]) -> list[list[int]]:
        if not queries or not index:
            return [[] for _ in queries]
        q, x = self.limbs(queries), self.limbs(index)
        out = np.zeros((len(queries) * len(index), self.words), dtype=np.uint32)
        self.mulmod_outer_array(q, len(queries), x, len(index), out)
        flat = from_limbs(out)
        return [flat[i * len(index):(i + 1) * len(index)] for i in range(len(queries))]

    def modexp(self, bases: Sequence[int], exponent: int) -> list[int]:
        if not bases:
            return []
        b = self.limbs(bases)
        out = self.empty(len(bases))
        self.modexp_array(b, exponent, out, len(bases))
        return from_limbs(out)

    def modexp_each(self, bases: Sequence[int], exponents: Sequence[int]) -> list[int]:
        if len(bases) != len(exponents):
            raise ValueError("one exponent per base is required")
        if not bases:
            return []
        ew = max(words_for(e) for e in exponents)
        ew = min(self.words, ew)
        if any(int(e) < 0 or words_for(e) > self.words for e in exponents):
            raise ValueError("exponents must be nonnegative and fit the context width")
        b = self.limbs(bases)
        e = to_limbs([int(v) for v in exponents], ew)
        out = self.empty(len(bases))
        self.modexp_each_array(b, e, ew, out, len(bases))
        return from_limbs(out)

    def decode_hamming(self, ciphers: Sequence[Sequence[int]], chunk_num: int, chunk_len: int) -> list[int]:
        if not ciphers:
            return []
        for row in ciphers:
            if len(row) != chunk_num:
                raise ValueError("each inner list must have length == chunk_num")
        flat = [int(c) for row in ciphers for c in row]
        for c in flat:
            if not 0 <= c < self.n_squared:
                raise ValueError("ciphertext must be in range [0, n^2)")
        c = self.limbs(flat)
        out = np.zeros(len(ciphers), dtype=np.int64)
        self.decode_array(c, len(ciphers), chunk_num, chunk_len, out)
        return [int(v) for v in out]

    # -- Paillier-Lookup tables ---------------------------------------------
    def set_tables(self, g_table: Sequence[Sequence[int]], noise: Sequence[int]) -> None:
        chunks = len(g_table)
        flat = [int(v) for row in g_table for v in row]
        if any(len(row) != 256 for row in g_table):
            raise ValueError("every g_table row must hold 256 entries")
        g = self.limbs(flat)
        z = self.limbs([int(v) for v in noise])
        self._check(self._lib.cuhe_lookup_set_tables(self._ctx, _ptr(g), chunks, _ptr(z), len(noise)))
        self.tables = (chunks, len(noise))

    def build_tables(self, g: int, message_chunks: int, noise: Sequence[int] | None) -> None:
        gl = self.limbs([int(g) % self.n_squared])
        if noise is None:
            rc = self._lib.cuhe_lookup_build_tables(self._ctx, _ptr(gl), int(message_chunks), None, 0)
            entries = self.tables[1] if self.tables else 0
        else:
            z = self.limbs([int(v) for v in noise])
            rc = self._lib.cuhe_lookup_build_tables(self._ctx, _ptr(gl), int(message_chunks), _ptr(z), len(noise))
            entries = len(noise)
        self._check(rc)
        self.tables = (int(message_chunks), entries)

    def g_table(self) -> list[list[int]]:
        if not self.tables:
            raise RuntimeError("tables not installed")
        chunks = self.tables[0]
        out = np.zeros((chunks * 256, self.words), dtype=np.uint32)
        self._check(self._lib.cuhe_lookup_get_g_table(self._ctx, _ptr(out)))
        flat = from_limbs(out)
        return [flat[i * 256:(i + 1) * 256] for i in range(chunks)]

    def lookup_encrypt_bits(self, bits: np.ndarray, chunk_len: int, chunk_num: int,
                            noise_index: np.ndarray) -> list[list[int]]:
        bits = np.ascontiguousarray(bits, dtype=np.uint8)
        vectors, embed_len = bits.shape
        total = vectors * chunk_num
        idx = np.ascontiguousarray(noise_index, dtype=np.uint8).reshape(total, NOISE_MULTIPLES)
        out = self.empty(total)
        self.lookup_encrypt_bits_array(bits, vectors, embed_len, chunk_len, chunk_num, idx, out)
        flat = from_limbs(out)
        return [flat[i * chunk_num:(i + 1) * chunk_num] for i in range(vectors)]

    def lookup_encrypt_ints(self, plaintexts: Sequence[int], noise_index: np.ndarray) -> list[int]:
        for m in plaintexts:
            if not 0 <= int(m) < self.n:
                raise ValueError("plaintext must be in range [0, n)")
        if not plaintexts:
            return []
        m = self.limbs(plaintexts)
        idx = np.ascontiguousarray(noise_index, dtype=np.uint8).reshape(len(plaintexts), NOISE_MULTIPLES)
        out = self.empty(len(plaintexts))
        self.lookup_encrypt_ints_array(m, len(plaintexts), idx, out)
        return from_limbs(out)


_cache: "OrderedDict[tuple, PaillierDevice]" = OrderedDict()
_cache_lock = threading.Lock()
_CACHE_MAX = 8


def device_for(n: int, secret: tuple[int, int] | None = None, device: int = 0,
               phi: int | None = None) -> PaillierDevice:
    """Cached context for modulus n (and secret, when given).  With phi, the
    factors of n are recovered and installed, so decrypt / decode use the CRT
    kernel (identical results)."""
    key = (int(n), secret, int(device), None if phi is None else int(phi))
    with _cache_lock:
        ctx = _cache.get(key)
        if ctx is not None:
            _cache.move_to_end(key)
            return ctx
    ctx = PaillierDevice(n, device)
    if secret is not None:
        ctx.set_secret(*secret)
    if phi is not None:
        factors = factors_from_phi(int(n), int(phi))
        if factors is not None:
            try:
                ctx.set_factors(*factors)
            except ValueError:
                pass  # unbalanced factors: the direct kernel serves this key
    with _cache_lock:
        _cache[key] = ctx
        while len(_cache) > _CACHE_MAX:
            _, old = _cache.popitem(last=False)
            old.close()
    return ctx
