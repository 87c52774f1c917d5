"""ctypes access to the system GMP runtime (libgmp.so.10) for the CPU oracle.

TEST INFRASTRUCTURE ONLY.  This module is imported by the oracle, by the
test-suite and by the CPU-baseline leg of ``bench.py``; the product package
never imports it.

Only GMP's documented public API is used (``mpz_init``, ``mpz_import``,
``mpz_export``, ``mpz_powm``, ``mpz_mul`` ...).  The exported symbol names
carry GMP's ``__g`` prefix (``mpz_powm`` is exported as ``__gmpz_powm``) and an
``mpz_t`` is the documented three-field struct ``{int alloc; int size;
mp_limb_t *d}``.  When the library is missing every helper falls back to
CPython's own big-integer arithmetic, which gives identical results (modular
arithmetic is fully determined), only slower.
"""

from __future__ import annotations

import ctypes
import ctypes.util
import threading

__all__ = ["available", "powmod", "mul", "version"]


class _MPZ(ctypes.Structure):
    _fields_ = [("alloc", ctypes.c_int), ("size", ctypes.c_int), ("d", ctypes.c_void_p)]


def _load():
    for name in ("libgmp.so.10", ctypes.util.find_library("gmp")):
        if not name:
            continue
        try:
            return ctypes.CDLL(name)
        except OSError:
            continue
    return None


_lib = _load()
_local = threading.local()

if _lib is not None:
    _P = ctypes.POINTER(_MPZ)
    _lib.__gmpz_init.argtypes = [_P]
    _lib.__gmpz_clear.argtypes = [_P]
    _lib.__gmpz_import.argtypes = [_P, ctypes.c_size_t, ctypes.c_int, ctypes.c_size_t,
                                   ctypes.c_int, ctypes.c_size_t, ctypes.c_void_p]
    _lib.__gmpz_export.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_size_t), ctypes.c_int,
                                   ctypes.c_size_t, ctypes.c_int, ctypes.c_size_t, _P]
    _lib.__gmpz_export.restype = ctypes.c_void_p
    _lib.__gmpz_powm.argtypes = [_P, _P, _P, _P]
    _lib.__gmpz_mul.argtypes = [_P, _P, _P]
    _lib.__gmpz_sizeinbase.argtypes = [_P, ctypes.c_int]
    _lib.__gmpz_sizeinbase.restype = ctypes.c_size_t


def available() -> bool:
    return _lib is not None


def version() -> str:
    if _lib is None:
        return "unavailable (CPython int fallback)"
    return ctypes.c_char_p.in_dll(_lib, "__gmp_version").value.decode()


def _slots(count: int):
    pool = getattr(_local, "pool", None)
    if pool is None or len(pool) < count:
        pool = [_MPZ() for _ in range(count)]
        for value in pool:
            _lib.__gmpz_init(ctypes.byref(value))
        _local.pool = pool
    return pool[:count]


def _set(slot: _MPZ, value: int) -> None:
    if value < 0:
        raise ValueError("only nonnegative integers cross the GMP boundary")
    data = value.to_bytes(max(1, (value.bit_length() + 7) // 8), "little")
    _lib.__gmpz_import(ctypes.byref(slot), len(data), -1, 1, 0, 0, data)


def _get(slot: _MPZ) -> int:
    if slot.size == 0:
        return 0
    nbytes = (_lib.__gmpz_sizeinbase(ctypes.byref(slot), 2) + 7) // 8
    buf = ctypes.create_string_buffer(nbytes + 8)
    count = ctypes.c_size_t(0)
    _lib.__gmpz_export(buf, ctypes.byref(count), -1, 1, 0, 0, ctypes.byref(slot))
    return int.from_bytes(buf.raw[: count.value], "little")


def powmod(base: int, exponent: int, modulus: int) -> int:
    """base**exponent mod modulus for exponent >= 0 and modulus > 0."""
    if _lib is None or exponent < 0 or modulus <= 0 or modulus.bit_length() < 256:
        return pow(base, exponent, modulus)
    r, b, e, m = _slots(4)
    _set(b, base % modulus)
    _set(e, exponent)
    _set(m, modulus)
    _lib.__gmpz_powm(ctypes.byref(r), ctypes.byref(b), ctypes.byref(e), ctypes.byref(m))
    return _get(r)


def mul(lhs: int, rhs: int) -> int:
    """Exact product of two nonnegative integers (GMP's FFT multiply for huge ones)."""
    if _lib is None or min(lhs.bit_length(), rhs.bit_length()) < 200_000:
        return lhs * rhs
    r, a, b = _slots(3)
    _set(a, lhs)
    _set(b, rhs)
    _lib.__gmpz_mul(ctypes.byref(r), ctypes.byref(a), ctypes.byref(b))
    return _get(r)
