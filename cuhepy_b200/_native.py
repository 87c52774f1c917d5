"""ctypes bindings of the sm_100a shared libraries built from ``csrc/``.

There is no CPU fallback: if a library is missing, or no CUDA device is
present when a context is created, the call raises.  ``load()`` only needs the
file to exist, so symbol checks work on machines without a GPU.
"""

from __future__ import annotations

import ctypes
import os
import threading
from pathlib import Path

LIB_DIR = Path(__file__).resolve().parent / "lib"
PAILLIER_LIB = "libcuhe_b200.so"

_lock = threading.Lock()
_libs: dict[str, ctypes.CDLL] = {}

c_u32_p = ctypes.POINTER(ctypes.c_uint32)
c_u8_p = ctypes.POINTER(ctypes.c_uint8)
c_i64_p = ctypes.POINTER(ctypes.c_int64)

STATUS = {
    0: "CUHE_OK",
    -1: "CUHE_INVALID_ARGUMENT",
    -2: "CUHE_OUT_OF_MEMORY",
    -3: "CUHE_CUDA_ERROR",
    -4: "CUHE_NOT_READY",
    -5: "CUHE_RANGE",
}

# name -> (restype, argtypes); mirrors include/cuhe_paillier.h
PAILLIER_SIGNATURES: dict[str, tuple] = {
    "cuhe_version": (ctypes.c_char_p, []),
    "cuhe_last_error": (ctypes.c_char_p, [ctypes.c_void_p]),
    "cuhe_paillier_create": (ctypes.c_int, [c_u32_p, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]),
    "cuhe_paillier_destroy": (None, [ctypes.c_void_p]),
    "cuhe_paillier_words": (ctypes.c_int, [ctypes.c_void_p]),
    "cuhe_paillier_set_stream": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "cuhe_synchronize": (ctypes.c_int, [ctypes.c_void_p]),
    "cuhe_paillier_set_secret": (ctypes.c_int, [ctypes.c_void_p, c_u32_p, ctypes.c_int, c_u32_p, ctypes.c_int]),
    "cuhe_paillier_set_factors": (ctypes.c_int, [ctypes.c_void_p, c_u32_p, ctypes.c_int, c_u32_p, ctypes.c_int]),
    "cuhe_paillier_has_factors": (ctypes.c_int, [ctypes.c_void_p]),
    "cuhe_paillier_set_fp64": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "cuhe_paillier_from_hex": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_void_p, ctypes.c_int64,
                                              ctypes.c_int, ctypes.c_void_p]),
    "cuhe_paillier_to_hex": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p]),
    "cuhe_paillier_get_fp64": (ctypes.c_int, [ctypes.c_void_p]),
    "cuhe_paillier_encrypt": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                             ctypes.c_int64]),
    "cuhe_paillier_decrypt": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64]),
    "cuhe_paillier_decode_hamming": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int,
                                                    ctypes.c_int, ctypes.c_void_p]),
    "cuhe_paillier_decode_hamming_static": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64,
                                                           ctypes.c_int, ctypes.c_int, ctypes.c_void_p]),
    "cuhe_paillier_modexp": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, c_u32_p, ctypes.c_int,
                                            ctypes.c_void_p, ctypes.c_int64]),
    "cuhe_paillier_modexp_each": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                                 ctypes.c_void_p, ctypes.c_int64]),
    "cuhe_paillier_mulmod": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                            ctypes.c_int64]),
    "cuhe_paillier_mulmod_outer": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64,
                                                  ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p]),
    "cuhe_lookup_set_tables": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                              ctypes.c_int]),
    "cuhe_lookup_build_tables": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                                ctypes.c_int]),
    "cuhe_lookup_get_g_table": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "cuhe_lookup_set_wide_table": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "cuhe_lookup_wide_table_ready": (ctypes.c_int, [ctypes.c_void_p]),
    "cuhe_lookup_encrypt_bits": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int,
                                                ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]),
    "cuhe_lookup_encrypt_ints": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p,
                                                ctypes.c_void_p]),
    "cuhe_imad_peak": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(ctypes.c_double)]),
    "cuhe_fp64_peak": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(ctypes.c_double)]),
    "cuhe_window_schedule": (ctypes.c_int, [c_u32_p, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int32),
                                            ctypes.c_int]),
    "cuhe_paillier_set_tuning": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]),
    "cuhe_mix_create": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]),
    "cuhe_mix_destroy": (None, [ctypes.c_void_p]),
    "cuhe_mix_last_error": (ctypes.c_char_p, [ctypes.c_void_p]),
    "cuhe_mix_add_modexp": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                           ctypes.c_int64, c_u32_p, ctypes.c_int]),
    "cuhe_mix_set_tuning": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    "cuhe_mix_plan": (ctypes.c_int, [ctypes.c_void_p]),
    "cuhe_mix_launch": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "cuhe_mix_check": (ctypes.c_int, [ctypes.c_void_p]),
    "cuhe_mix_widths": (ctypes.c_int, [ctypes.c_void_p]),
    "cuhe_mix_info": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                     ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                     ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int64),
                                     ctypes.POINTER(ctypes.c_int)]),
    "cuhe_paillier_get_tuning": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int),
                                                ctypes.POINTER(ctypes.c_int)]),
}


class NativeLibraryMissing(ImportError):
    """The sm_100a shared library has not been built (run ``cuhepy_b200.build``)."""


def library_path(name: str) -> Path:
    override = os.environ.get("CUHE_B200_LIB_DIR")
    return (Path(override) if override else LIB_DIR) / name


def _load(name: str, signatures: dict[str, tuple]) -> ctypes.CDLL:
    with _lock:
        lib = _libs.get(name)
        if lib is not None:
            return lib
        path = library_path(name)
        if not path.exists():
            raise NativeLibraryMissing(
                f"{path} is missing; build it with `python -m cuhepy_b200.build` (nvcc, sm_100a)"
            )
        lib = ctypes.CDLL(str(path))
        for symbol, (restype, argtypes) in signatures.items():
            fn = getattr(lib, symbol)
            fn.restype = restype
            fn.argtypes = argtypes
        _libs[name] = lib
        return lib


def paillier_lib() -> ctypes.CDLL:
    return _load(PAILLIER_LIB, PAILLIER_SIGNATURES)


def raise_for_status(rc: int, lib: ctypes.CDLL, ctx) -> None:
    if rc == 0:
        return
    message = lib.cuhe_last_error(ctx)
    text = message.decode() if message else STATUS.get(rc, str(rc))
    if rc in (-1, -5):
        raise ValueError(text)
    if rc == -2:
        raise MemoryError(text)
    raise RuntimeError(text)
