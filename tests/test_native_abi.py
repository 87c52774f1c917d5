"""The C ABI library loads, exports every declared symbol with the declared
number of parameters, its host-only logic behaves, and without a CUDA device
the Paillier context, the client and the BFV ring refuse to start; no kernel
is launched here."""

import ctypes
import random
import re

import numpy as np
import pytest

from conftest import REPO
from cuhepy_b200 import _native
from cuhepy_b200._limbs import from_limbs, to_limbs


def declared(header: str) -> list[str]:
    text = (REPO / "include" / header).read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(cuhe_[a-z0-9_]+)\s*\(", text)))


def parameter_counts(header: str) -> dict[str, int]:
    """Number of parameters of every prototype the header declares."""
    text = (REPO / "include" / header).read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    text = re.sub(r"//[^\n]*", "", text)
    counts = {}
    for m in re.finditer(r"\b(cuhe_[a-z0-9_]+)\s*\(([^;{]*?)\)\s*;", text, flags=re.S):
        args = m.group(2).strip()
        counts[m.group(1)] = 0 if args in ("", "void") else args.count(",") + 1
    return counts


@pytest.mark.parametrize("header", ["cuhe_paillier.h", "cuhe_bfv.h"])
def test_ctypes_signatures_take_the_declared_parameter_counts(header):
    from cuhepy_b200.bfv import _bfv_rns

    table = _native.PAILLIER_SIGNATURES if header == "cuhe_paillier.h" else _bfv_rns.BFV_SIGNATURES
    counts = parameter_counts(header)
    assert sorted(counts) == declared(header)  # every declaration parsed
    for name, count in counts.items():
        assert len(table[name][1]) == count, name


def test_paillier_library_exports_every_declared_symbol():
    lib = _native.paillier_lib()
    names = declared("cuhe_paillier.h")
    assert "cuhe_paillier_encrypt" in names and len(names) > 15
    for name in names:
        assert hasattr(lib, name), name
        assert name in _native.PAILLIER_SIGNATURES, name
    assert lib.cuhe_version().startswith(b"cuhe_b200")


def test_bfv_library_exports_every_declared_symbol():
    from cuhepy_b200.bfv import _bfv_rns

    lib = _bfv_rns.lib()
    names = declared("cuhe_bfv.h")
    assert "cuhe_bfv_packed_search" in names and len(names) > 15
    for name in names:
        assert hasattr(lib, name), name
        assert name in _bfv_rns.BFV_SIGNATURES, name
    assert _bfv_rns.ABI_VERSION == 4


def test_bfv_boundary_validation_without_a_device():
    from cuhepy_b200.bfv import _bfv_rns

    with pytest.raises(TypeError):
        _bfv_rns.create_ring(16, 7, 4)
    with pytest.raises(ValueError):
        _bfv_rns.create_ring(1 << 20, "f", 4, True, True)
    with pytest.raises((TypeError, ValueError, OverflowError)):
        _bfv_rns.create_ring(16, "f", 4, True, True, -1)


def test_context_creation_reports_errors_without_crashing():
    lib = _native.paillier_lib()
    handle = ctypes.c_void_p()
    even = to_limbs([10], 1)[0]
    rc = lib.cuhe_paillier_create(even.ctypes.data_as(_native.c_u32_p), 1, 0, ctypes.byref(handle))
    assert rc == -1 and b"odd" in lib.cuhe_last_error(None)
    big = to_limbs([(1 << 4200) + 1], 132)[0]
    rc = lib.cuhe_paillier_create(big.ctypes.data_as(_native.c_u32_p), 132, 0, ctypes.byref(handle))
    assert rc == -1 and b"wider" in lib.cuhe_last_error(None)


def schedule(e: int, window: int) -> list[int]:
    lib = _native.paillier_lib()
    words = max(1, (e.bit_length() + 31) // 32)
    limbs = to_limbs([e], words)[0]
    ops = (ctypes.c_int32 * 8192)()
    n = lib.cuhe_window_schedule(limbs.ctypes.data_as(_native.c_u32_p), words, window, ops, 8192)
    assert 0 <= n <= 8192
    return list(ops[:n])


def replay(ops: list[int]) -> int:
    """Evaluate a schedule on exponents: table entry t holds exponent 2t+1."""
    if not ops:
        return 0
    value = 2 * ((ops[0] & 0xFFFF) - 1) + 1
    for op in ops[1:]:
        value <<= op >> 16
        if op & 0xFFFF:
            value += 2 * ((op & 0xFFFF) - 1) + 1
    return value


@pytest.mark.parametrize("window", [1, 3, 4, 5, 6])
def test_window_schedule_reconstructs_the_exponent(window):
    rng = random.Random(window)
    cases = [0, 1, 2, 3, 255, 256, 2 ** 64 - 1, 2 ** 64, (1 << 2047) | 1, rng.getrandbits(2048), rng.getrandbits(280)]
    for e in cases:
        ops = schedule(e, window)
        assert replay(ops) == e
        for op in ops:
            assert (op & 0xFFFF) <= 1 << (window - 1)


def test_window_schedule_cost_matches_convention():
    rng = random.Random(7)
    e = rng.getrandbits(2048) | (1 << 2047)
    ops = schedule(e, 5)
    squarings = sum(op >> 16 for op in ops)
    multiplies = sum(1 for op in ops[1:] if op & 0xFFFF)
    # the leading window is loaded from the table without squaring
    assert 2048 - 5 <= squarings <= 2047
    assert multiplies < 2048 / 5


def test_limb_roundtrip():
    rng = random.Random(3)
    values = [0, 1, 2 ** 32 - 1, 2 ** 32] + [rng.getrandbits(4096) for _ in range(20)]
    arr = to_limbs(values, 128)
    assert arr.shape == (len(values), 128) and arr.dtype == np.uint32
    assert from_limbs(arr) == values
    with pytest.raises(ValueError):
        to_limbs([1 << 4096], 128)
    with pytest.raises(ValueError):
        to_limbs([-1], 4)


def test_no_cpu_fallback_without_a_device():
    """Without a CUDA device the Paillier context, the client and the BFV ring
    raise instead of computing on the host (on a machine with a GPU this test
    has nothing to show)."""
    import torch

    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    from cuhepy_b200.bfv import _bfv_rns
    from cuhepy_b200.hamming.paillier_lookup import PaillierLookupClient
    from cuhepy_b200.paillier.gpu import PaillierDevice

    with pytest.raises(RuntimeError, match="no CUDA device"):
        PaillierDevice(10**30 + 1)
    with pytest.raises(RuntimeError, match="no CUDA device"):
        PaillierLookupClient(key_len=512, device="gpu")
    with pytest.raises(RuntimeError, match="no CUDA device"):
        _bfv_rns.create_ring(16, "ffffffffffffffc5", 4, True, True)
    with pytest.raises(NotImplementedError):
        PaillierLookupClient(key_len=512, device="cpu")
