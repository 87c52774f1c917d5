"""The allocation-free Hamming decode: same distances as the allocating entry point.

cuhe_paillier_decode_hamming_static serves callers that cannot allocate GPU
memory while they run (code inside a CUDA graph capture, or a serving
process whose device memory is owned by a caching allocator or a fixed
reservation): its scratch is a fixed 65,536-count device array compiled into
the library instead of the context workspace.  This file is collected last on
purpose, so that a run stopping at the first failure has already run every
other test; it creates its own context, so it also passes alone in a fresh
process.
"""

import ctypes
import random

import numpy as np
import pytest

from conftest import hx, load_golden

pytestmark = pytest.mark.gpu


def _setup():
    import torch

    from cuhepy_b200 import _native
    from cuhepy_b200.paillier.gpu import PaillierDevice

    data = load_golden("paillier_512.json")  # textbook keys: ctx.encrypt below is g^m r^n
    pk = {k: hx(v) for k, v in data["pk"].items()}
    sk = {k: hx(v) for k, v in data["sk"].items()}
    ctx = PaillierDevice(pk["n"])
    ctx.set_secret(sk["phi"], sk["inv"])
    return torch, _native, ctx, pk, sk


def test_static_scratch_decode_matches_allocating_decode():
    torch, _native, ctx, pk, sk = _setup()
    lib = _native.paillier_lib()
    stream = torch.cuda.Stream()
    ctx.set_stream(stream.cuda_stream)
    rng = random.Random(4242)
    n, n2 = pk["n"], pk["n_squared"]
    key_len = (n.bit_length() + 1) // 2
    chunk_len = 2 * key_len
    # server products of encryptions of random Hamming-coded plaintexts
    for call, (vectors, chunk_num) in enumerate(((3000, 1), (1500, 3))):
        ms = [rng.getrandbits(chunk_len - 1) % n for _ in range(vectors * chunk_num)]
        rs = [rng.randrange(1, n) for _ in ms]
        cts = ctx.encrypt(ms, rs)
        c_dev = torch.from_numpy(ctx.limbs(cts).view(np.int32)).cuda()
        want = torch.full((vectors,), -1, dtype=torch.int64, device="cuda")
        got = torch.full((vectors,), -2, dtype=torch.int64, device="cuda")
        with torch.cuda.stream(stream):
            ctx.decode_array(c_dev, vectors, chunk_num, chunk_len, want)
            rc = lib.cuhe_paillier_decode_hamming_static(ctx._ctx, c_dev.data_ptr(), vectors, chunk_num,
                                                         chunk_len, got.data_ptr())
        assert rc == 0, lib.cuhe_last_error(ctx._ctx)
        ctx.synchronize()
        assert torch.equal(got, want), f"call {call}"
        # independent check of a few distances against the plaintexts
        want_h = want.cpu().tolist()
        for v in range(0, vectors, max(1, vectors // 7)):
            expect = sum(bin(m & int("01" * (chunk_len // 2), 2)).count("1")
                         for m in ms[v * chunk_num:(v + 1) * chunk_num])
            assert want_h[v] == expect


def test_static_scratch_decode_rejects_oversize_and_host_buffers():
    torch, _native, ctx, pk, sk = _setup()
    lib = _native.paillier_lib()
    n_chunks = 65536 + 1
    c_dev = torch.zeros((2, ctx.words), dtype=torch.int32, device="cuda")
    out = torch.zeros(2, dtype=torch.int64, device="cuda")
    rc = lib.cuhe_paillier_decode_hamming_static(ctx._ctx, c_dev.data_ptr(), n_chunks, 1, 1024, out.data_ptr())
    assert rc == -1 and b"static scratch" in lib.cuhe_last_error(ctx._ctx)
    host = np.zeros((2, ctx.words), dtype=np.uint32)
    host_out = np.zeros(2, dtype=np.int64)
    rc = lib.cuhe_paillier_decode_hamming_static(ctx._ctx, host.ctypes.data, 2, 1, 1024, host_out.ctypes.data)
    assert rc == -1 and b"device buffers" in lib.cuhe_last_error(ctx._ctx)
    assert ctypes.sizeof(ctypes.c_int64) == 8
