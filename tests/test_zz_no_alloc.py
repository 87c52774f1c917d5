"""The allocation-free Hamming decode: same distances as the allocating entry point.

cuhe_paillier_decode_hamming_static serves callers that must not allocate GPU
memory while they run: a serving process whose device memory is owned by a
caching allocator or a fixed reservation, or an embedding runtime that hands
the library only the buffers it already owns.  Its scratch is a fixed
65,536-count device array compiled into the library instead of the context
workspace.  Here it is called through the C ABI, several calls in a row, on
the direct and on the CRT decryption kernel, at up to exactly its stated
maximum, and compared with cuhe_paillier_decode_hamming on the same
ciphertexts; the device's free memory is checked unchanged across the calls
(a growing workspace or any other device allocation would lower it), and
one call is captured in a CUDA graph and replayed.  This
file is collected last on purpose, so that a run stopping at the first
failure has already run every other test; it creates its own contexts, so it
also passes alone in a fresh process.
"""

import ctypes
import random

import numpy as np
import pytest

from conftest import hx, load_golden

pytestmark = pytest.mark.gpu

MAX_CHUNKS = 65536  # CUHE_STATIC_DECODE_MAX_CHUNKS in include/cuhe_paillier.h


def _keys():
    data = load_golden("paillier_512.json")  # textbook keys: ctx.encrypt below is g^m r^n
    pk = {k: hx(v) for k, v in data["pk"].items()}
    sk = {k: hx(v) for k, v in data["sk"].items()}
    return pk, sk


def _context(pk, sk, crt):
    from cuhepy_b200._numbers import factors_from_phi
    from cuhepy_b200.paillier.gpu import PaillierDevice

    ctx = PaillierDevice(pk["n"])
    ctx.set_secret(sk["phi"], sk["inv"])
    if crt:
        ctx.set_factors(*factors_from_phi(pk["n"], sk["phi"]))
    assert ctx.has_factors == crt
    return ctx


@pytest.mark.parametrize("crt", [False, True], ids=["direct", "crt"])
def test_static_scratch_decode_matches_allocating_decode(crt):
    import torch

    from cuhepy_b200 import _native

    lib = _native.paillier_lib()
    pk, sk = _keys()
    n = pk["n"]
    key_len = (n.bit_length() + 1) // 2
    chunk_len = 2 * key_len
    rng = random.Random(4242 + crt)
    reference = _context(pk, sk, crt)  # the allocating entry point
    ctx = _context(pk, sk, crt)        # only ever calls the static entry point
    stream = torch.cuda.Stream()
    ctx.set_stream(stream.cuda_stream)
    # every input and output exists before the first static call
    cases = []
    for vectors, chunk_num in ((3000, 1), (1500, 3)):
        ms = [rng.getrandbits(chunk_len - 1) % n for _ in range(vectors * chunk_num)]
        cts = reference.encrypt(ms, [rng.randrange(1, n) for _ in ms])
        cases.append((vectors, chunk_num, ms, torch.from_numpy(reference.limbs(cts).view(np.int32)).cuda()))
    # exactly the stated maximum: 16,384 vectors x 4 chunks of values below n^2
    words = ctx.words
    gen = torch.Generator(device="cuda")
    gen.manual_seed(77 + crt)
    full = torch.randint(-(1 << 31), 1 << 31, (MAX_CHUNKS, words), dtype=torch.int32, device="cuda", generator=gen)
    full[:, words - 1] = 0
    cases.append((MAX_CHUNKS // 4, 4, None, full))
    wants, gots = [], []
    for vectors, chunk_num, _, c_dev in cases:
        want = torch.full((vectors,), -1, dtype=torch.int64, device="cuda")
        reference.decode_array(c_dev, vectors, chunk_num, chunk_len, want)
        wants.append(want)
        gots.append(torch.full((vectors,), -2, dtype=torch.int64, device="cuda"))
    reference.synchronize()
    torch.cuda.synchronize()

    def static(i):
        vectors, chunk_num, _, c_dev = cases[i]
        gots[i].fill_(-2)
        torch.cuda.synchronize()
        rc = lib.cuhe_paillier_decode_hamming_static(ctx._ctx, c_dev.data_ptr(), vectors, chunk_num, chunk_len,
                                                     gots[i].data_ptr())
        assert rc == 0, lib.cuhe_last_error(ctx._ctx)
        ctx.synchronize()
        assert torch.equal(gots[i], wants[i]), f"case {i}"

    static(0)  # first call on the device: looks up the array's address
    free_before = torch.cuda.mem_get_info()[0]
    for i in (0, 1, 2, 2, 1, 0):  # calls in a row; the shared array keeps the last call's counts
        static(i)
    assert torch.cuda.mem_get_info()[0] == free_before

    # the same call captured in a CUDA graph on the context stream and
    # replayed: a capture in global mode ends with an error at any device
    # allocation or synchronisation inside the call
    vectors, chunk_num, _, c_dev = cases[1]
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=stream, capture_error_mode="global"):
        rc = lib.cuhe_paillier_decode_hamming_static(ctx._ctx, c_dev.data_ptr(), vectors, chunk_num, chunk_len,
                                                     gots[1].data_ptr())
    assert rc == 0, lib.cuhe_last_error(ctx._ctx)
    graph.replay()
    torch.cuda.synchronize()
    free_graph = torch.cuda.mem_get_info()[0]
    for _ in range(3):
        gots[1].fill_(-2)
        torch.cuda.synchronize()
        graph.replay()
        torch.cuda.synchronize()
        assert torch.equal(gots[1], wants[1])
    assert torch.cuda.mem_get_info()[0] == free_graph
    ctx.synchronize()
    del graph
    # independent check of a few distances against the plaintexts
    for (vectors, chunk_num, ms, _), want in zip(cases[:2], wants[:2]):
        want_h = want.cpu().tolist()
        for v in range(0, vectors, max(1, vectors // 7)):
            expect = sum(bin(m & int("01" * (chunk_len // 2), 2)).count("1")
                         for m in ms[v * chunk_num:(v + 1) * chunk_num])
            assert want_h[v] == expect


def test_static_scratch_decode_rejects_oversize_and_host_buffers():
    import torch

    from cuhepy_b200 import _native

    lib = _native.paillier_lib()
    pk, sk = _keys()
    ctx = _context(pk, sk, False)
    c_dev = torch.zeros((2, ctx.words), dtype=torch.int32, device="cuda")
    out = torch.zeros(2, dtype=torch.int64, device="cuda")
    for vectors, chunk_num in ((MAX_CHUNKS + 1, 1), (MAX_CHUNKS // 4 + 1, 4)):
        rc = lib.cuhe_paillier_decode_hamming_static(ctx._ctx, c_dev.data_ptr(), vectors, chunk_num, 1024,
                                                     out.data_ptr())
        assert rc == -1 and b"static scratch" in lib.cuhe_last_error(ctx._ctx)
    host = np.zeros((2, ctx.words), dtype=np.uint32)
    host_out = np.zeros(2, dtype=np.int64)
    rc = lib.cuhe_paillier_decode_hamming_static(ctx._ctx, host.ctypes.data, 2, 1, 1024, host_out.ctypes.data)
    assert rc == -1 and b"device buffers" in lib.cuhe_last_error(ctx._ctx)
    assert ctypes.sizeof(ctypes.c_int64) == 8
