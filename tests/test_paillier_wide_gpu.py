"""The 16-bit-digit encryption table (cuhe_lookup_set_wide_table): one table
entry per pair of 8-bit digits gives the same ciphertexts as the 8-bit
table, as 32-bit words on the integer pipe and as 52-bit limbs on the FP64
pipe, for the reference's golden vectors, random embeddings over several
chunks, random plaintext words, an odd number of digit rows and n² of 8192
bits; and the table is built only when asked or for a large call; a noise
index past a short noise table is a range error on both pipes.  Integer
work: every comparison is exact."""

import random

import numpy as np
import pytest

from conftest import hx, load_golden
from oracle import paillier as oracle

pytestmark = pytest.mark.gpu


def _context(data):
    from cuhepy_b200.paillier.gpu import PaillierDevice

    pk = {k: hx(v) for k, v in data["pk"].items()}
    ctx = PaillierDevice(pk["n"])
    noise = oracle.noise_table(pk["g"], pk["n"], [hx(r) for r in data["noise_exponents"]])
    ctx.build_tables(pk["g"], data["message_chunks"], noise)
    return pk, ctx, noise


@pytest.mark.parametrize("name", ["lookup_512.json", "lookup_1024.json"])
def test_wide_table_gives_the_same_ciphertexts(name):
    data = load_golden(name)
    pk, ctx, noise = _context(data)
    try:
        key_len = data["key_len"]
        rng = random.Random(17)
        ms = [hx(c["m"]) for c in data["encrypt"]]
        idx = np.array([c["indices"] for c in data["encrypt"]], dtype=np.uint8)
        embed_len = key_len + 300  # two chunks, the last partial
        chunk_len, chunk_num = oracle.chunk_layout(embed_len, key_len)
        vecs = np.array([[rng.getrandbits(1) for _ in range(embed_len)] for _ in range(24)], dtype=np.uint8)
        vidx = np.array([[rng.randrange(256) for _ in range(14)] for _ in range(24 * chunk_num)], dtype=np.uint8)
        plain = [rng.randrange(pk["n"]) for _ in range(40)] + [0, 1, pk["n"] - 1]
        pidx = np.array([[rng.randrange(256) for _ in range(14)] for _ in range(len(plain))], dtype=np.uint8)

        ctx.set_wide_table(0)
        narrow_bits = ctx.lookup_encrypt_bits(vecs, chunk_len, chunk_num, vidx)
        narrow_ints = ctx.lookup_encrypt_ints(plain, pidx)
        assert not ctx.wide_table_ready()

        ctx.set_wide_table(2)
        assert ctx.lookup_encrypt_ints(ms, idx) == [hx(c["c"]) for c in data["encrypt"]]
        assert ctx.wide_table_ready()
        if data["hamming"]:
            vectors = data["hamming"]["vectors"]
            bits = np.array([[int(b) for b in v["bits"]] for v in vectors], dtype=np.uint8)
            hidx = np.array([v["indices"] for v in vectors], dtype=np.uint8)
            assert ctx.lookup_encrypt_bits(bits, 2 * key_len, 1, hidx) == [[hx(v["c"][0])] for v in vectors]
        assert ctx.lookup_encrypt_bits(vecs, chunk_len, chunk_num, vidx) == narrow_bits
        assert ctx.lookup_encrypt_ints(plain, pidx) == narrow_ints
        # the other pipe's table (n^2 of 4096 bits: FP64 by default, 52-bit
        # limbs; 2048 bits: the FP64 pipe only when asked for)
        other = 0 if ctx.fp64 == 1 and ctx.words >= 128 else 2
        ctx.set_wide_table(0)
        ctx.set_fp64(other)
        ctx.set_wide_table(2)
        assert ctx.lookup_encrypt_ints(ms, idx) == [hx(c["c"]) for c in data["encrypt"]]
        assert ctx.lookup_encrypt_bits(vecs, chunk_len, chunk_num, vidx) == narrow_bits
        assert ctx.lookup_encrypt_ints(plain, pidx) == narrow_ints
        ctx.set_wide_table(0)
        ctx.set_fp64(1)
        ctx.set_wide_table(2)
        # and the 8-bit path is still the oracle's
        table = ctx.g_table()
        for k in (0, 7, len(plain) - 1):
            assert narrow_ints[k] == oracle.lookup_encrypt(plain[k], pk, table, noise, list(pidx[k]), len(table))
        # installing new tables drops the wide table
        ctx.build_tables(pk["g"], data["message_chunks"], noise)
        assert not ctx.wide_table_ready()
    finally:
        ctx.close()


def test_wide_table_with_an_odd_digit_count_and_the_build_policy():
    import torch

    data = load_golden("lookup_512.json")
    pk, ctx, noise = _context(data)
    try:
        chunks = 127  # the last 16-bit row pairs digit 126 with nothing
        ctx.build_tables(pk["g"], chunks, noise)
        rng = random.Random(23)
        plain = [rng.randrange(1 << (8 * chunks)) for _ in range(30)] + [(1 << (8 * chunks)) - 1, 255 << 1008]
        pidx = np.array([[rng.randrange(256) for _ in range(14)] for _ in range(len(plain))], dtype=np.uint8)
        ctx.set_wide_table(0)
        narrow = ctx.lookup_encrypt_ints(plain, pidx)
        table = ctx.g_table()
        assert narrow[-1] == oracle.lookup_encrypt(plain[-1], pk, table, noise, list(pidx[-1]), len(table))
        ctx.set_wide_table(2)
        assert ctx.lookup_encrypt_ints(plain, pidx) == narrow
        assert ctx.wide_table_ready()
        ctx.set_wide_table(0)
        ctx.set_fp64(2)  # the table as 52-bit limbs on the FP64 pipe
        ctx.set_wide_table(2)
        assert ctx.lookup_encrypt_ints(plain, pidx) == narrow
        ctx.set_fp64(1)

        # mode 1 (the default): a small call keeps the 8-bit table, a call of
        # 65,536 ciphertexts builds the wide one, with the same results
        ctx.build_tables(pk["g"], data["message_chunks"], noise)
        ctx.set_wide_table(1)
        vectors, embed = 1 << 16, 512
        bits = torch.from_numpy(np.random.default_rng(3).integers(0, 2, size=(vectors, embed), dtype=np.uint8)).cuda()
        nidx = torch.from_numpy(np.random.default_rng(4).integers(0, 256, size=(vectors, 14), dtype=np.uint8)).cuda()
        small = torch.empty((64, ctx.words), dtype=torch.int32, device="cuda")
        ctx.lookup_encrypt_bits_array(bits[:64], 64, embed, 2 * data["key_len"], 1, nidx[:64], small)
        torch.cuda.synchronize()
        assert not ctx.wide_table_ready()
        big = torch.empty((vectors, ctx.words), dtype=torch.int32, device="cuda")
        ctx.lookup_encrypt_bits_array(bits, vectors, embed, 2 * data["key_len"], 1, nidx, big)
        torch.cuda.synchronize()
        assert ctx.wide_table_ready()
        assert torch.equal(big[:64], small)
        with pytest.raises(ValueError):
            ctx.set_wide_table(3)
    finally:
        ctx.close()


@pytest.mark.parametrize("fp64", [1, 0], ids=["fp64", "integer"])
def test_noise_index_beyond_a_short_noise_table_is_a_range_error(fp64):
    from cuhepy_b200.paillier.gpu import PaillierDevice

    data = load_golden("lookup_1024.json")
    pk = {k: hx(v) for k, v in data["pk"].items()}
    ctx = PaillierDevice(pk["n"])
    try:
        ctx.set_fp64(fp64)
        entries = 16
        noise = oracle.noise_table(pk["g"], pk["n"], [hx(r) for r in data["noise_exponents"][:entries]])
        ctx.build_tables(pk["g"], data["message_chunks"], noise)
        table = ctx.g_table()
        ms = [hx(c["m"]) for c in data["encrypt"][:4]]
        good = np.array([[(3 * i + k) % entries for k in range(14)] for i in range(len(ms))], dtype=np.uint8)
        want = [oracle.lookup_encrypt(m, pk, table, noise, list(good[i]), len(table)) for i, m in enumerate(ms)]
        bad = good.copy()
        bad[2, 5] = entries  # the first index past the table
        for wide in (0, 2):  # the 8-bit table, then the 16-bit-digit table
            ctx.set_wide_table(wide)
            assert ctx.lookup_encrypt_ints(ms, good) == want
            with pytest.raises(ValueError, match="noise index"):
                ctx.lookup_encrypt_ints(ms, bad)
            # the status is cleared and the context stays usable
            assert ctx.lookup_encrypt_ints(ms, good) == want
            assert ctx.wide_table_ready() == (wide == 2)
    finally:
        ctx.close()


def test_wide_table_at_n_squared_of_8192_bits():
    """n of 4096 bits (key_len 2048, 256 words, 160 limbs of 52 bits) with 9
    message digits (five 16-bit rows, the last one half empty), so that both
    tables stay small; Montgomery arithmetic needs only an odd n."""
    from cuhepy_b200.paillier.gpu import PaillierDevice

    rng = random.Random(8192)
    n = rng.getrandbits(4096) | (1 << 4095) | 1
    pk = {"n": n, "g": n + 1, "n_squared": n * n}
    ctx = PaillierDevice(n)
    try:
        assert ctx.words == 256
        chunks, entries = 9, 32
        noise = oracle.noise_table(pk["g"], n, [rng.getrandbits(256) for _ in range(entries)])
        ctx.build_tables(pk["g"], chunks, noise)
        table = ctx.g_table()
        plain = [rng.getrandbits(8 * chunks) for _ in range(20)] + [0, (1 << (8 * chunks)) - 1, 1 << (8 * chunks - 1)]
        idx = np.array([[rng.randrange(entries) for _ in range(14)] for _ in plain], dtype=np.uint8)
        want = [oracle.lookup_encrypt(m, pk, table, noise, list(idx[i]), len(table)) for i, m in enumerate(plain)]
        for fp64 in (1, 0):  # 52-bit limbs on the FP64 pipe (the default at this width), then words
            ctx.set_fp64(fp64)
            for wide in (0, 2):
                ctx.set_wide_table(wide)
                assert ctx.lookup_encrypt_ints(plain, idx) == want, (fp64, wide)
                assert ctx.wide_table_ready() == (wide == 2)
            ctx.set_wide_table(0)
        ctx.set_fp64(1)
    finally:
        ctx.close()
