"""Decrypt / decode by the Chinese remainder theorem (k_modexp_crt).

With the factors of n installed, c^e mod n^2 is computed as c^e mod p^2 and
c^e mod q^2 and recombined; every result must equal the direct kernel's and
the oracle's, for ciphertexts and for arbitrary values below n^2 (zero,
multiples of p, p^2, q, n, ...).  Integer work: equality is exact.
"""

import random

import numpy as np
import pytest

from conftest import hx, load_golden
from oracle import paillier as oracle

pytestmark = pytest.mark.gpu


def _keys(data):
    pk = {k: hx(v) for k, v in data["pk"].items()}
    return pk, {"pk": pk, "sk": {k: hx(v) for k, v in data["sk"].items()}}


def _pair(n, secret, phi):
    """(direct context, CRT context) for the same key."""
    from cuhepy_b200._numbers import factors_from_phi
    from cuhepy_b200.paillier.gpu import PaillierDevice

    direct = PaillierDevice(n)
    direct.set_secret(*secret)
    crt = PaillierDevice(n)
    crt.set_secret(*secret)
    p, q = factors_from_phi(n, phi)
    crt.set_factors(p, q)
    assert crt.has_factors and not direct.has_factors
    return direct, crt, p, q


def _awkward(n, p, q, rng, count=48):
    """Values below n^2 that stress the recombination: zero, units, multiples
    of p, q, p^2, q^2 and n, the top of the range, and random values."""
    n2 = n * n
    vals = [0, 1, 2, n - 1, n, n + 1, p, q, p * p, q * q, p * p * q, q * q * p, n2 - 1, n2 - n, n2 - p, n2 - 2]
    vals += [p * rng.randrange(1, q * q) for _ in range(8)]
    vals += [q * q * rng.randrange(1, p * p) for _ in range(4)]
    vals += [rng.randrange(n2) for _ in range(count)]
    return [v for v in vals if 0 <= v < n2]


@pytest.mark.parametrize("name", ["paillier_512.json", "paillier_1024.json"])
def test_crt_textbook_golden_and_edges(name):
    data = load_golden(name)
    pk, keys = _keys(data)
    n = pk["n"]
    direct, crt, p, q = _pair(n, (keys["sk"]["phi"], keys["sk"]["inv"]), keys["sk"]["phi"])
    ms = [hx(c["m"]) for c in data["encrypt"]]
    cs = [hx(c["c"]) for c in data["encrypt"]]
    vals = _awkward(n, p, q, random.Random(3))
    want = [oracle.decrypt(c, keys) for c in vals]
    for tpi, w in crt.VARIANTS[crt.words]:
        crt.set_tuning(tpi, w)
        assert crt.decrypt(cs) == ms, (tpi, w)
        assert crt.decrypt(vals) == want, (tpi, w)
    assert direct.decrypt(vals) == want
    sums = crt.mulmod([cs[s["i"]] for s in data["add"]], [cs[s["j"]] for s in data["add"]])
    assert crt.decrypt(sums) == [hx(s["m"]) for s in data["add"]]


@pytest.mark.parametrize("name", ["lookup_512.json", "lookup_1024.json"])
def test_crt_lookup_golden_decode_and_edges(name):
    data = load_golden(name)
    pk, keys = _keys(data)
    n = pk["n"]
    direct, crt, p, q = _pair(n, (keys["sk"]["a"], keys["sk"]["g_a_inv"]), keys["sk"]["phi"])
    ms = [hx(c["m"]) for c in data["encrypt"]]
    cs = [hx(c["c"]) for c in data["encrypt"]]
    vals = _awkward(n, p, q, random.Random(4))
    want = [oracle.lookup_decrypt(c, keys) for c in vals]
    chunk_len = 2 * data["key_len"]
    pairs = data["hamming"]["pairs"] if data["hamming"] else []
    for tpi, w in crt.VARIANTS[crt.words]:
        crt.set_tuning(tpi, w)
        assert crt.decrypt(cs) == ms, (tpi, w)
        assert crt.decrypt(vals) == want, (tpi, w)
        if pairs:
            server = [[hx(pr["c"])] for pr in pairs]
            assert crt.decode_hamming(server, 1, chunk_len) == [pr["distance"] for pr in pairs], (tpi, w)
    # decode of arbitrary values: popcount of the even bits of the decrypted value
    rows = [[v] for v in vals]
    got = crt.decode_hamming(rows, 1, chunk_len)
    assert got == direct.decode_hamming(rows, 1, chunk_len)
    assert got == [oracle.decode_distance([m], data["key_len"]) for m in want]


def test_crt_matches_direct_on_a_large_device_batch():
    """A device-resident batch several waves deep, through the array API."""
    import torch

    data = load_golden("lookup_1024.json")
    pk, keys = _keys(data)
    n = pk["n"]
    direct, crt, p, q = _pair(n, (keys["sk"]["a"], keys["sk"]["g_a_inv"]), keys["sk"]["phi"])
    rng = random.Random(77)
    vals = _awkward(n, p, q, rng, count=6000)
    limbs = torch.from_numpy(crt.limbs(vals).view(np.int32)).cuda()
    out_a = torch.zeros((len(vals), crt.words), dtype=torch.int32, device="cuda")
    out_b = torch.zeros_like(out_a)
    crt.decrypt_array(limbs, out_a, len(vals))
    direct.decrypt_array(limbs, out_b, len(vals))
    torch.cuda.synchronize()
    assert torch.equal(out_a, out_b)
    sample = rng.sample(range(len(vals)), 64)
    got = out_a.cpu().numpy().view(np.uint32)
    from cuhepy_b200._limbs import from_limbs

    decoded = from_limbs(got[sample])
    assert decoded == [oracle.lookup_decrypt(vals[i], keys) for i in sample]


@pytest.mark.parametrize("name", ["paillier_512.json", "lookup_1024.json", "paillier_1024.json"])
def test_fp64_pipe_equals_integer_pipe(name):
    """The exponentiations as 52-bit-limb products on the FP64 pipe give the
    integer-pipe kernels' results: by the CRT (decrypt and decode) and mod
    n^2 itself (decrypt and decode without the factors, encryption, public
    powers) and the server's products, on ciphertexts and on awkward values
    (several waves of a device batch)."""
    import torch

    data = load_golden(name)
    pk, keys = _keys(data)
    n = pk["n"]
    sk = keys["sk"]
    secret = (sk["a"], sk["g_a_inv"]) if "a" in sk else (sk["phi"], sk["inv"])
    _, crt, p, q = _pair(n, secret, sk["phi"])
    assert crt.fp64 == 1
    rng = random.Random(52)
    vals = _awkward(n, p, q, rng, count=3000)
    limbs = torch.from_numpy(crt.limbs(vals).view(np.int32)).cuda()
    outs, dists = [], []
    for fp64 in (2, 0):
        crt.set_fp64(fp64)
        assert crt.fp64 == fp64
        out = torch.zeros((len(vals), crt.words), dtype=torch.int32, device="cuda")
        dist = torch.full((len(vals) // 2,), -1, dtype=torch.int64, device="cuda")
        crt.decrypt_array(limbs, out, len(vals))
        crt.decode_array(limbs, len(vals) // 2, 2, 64, dist)
        crt.synchronize()
        outs.append(out)
        dists.append(dist)
    crt.set_fp64(1)
    assert torch.equal(outs[0], outs[1]) and torch.equal(dists[0], dists[1])
    from cuhepy_b200._limbs import from_limbs

    sample = rng.sample(range(len(vals)), 40)
    decrypt = oracle.lookup_decrypt if "a" in sk else oracle.decrypt
    assert from_limbs(outs[0].cpu().numpy().view(np.uint32)[sample]) == [decrypt(vals[i], keys) for i in sample]

    # the exponentiation mod n^2 itself (k_modexp52): decryption and decoding
    # without the factors, encryption r^n (1 + m n), public powers
    direct = _pair(n, secret, sk["phi"])[0]
    n2 = n * n
    ms = [rng.randrange(n) for _ in range(700)] + [0, 1, n - 1]
    rs = [rng.randrange(1, n) for _ in range(len(ms))]
    exps = [0, 1, 2, 3, n, rng.getrandbits(300), rng.getrandbits(2 * n.bit_length())]
    bases = [rng.randrange(n2) for _ in range(300)] + [0, 1, n2 - 1]
    # encode_hamming_server products: a device batch, and a host output
    # large enough for the piecewise download
    queries = [rng.randrange(n2) for _ in range(5)] + [0, 1, n2 - 1]
    qx = torch.from_numpy(direct.limbs(queries).view(np.int32)).cuda()
    big_q = 2 + (64 << 20) // (len(vals) * direct.words * 4)
    bq = np.ascontiguousarray(np.repeat(direct.limbs(queries[:1]), big_q, axis=0))
    got = []
    for fp64 in (2, 0):
        direct.set_fp64(fp64)
        out = torch.zeros((len(vals), direct.words), dtype=torch.int32, device="cuda")
        dist = torch.full((len(vals) // 2,), -1, dtype=torch.int64, device="cuda")
        outer = torch.zeros((len(queries) * len(vals), direct.words), dtype=torch.int32, device="cuda")
        direct.decrypt_array(limbs, out, len(vals))
        direct.decode_array(limbs, len(vals) // 2, 2, 64, dist)
        direct.mulmod_outer_array(qx, len(queries), limbs, len(vals), outer)
        direct.synchronize()
        host_out = np.zeros((big_q * len(vals), direct.words), dtype=np.uint32)
        direct.mulmod_outer_array(bq, big_q, direct.limbs(vals), len(vals), host_out)
        got.append((out, dist, direct.encrypt(ms, rs), [direct.modexp(bases, e) for e in exps], outer, host_out))
    direct.set_fp64(1)
    (o2, d2, c2, p2, x2, h2), (o0, d0, c0, p0, x0, h0) = got
    assert torch.equal(o2, o0) and torch.equal(d2, d0) and torch.equal(o2, outs[0])
    assert c2 == c0 and p2 == p0
    assert torch.equal(x2, x0) and np.array_equal(h2, h0)
    xs = from_limbs(x2.cpu().numpy().view(np.uint32))
    for qi in (0, len(queries) - 1):
        for k in (0, 9, len(vals) - 1):
            assert xs[qi * len(vals) + k] == queries[qi] * vals[k] % n2
    assert from_limbs(h2[:3]) == [queries[0] * v % n2 for v in vals[:3]]
    for k in (0, 5, len(ms) - 1):
        assert c2[k] == (1 + ms[k] * n) * pow(rs[k], n, n2) % n2
    for e, row in zip(exps, p2):
        assert [row[k] for k in (0, 7, len(bases) - 1)] == [pow(bases[k], e, n2) for k in (0, 7, len(bases) - 1)]


def test_crt_8192_bit_modulus_vs_oracle():
    rng = random.Random(4096)
    from oracle.gmp import powmod

    def is_prime(x):
        if x % 2 == 0:
            return False
        d, s = x - 1, 0
        while d % 2 == 0:
            d //= 2
            s += 1
        for _ in range(20):
            a = rng.randrange(2, x - 1)
            y = powmod(a, d, x)
            if y in (1, x - 1):
                continue
            for _ in range(s - 1):
                y = y * y % x
                if y == x - 1:
                    break
            else:
                return False
        return True

    def get_prime(bits):
        while True:
            c = rng.getrandbits(bits) | (1 << (bits - 1)) | 1
            if all(c % s for s in (3, 5, 7, 11, 13, 17, 19, 23)) and is_prime(c):
                return c

    p, q = get_prime(2048), get_prime(2048)
    keys = oracle.keys_from_primes(p, q)
    pk = keys["pk"]
    direct, crt, _, _ = _pair(pk["n"], (keys["sk"]["phi"], keys["sk"]["inv"]), keys["sk"]["phi"])
    assert crt.words == 256
    ms = [rng.randrange(pk["n"]) for _ in range(8)]
    cs = [oracle.encrypt(m, rng.randrange(1, pk["n"]), pk) for m in ms]
    vals = _awkward(pk["n"], p, q, rng, count=4)
    want = [oracle.decrypt(c, keys) for c in vals]
    for tpi, w in crt.VARIANTS[256]:
        crt.set_tuning(tpi, w)
        assert crt.decrypt(cs) == ms, (tpi, w)
        assert crt.decrypt(vals) == want, (tpi, w)


def test_set_factors_rejects_bad_factorisations_and_can_be_removed():
    from cuhepy_b200.paillier.gpu import PaillierDevice

    data = load_golden("paillier_512.json")
    pk, keys = _keys(data)
    n = pk["n"]
    from cuhepy_b200._numbers import factors_from_phi

    p, q = factors_from_phi(n, keys["sk"]["phi"])
    ctx = PaillierDevice(n)
    ctx.set_secret(keys["sk"]["phi"], keys["sk"]["inv"])
    with pytest.raises(ValueError):
        ctx.set_factors(p + 2, q)          # p * q != n
    with pytest.raises(ValueError):
        ctx.set_factors(1, n)              # unit factor
    assert not ctx.has_factors
    ctx.set_factors(q, p)                  # either order
    assert ctx.has_factors
    c = hx(data["encrypt"][1]["c"])
    assert ctx.decrypt([c]) == [hx(data["encrypt"][1]["m"])]
    ctx.set_factors(None, None)
    assert not ctx.has_factors
    assert ctx.decrypt([c]) == [hx(data["encrypt"][1]["m"])]
    # unbalanced factors (p^2 wider than half of n^2) stay on the direct kernel
    small, big = 1000003, (1 << 1000) + 1  # set_factors checks the product, not primality
    lop = PaillierDevice(small * big)
    with pytest.raises(ValueError):
        lop.set_factors(small, big)
    assert not lop.has_factors


def test_reference_facing_apis_install_factors_from_phi():
    from cuhepy_b200.paillier import lookup, scheme
    from cuhepy_b200.paillier.gpu import device_for

    data = load_golden("paillier_512.json")
    _, keys = _keys(data)
    c, m = hx(data["encrypt"][0]["c"]), hx(data["encrypt"][0]["m"])
    assert scheme.Paillier.decrypt(c, keys) == m
    sk = keys["sk"]
    assert device_for(keys["pk"]["n"], (sk["phi"], sk["inv"]), phi=sk["phi"]).has_factors
    data = load_golden("lookup_512.json")
    _, keys = _keys(data)
    c, m = hx(data["encrypt"][0]["c"]), hx(data["encrypt"][0]["m"])
    assert lookup.PaillierLookup.decrypt(c, keys) == m
    sk = keys["sk"]
    assert device_for(keys["pk"]["n"], (sk["a"], sk["g_a_inv"]), phi=sk["phi"]).has_factors


def test_static_decode_with_factors_matches_allocating_decode():
    import torch

    from cuhepy_b200 import _native

    data = load_golden("lookup_512.json")
    pk, keys = _keys(data)
    direct, crt, _, _ = _pair(pk["n"], (keys["sk"]["a"], keys["sk"]["g_a_inv"]), keys["sk"]["phi"])
    rng = random.Random(12)
    vectors, chunk_num, chunk_len = 200, 3, 2 * data["key_len"]
    vals = [rng.randrange(pk["n_squared"]) for _ in range(vectors * chunk_num)]
    c = torch.from_numpy(crt.limbs(vals).view(np.int32)).cuda()
    a = torch.zeros(vectors, dtype=torch.int64, device="cuda")
    b = torch.zeros_like(a)
    crt.decode_array(c, vectors, chunk_num, chunk_len, a)
    lib = _native.paillier_lib()
    rc = lib.cuhe_paillier_decode_hamming_static(crt._ctx, c.data_ptr(), vectors, chunk_num, chunk_len, b.data_ptr())
    assert rc == 0
    torch.cuda.synchronize()
    assert torch.equal(a, b)
    rows = [vals[chunk_num * i:chunk_num * i + chunk_num] for i in range(vectors)]
    want = np.array(direct.decode_hamming(rows, chunk_num, chunk_len))
    assert np.array_equal(a.cpu().numpy(), want)


def test_host_buffer_pipelines_match_device_buffers():
    """Host inputs of decode and host outputs of mulmod_outer above 64 MiB
    move piece by piece beside the compute (copy and side streams); the
    results equal the same calls on device buffers, from pageable and from
    pinned host memory."""
    import torch

    data = load_golden("lookup_1024.json")
    pk, keys = _keys(data)
    _, crt, _, _ = _pair(pk["n"], (keys["sk"]["a"], keys["sk"]["g_a_inv"]), keys["sk"]["phi"])
    rng = np.random.default_rng(64)

    def below_n2(count):
        # a zero top word keeps every value below n^2 (a 4096-bit modulus)
        x = rng.integers(0, 2**32, size=(count, crt.words), dtype=np.uint64).astype(np.uint32)
        x[:, -1] = 0
        return x

    vectors, chunk_num, chunk_len = 70_001, 2, 2 * data["key_len"]
    c_host = below_n2(vectors * chunk_num)
    assert c_host.nbytes >= 64 << 20
    want = torch.zeros(vectors, dtype=torch.int64, device="cuda")
    crt.decode_array(torch.from_numpy(c_host.view(np.int32)).cuda(), vectors, chunk_num, chunk_len, want)
    torch.cuda.synchronize()
    want = want.cpu().numpy()
    got = np.zeros(vectors, dtype=np.int64)
    crt.decode_array(c_host, vectors, chunk_num, chunk_len, got)
    assert np.array_equal(got, want)
    pinned = torch.from_numpy(c_host.view(np.int32)).pin_memory()
    got_pinned = torch.zeros(vectors, dtype=torch.int64).pin_memory()
    crt.decode_array(pinned.numpy(), vectors, chunk_num, chunk_len, got_pinned.numpy())
    assert np.array_equal(got_pinned.numpy(), want)

    nq, nx = 3, 44_000
    q_host, x_host = below_n2(nq), below_n2(nx)
    dev = torch.zeros((nq * nx, crt.words), dtype=torch.int32, device="cuda")
    crt.mulmod_outer_array(torch.from_numpy(q_host.view(np.int32)).cuda(), nq,
                           torch.from_numpy(x_host.view(np.int32)).cuda(), nx, dev)
    torch.cuda.synchronize()
    out = np.zeros((nq * nx, crt.words), dtype=np.uint32)
    assert out.nbytes >= 64 << 20
    crt.mulmod_outer_array(q_host, nq, x_host, nx, out)
    assert np.array_equal(out.view(np.int32), dev.cpu().numpy())
