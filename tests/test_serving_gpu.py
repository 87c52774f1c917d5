"""The served evaluator (cuhepy_b200.serving) on the GPU: every answer is the
same alone and in a mix of concurrent Paillier-Lookup and BFV requests,
including under a memory budget that forces queueing.  Integer work:
equality is exact."""

import random

import numpy as np
import pytest

from bfv_helpers import Seeded, key_bytes, packed, regenerate_fixture
from conftest import hx, load_golden
from oracle import bfv as ob
from oracle import paillier as oracle

pytestmark = pytest.mark.gpu


def _paillier_setup(vectors=1500, seed=3):
    import torch

    from cuhepy_b200.paillier.gpu import PaillierDevice

    data = load_golden("lookup_512.json")
    pk = {k: hx(v) for k, v in data["pk"].items()}
    keys = {"pk": pk, "sk": {k: hx(v) for k, v in data["sk"].items()}}
    key_len = data["key_len"]
    ctx = PaillierDevice(pk["n"])
    ctx.set_secret(keys["sk"]["a"], keys["sk"]["g_a_inv"])
    noise = oracle.noise_table(pk["g"], pk["n"], [hx(r) for r in data["noise_exponents"]])
    ctx.set_tables(oracle.g_table(pk["g"], pk["n"], key_len), noise)
    rng = np.random.default_rng(seed)
    embed = 512
    bits = rng.integers(0, 2, size=(vectors, embed), dtype=np.uint8)
    idx = rng.integers(0, 256, size=(vectors, 14), dtype=np.uint8)
    cts = torch.zeros((vectors, ctx.words), dtype=torch.int32, device="cuda")
    ctx.lookup_encrypt_bits_array(torch.from_numpy(bits).cuda(), vectors, embed, 2 * key_len, 1,
                                  torch.from_numpy(idx).cuda(), cts)
    torch.cuda.synchronize()
    return ctx, keys, key_len, bits, cts


def _queries(ctx, key_len, count, seed):
    import torch

    rng = np.random.default_rng(seed)
    bits = rng.integers(0, 2, size=(count, 512), dtype=np.uint8)
    idx = rng.integers(0, 256, size=(count, 14), dtype=np.uint8)
    out = torch.zeros((count, ctx.words), dtype=torch.int32, device="cuda")
    ctx.lookup_encrypt_bits_array(torch.from_numpy(bits).cuda(), count, 512, 2 * key_len, 1,
                                  torch.from_numpy(idx).cuda(), out)
    torch.cuda.synchronize()
    return bits, out.cpu()


def _bfv_setup():
    from cuhepy_b200.bfv import _bfv_rns as m

    data = load_golden("bfv_n256_q180_g30.json")
    params, layout, keys, query, index, vectors = regenerate_fixture(data)
    q, n = params.q, params.n
    ring = m.create_ring(n, format(q, "x"), params.gadget_bits, True, True, 2)
    relin = m.compile_key(ring, key_bytes(keys["relin"], q))
    exps = sorted(set(layout.left()) | set(layout.right()))
    galois = tuple((g, m.compile_key(ring, key_bytes(keys["galois"][g], q))) for g in exps)
    target = min(ob.coefficient_modulus(data["response_modulus_bits"]), q)
    server = m.create_server(relin, galois, layout.padded, params.t, format(target, "x"))
    bits = q.bit_length()
    ip = tuple((packed(c[0], bits), packed(c[1], bits)) for c in index)
    resident = m.upload_index(server, ip)
    rng = Seeded(99)
    queries = [(packed(query[0], bits), packed(query[1], bits))]
    r = random.Random(5)
    for _ in range(3):
        qb = [r.getrandbits(1) for _ in range(data["embed_len"])]
        ct = ob.encrypt(ob.batch_encode(layout.query_slots(qb), n, params.t), keys, rng)
        queries.append((packed(ct[0], bits), packed(ct[1], bits)))
    golden = next(v for k, v in data["results"].items() if k.endswith("compact"))
    width = (n * target.bit_length() + 7) // 8
    want0 = [(int(w[6], 16).to_bytes(width, "little"), int(w[7], 16).to_bytes(width, "little")) for w in golden]
    return m, server, resident, len(vectors), queries, want0


def test_served_answers_equal_alone_answers_in_a_mix():
    import torch

    from cuhepy_b200.serving import KnnEvaluator

    ctx, keys, key_len, index_bits, index_ct = _paillier_setup()
    m, server, resident, count, bfv_queries, want0 = _bfv_setup()
    V, K = index_ct.shape
    ev = KnnEvaluator(paillier_lanes=2, bfv_lanes=2, max_batch=16)
    ev.add_paillier_index("p512", keys["pk"]["n"], index_ct.view(V, 1, K))
    ev.add_bfv_index("b256", server, resident, count, compact=True)
    # budget for about two 8-query answers at once: forces admission waits
    budget = 2 * ev.paillier_answer_bytes("p512", 8) + 1
    ev._budget_override = budget
    sizes = [1, 5, 8, 2, 3, 7, 1, 4]
    qsets = [_queries(ctx, key_len, b, 100 + i) for i, b in enumerate(sizes)]
    alone_p = [ev.run_plain("paillier", "p512", q.view(b, 1, K)) for (_, q), b in zip(qsets, sizes)]
    alone_b = [ev.run_plain("bfv", "b256", q) for q in bfv_queries]
    assert alone_b[0] == want0
    ev.start()
    try:
        futs = []
        for i, (_, q) in enumerate(qsets):
            futs.append(("p", i, ev.submit_paillier("p512", q.view(sizes[i], 1, K))))
            if i < len(bfv_queries):
                futs.append(("b", i, ev.submit_bfv("b256", bfv_queries[i])))
        for kind, i, f in futs:
            got = f.result(120)
            if kind == "b":
                assert got == alone_b[i], i
            else:
                assert torch.equal(got.tensor, alone_p[i]), i
                if i == 0:
                    # decode one query's row against the oracle
                    row = got.tensor[0, 0, :64].contiguous()
                    dist = torch.zeros(64, dtype=torch.int64, device="cuda")
                    ctx.decode_array(row, 64, 1, 2 * key_len, dist)
                    torch.cuda.synchronize()
                    limbs = row.cpu().numpy().view(np.uint32)
                    from cuhepy_b200._limbs import from_limbs

                    want = [oracle.decode_distance([oracle.lookup_decrypt(c, keys)], key_len)
                            for c in from_limbs(limbs)]
                    assert dist.cpu().tolist() == want
                got.release()
        sched = ev.scheduler
        assert sched.peak_in_use <= budget
        assert sched.in_use == 0
        assert sched.launches < len(futs)          # some Paillier requests were merged
    finally:
        ev.stop()


def test_oversize_paillier_request_is_refused():
    from cuhepy_b200.serving import KnnEvaluator

    ctx, keys, key_len, _, index_ct = _paillier_setup(vectors=64)
    V, K = index_ct.shape
    ev = KnnEvaluator(paillier_lanes=1, bfv_lanes=1, max_batch=8, budget_bytes=ev_bytes(V, K, 2))
    ev.add_paillier_index("p", keys["pk"]["n"], index_ct.view(V, 1, K))
    ev.start()
    try:
        _, q = _queries(ctx, key_len, 3, 1)
        with pytest.raises(MemoryError):
            ev.submit_paillier("p", q.view(3, 1, K))
        _, q2 = _queries(ctx, key_len, 2, 2)
        ans = ev.submit_paillier("p", q2.view(2, 1, K)).result(60)
        import torch

        assert torch.equal(ans.tensor, ev.run_plain("paillier", "p", q2.view(2, 1, K)))
        ans.release()
    finally:
        ev.stop()


def ev_bytes(vectors, words, queries):
    return vectors * words * 4 * queries
