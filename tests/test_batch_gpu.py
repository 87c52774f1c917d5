"""The batched uneven mix (cuhepy_b200.batch): Paillier exponentiations of
two widths and uneven sizes in persistent work-stealing launches, plus BFV
NTT / INTT batches at three degrees, captured in one CUDA graph; every
result equals one launch per operation and the oracle.  Integer work:
equality is exact."""

import random

import pytest

from conftest import hx, load_golden
from oracle import bfv as ob

pytestmark = pytest.mark.gpu


def _keys():
    from cuhepy_b200.paillier.gpu import PaillierDevice

    ctxs = []
    for name in ("paillier_512.json", "lookup_512.json", "paillier_1024.json"):
        n = hx(load_golden(name)["pk"]["n"])
        ctxs.append(PaillierDevice(n))
    return ctxs


def _bases(ctx, count, rng):
    import torch

    vals = [rng.randrange(ctx.n_squared) for _ in range(count)]
    return vals, torch.from_numpy(ctx.limbs(vals).view("int32")).cuda()


def _ring(n, limbs):
    from cuhepy_b200.bfv import _bfv_rns as m

    q = 1
    for p in ob.rns_primes(n, 60 * limbs):
        q *= p
    ring = m.create_ring(n, format(q, "x"), 30, True, True, 2)
    return ring, m.ring_info(ring)["primes"][:limbs]


def _planes(n, primes, count, seed):
    import numpy as np
    import torch

    rng = np.random.default_rng(seed)
    rows = [rng.integers(0, primes[b % len(primes)], size=n, dtype=np.uint64) for b in range(count)]
    return torch.from_numpy(np.stack(rows).view(np.int64)).cuda()


def test_mixed_graph_matches_plain_and_oracle():
    import numpy as np
    import torch

    from cuhepy_b200._limbs import from_limbs
    from cuhepy_b200.batch import MixedBatch

    rng = random.Random(21)
    ctxs = _keys()
    mb = MixedBatch()
    jobs = []
    for ctx, count, e in ((ctxs[0], 37, rng.getrandbits(2048)), (ctxs[1], 1000, rng.getrandbits(280)),
                          (ctxs[2], 513, rng.getrandbits(2048)), (ctxs[0], 5, 0), (ctxs[2], 9, 1),
                          (ctxs[1], 2, 3)):
        vals, bases = _bases(ctx, count, rng)
        jobs.append((ctx, vals, e, mb.add_modexp(ctx, bases, e)))
    rings = [_ring(4096, 2), _ring(8192, 3), _ring(16384, 8)]
    ntt_items = []
    for k, (ring, primes) in enumerate(rings):
        fwd = _planes(ring.n, primes, 2 * len(primes), 100 + k)
        inv = _planes(ring.n, primes, len(primes), 200 + k)
        mb.add_ntt(ring, fwd, len(primes), inverse=False)
        mb.add_ntt(ring, inv, len(primes), inverse=True)
        ntt_items.append((fwd, inv))
    widths = mb.widths()
    assert [w["words"] for w in widths] == [64, 128]
    assert sum(w["batches"] for w in widths) == len(jobs)
    mb.capture()
    mb.replay()
    mb.check()
    graph_out = [out.clone() for *_, out in jobs]
    graph_ntt = [(f.clone(), i.clone()) for f, i in ntt_items]
    for ctx, vals, e, out in jobs:
        got = from_limbs(out.cpu().numpy().view(np.uint32))
        sample = range(len(vals)) if len(vals) < 64 else random.Random(1).sample(range(len(vals)), 24)
        for i in sample:
            assert got[i] == pow(vals[i], e, ctx.n_squared)
    # the same work as one launch per operation
    mb.restore_ntt_inputs()
    for *_, out in jobs:
        out.zero_()
    mb.run_plain()
    torch.cuda.synchronize()
    for (*_, out), g in zip(jobs, graph_out):
        assert torch.equal(out, g)
    for (f, i), (gf, gi) in zip(ntt_items, graph_ntt):
        assert torch.equal(f, gf) and torch.equal(i, gi)
    # forward then inverse is the identity
    from cuhepy_b200.bfv import _bfv_rns as m

    mb.restore_ntt_inputs()
    for (ring, primes), (f, _) in zip(rings, ntt_items):
        orig = f.clone()
        m.ntt(ring, f, len(primes))
        m.ntt(ring, f, len(primes), inverse=True)
        torch.cuda.synchronize()
        assert torch.equal(f, orig)
    mb.close()


def test_ntt_launch_shapes_agree_and_match_the_oracle():
    import numpy as np
    import torch

    from cuhepy_b200.bfv import _bfv_rns as m

    ring, primes = _ring(4096, 2)
    base = _planes(4096, primes, 2, 7)
    ref = base.clone()
    m.ntt(ring, ref, 2)
    torch.cuda.synchronize()
    for threads in (128, 256, 512):
        for radix in (1, 2, 3, 4):
            for inverse in (False, True):
                x = base.clone()
                m.ntt(ring, x, 2, inverse=inverse, threads=threads, radix_log=radix)
                y = base.clone()
                m.ntt(ring, y, 2, inverse=inverse)
                torch.cuda.synchronize()
                assert torch.equal(x, y), (threads, radix, inverse)
    # the forward transform is a ring map: NTT(a * b mod X^N + 1) equals
    # NTT(a) * NTT(b) pointwise (checked at N = 256 against a schoolbook product)
    small, sp = _ring(256, 2)
    r = random.Random(11)
    for j, p in enumerate(sp):
        a = [r.randrange(p) for _ in range(256)]
        b = [r.randrange(p) for _ in range(256)]
        c = [0] * 256
        for i, ai in enumerate(a):
            for k, bk in enumerate(b):
                if i + k < 256:
                    c[i + k] += ai * bk
                else:
                    c[i + k - 256] -= ai * bk
        c = [v % p for v in c]
        rows = [a, b, c]
        planes = torch.from_numpy(np.array(rows, dtype=np.uint64).view(np.int64)).cuda()
        # plane b uses prime b % primes: put the three rows on prime j
        full = torch.zeros((3 * len(sp), 256), dtype=torch.int64, device="cuda")
        for k in range(3):
            full[k * len(sp) + j] = planes[k]
        m.ntt(small, full, len(sp))
        torch.cuda.synchronize()
        fa, fb, fc = ([int(v) for v in full[k * len(sp) + j].cpu().numpy().view(np.uint64)] for k in range(3))
        assert [x * y % p for x, y in zip(fa, fb)] == fc
    with pytest.raises(ValueError):
        m.ntt(ring, base.clone(), 2, threads=48)
    with pytest.raises(ValueError):
        m.ntt(ring, base.clone(), 99)


def test_autotune_keeps_results_and_range_errors_are_reported():
    import torch

    from cuhepy_b200.batch import MixedBatch

    rng = random.Random(3)
    ctxs = _keys()
    mb = MixedBatch()
    vals, bases = _bases(ctxs[0], 700, rng)
    e = rng.getrandbits(512)
    out = mb.add_modexp(ctxs[0], bases, e)
    ring, primes = _ring(8192, 3)
    planes = _planes(8192, primes, 6, 9)
    mb.add_ntt(ring, planes, 3)
    report = mb.autotune(reps=1)
    assert 64 in report["paillier"] and 8192 in report["ntt"]
    mb.replay()
    mb.check()
    want = out.clone()
    mb.restore_ntt_inputs()
    ntt_graph = None
    mb.replay()
    torch.cuda.synchronize()
    ntt_graph = planes.clone()
    out.zero_()
    mb.restore_ntt_inputs()
    mb.run_plain()
    torch.cuda.synchronize()
    assert torch.equal(out, want) and torch.equal(planes, ntt_graph)
    # a base >= n^2 is reported, not computed
    bad = MixedBatch()
    n2 = ctxs[0].n_squared
    big = torch.from_numpy(ctxs[0].limbs([n2 + 1 if (n2 + 1).bit_length() <= 32 * ctxs[0].words else n2]).view("int32")).cuda()
    bad.add_modexp(ctxs[0], big, 3)
    bad.replay()
    with pytest.raises(ValueError):
        bad.check()


def test_graph_replays_repeat_identically():
    """Three widths on forked streams inside one graph: every replay gives
    the same exponentiations, and the in-place NTT batches, restored between
    replays, the same transforms."""
    import torch

    from cuhepy_b200.batch import MixedBatch
    from cuhepy_b200.paillier.gpu import PaillierDevice

    rng = random.Random(17)
    ctxs = _keys()
    n8192 = (1 << 4095) + 2 * rng.getrandbits(4000) + 1  # odd modulus of the 8192-bit n^2 width
    ctxs.append(PaillierDevice(n8192))
    mb = MixedBatch()
    outs = []
    for ctx, count, bits in ((ctxs[0], 900, 1024), (ctxs[2], 300, 2048), (ctxs[3], 40, 4096), (ctxs[1], 77, 280)):
        _, bases = _bases(ctx, count, rng)
        outs.append(mb.add_modexp(ctx, bases, rng.getrandbits(bits)))
    ring, primes = _ring(8192, 3)
    planes = _planes(8192, primes, 6, 23)
    mb.add_ntt(ring, planes, 3)
    assert [w["words"] for w in mb.widths()] == [64, 128, 256]
    mb.capture()
    first = None
    for _ in range(4):
        for out in outs:
            out.zero_()
        mb.restore_ntt_inputs()
        mb.replay()
        mb.check()
        got = [out.clone() for out in outs] + [planes.clone()]
        if first is None:
            first = got
        else:
            assert all(torch.equal(a, b) for a, b in zip(got, first))
    assert all(int(out.abs().sum()) > 0 for out in outs)
    mb.close()


def test_ntt_extreme_values_round_trip_and_ring_map():
    """Planes of p - 1 everywhere (and alternating p - 1 / 0) drive the lazy
    forward butterflies to their bound: every degree's forward transform,
    at every radix that compiles, must invert exactly and, at N = 256, still
    be the ring map (NTT(a * b) = NTT(a) NTT(b) with a schoolbook product)."""
    import numpy as np
    import torch

    from cuhepy_b200.bfv import _bfv_rns as m

    for n in (8, 16, 64, 1024, 4096, 8192, 16384, 32768):
        ring, primes = _ring(n, 2)
        rows = []
        for b in range(4):
            p = primes[b % 2]
            if b < 2:
                rows.append([p - 1] * n)
            elif b == 2:
                rows.append([p - 1 if i % 2 == 0 else 0 for i in range(n)])
            else:
                rows.append([p - 1] * (n - 1) + [0])
        base = torch.from_numpy(np.array(rows, dtype=np.uint64).view(np.int64)).cuda()
        want = None
        for radix in ((1, 2, 3, 4) if n in (4096, 8192) else (0,)):
            x = base.clone()
            m.ntt(ring, x, 2, radix_log=radix)
            fwd = x.clone()
            m.ntt(ring, x, 2, inverse=True, radix_log=radix)
            torch.cuda.synchronize()
            assert torch.equal(x, base), (n, radix)
            vals = fwd.cpu().numpy().view(np.uint64)
            for b in range(4):
                assert int(vals[b].max()) < primes[b % 2], (n, radix, b)  # canonical outputs
            if want is None:
                want = fwd
            assert torch.equal(fwd, want), (n, radix)
    small, sp = _ring(256, 2)
    for j, p in enumerate(sp):
        a = [p - 1] * 256
        b = [p - 1 if i % 3 else 0 for i in range(256)]
        c = [0] * 256
        for i, ai in enumerate(a):
            for k, bk in enumerate(b):
                if i + k < 256:
                    c[i + k] += ai * bk
                else:
                    c[i + k - 256] -= ai * bk
        c = [v % p for v in c]
        full = torch.zeros((3 * len(sp), 256), dtype=torch.int64, device="cuda")
        for k, row in enumerate((a, b, c)):
            full[k * len(sp) + j] = torch.from_numpy(np.array(row, dtype=np.uint64).view(np.int64))
        m.ntt(small, full, len(sp))
        torch.cuda.synchronize()
        fa, fb, fc = ([int(v) for v in full[k * len(sp) + j].cpu().numpy().view(np.uint64)] for k in range(3))
        assert [x * y % p for x, y in zip(fa, fb)] == fc
