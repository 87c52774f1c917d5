"""Host-side number theory of the package (no GPU)."""

import random

from conftest import hx, load_golden


def test_factors_from_phi_recovers_the_golden_primes():
    from cuhepy_b200._numbers import factors_from_phi

    for name in ("paillier_512.json", "paillier_1024.json", "lookup_512.json", "lookup_1024.json"):
        data = load_golden(name)
        n, phi = hx(data["pk"]["n"]), hx(data["sk"]["phi"])
        p, q = factors_from_phi(n, phi)
        assert p * q == n and (p - 1) * (q - 1) == phi and 1 < p <= q, name


def test_factors_from_phi_rejects_inconsistent_pairs():
    from cuhepy_b200._numbers import factors_from_phi

    data = load_golden("paillier_512.json")
    n, phi = hx(data["pk"]["n"]), hx(data["sk"]["phi"])
    assert factors_from_phi(n, phi + 2) is None
    assert factors_from_phi(n, 0) is None
    rng = random.Random(1)
    for _ in range(20):
        assert factors_from_phi(n, rng.randrange(1, n)) is None
