"""Pin the CPU oracle to the golden vectors produced by the reference code."""

import numpy as np
import pytest

from conftest import hx, load_golden
from oracle import paillier as oracle


@pytest.mark.parametrize("name", ["paillier_512.json", "paillier_1024.json"])
def test_textbook_oracle_matches_reference(name):
    data = load_golden(name)
    pk = {k: hx(v) for k, v in data["pk"].items()}
    keys = {"pk": pk, "sk": {k: hx(v) for k, v in data["sk"].items()}}
    assert pk["g"] == pk["n"] + 1 and pk["n_squared"] == pk["n"] ** 2
    assert pk["n"].bit_length() == 2 * data["key_len"]
    for case in data["encrypt"]:
        m, r, c = hx(case["m"]), hx(case["r"]), hx(case["c"])
        assert oracle.encrypt(m, r, pk) == c
        assert oracle.decrypt(c, keys) == hx(case["d"]) == m
    for s in data["add"]:
        c1, c2 = hx(data["encrypt"][s["i"]]["c"]), hx(data["encrypt"][s["j"]]["c"])
        assert oracle.add(c1, c2, pk["n_squared"]) == hx(s["c"])
        assert oracle.decrypt(hx(s["c"]), keys) == hx(s["m"])


@pytest.mark.parametrize("name", ["lookup_512.json", "lookup_1024.json"])
def test_lookup_oracle_matches_reference(name):
    data = load_golden(name)
    pk = {k: hx(v) for k, v in data["pk"].items()}
    keys = {"pk": pk, "sk": {k: hx(v) for k, v in data["sk"].items()}}
    width = (pk["n_squared"].bit_length() + 7) // 8
    chunks = data["message_chunks"]
    assert chunks == oracle.message_chunks(data["key_len"])
    noise = oracle.noise_table(pk["g"], pk["n"], [hx(r) for r in data["noise_exponents"]])
    assert oracle.table_digest(noise, width) == data["noise_table_sha256"]
    table = oracle.g_table(pk["g"], pk["n"], data["key_len"])
    assert oracle.table_digest(table, width) == data["g_table_sha256"]
    for case in data["encrypt"]:
        m = hx(case["m"])
        c = oracle.lookup_encrypt(m, pk, table, noise, case["indices"], chunks)
        assert c == hx(case["c"])
        assert oracle.lookup_decrypt(c, keys) == hx(case["d"]) == m
    for s in data["add"]:
        c1, c2 = hx(data["encrypt"][s["i"]]["c"]), hx(data["encrypt"][s["j"]]["c"])
        assert oracle.add(c1, c2, pk["n_squared"]) == hx(s["c"])
        assert oracle.lookup_decrypt(hx(s["c"]), keys) == hx(s["m"])
    if data["hamming"]:
        vectors = data["hamming"]["vectors"]
        for v in vectors:
            bits = [int(b) for b in v["bits"]]
            (m,) = oracle.encode_bits(bits, data["key_len"])
            assert oracle.lookup_encrypt(m, pk, table, noise, v["indices"], chunks) == hx(v["c"][0])
        for p in data["hamming"]["pairs"]:
            d = oracle.lookup_decrypt(hx(p["c"]), keys)
            assert oracle.decode_distance([d], data["key_len"]) == p["distance"]
            a = np.array([int(b) for b in vectors[p["i"]]["bits"]])
            b = np.array([int(b) for b in vectors[p["j"]]["bits"]])
            assert p["distance"] == int((a != b).sum())


def test_oracle_rejects_out_of_range():
    data = load_golden("paillier_512.json")
    pk = {k: hx(v) for k, v in data["pk"].items()}
    keys = {"pk": pk, "sk": {k: hx(v) for k, v in data["sk"].items()}}
    with pytest.raises(ValueError):
        oracle.encrypt(pk["n"], 1, pk)
    with pytest.raises(ValueError):
        oracle.decrypt(pk["n_squared"], keys)
